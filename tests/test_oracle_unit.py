"""Unit checks of the oracle against independent numpy restatements."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from pscf_b200 import groups as G
from pscf_b200.system import chain_grid, make_unit_cell
from tests.cases import diblock, smooth_field

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("shape", [(32,), (30,), (27,), (20, 14), (15, 12), (16, 16, 16), (9, 10, 8), (7, 5, 6), (14, 6, 10)])
def test_fft_matches_numpy(shape):
    rng = np.random.default_rng(1)
    n = list(shape) + [1] * (3 - len(shape))
    f = rng.normal(size=(n[2], n[1], n[0]))
    spec = O.fft_r2c(f)
    ref = np.fft.rfftn(f, axes=(0, 1, 2))
    np.testing.assert_allclose(spec, ref, rtol=1e-13, atol=1e-12 * np.abs(ref).max())
    back = O.fft_c2r(ref, n[0])
    np.testing.assert_allclose(back, np.fft.irfftn(ref, s=(n[2], n[1], n[0]), axes=(0, 1, 2)) * f.size,
                               rtol=1e-12, atol=1e-11 * f.size)


def numpy_step(q, w, ksq, b, ds, shape):
    """Independent numpy restatement of step_exp (src/step_mod.f90:146-176)."""
    n3, n2, n1 = shape
    N = n1 * n2 * n3
    ksq = ksq.reshape(n3, n2, n1 // 2 + 1)
    q = q.reshape(shape)
    w = w.reshape(shape)
    eo1, eo2 = np.exp(-ds / 2 * w), np.exp(-ds / 4 * w)
    ek1, ek2 = np.exp(-ds * b * b / 6 * ksq), np.exp(-ds * b * b / 12 * ksq)
    F = lambda x: np.fft.rfftn(x, axes=(0, 1, 2))
    Fi = lambda X: np.fft.irfftn(X, s=shape, axes=(0, 1, 2)) * N
    q1 = eo1 * Fi(ek1 * F(eo1 * q)) / N
    qh = eo1 * Fi(ek2 * F(eo2 * q)) / N
    q2 = eo2 * Fi(ek2 * F(qh)) / N
    return ((4 * q2 - q1) / 3).ravel()


@pytest.mark.parametrize("dim,ngrid,crystal,cell", [
    (1, [32], "lamellar", [1.7]), (2, [24, 24], "hexagonal", [1.9]), (3, [12, 10, 8], "orthorhombic", [2.0, 2.5, 3.0])])
def test_step_matches_numpy(dim, ngrid, crystal, cell):
    s = diblock(dim, ngrid, crystal, cell)
    o = O.Oracle(s)
    ksq = o.ksq()
    w = 7.5 + smooth_field(s, 3, 2.0)
    q = 1.0 + 0.2 * smooth_field(s, 4, 1.0)
    n = s.n
    ref = numpy_step(q, w, ksq, 1.2, 0.01, (n[2], n[1], n[0]))
    got = O.step(s, ksq, 1.2, 0.01, w, q, 1)
    assert np.max(np.abs(got - ref)) < 1e-13 * np.max(np.abs(ref))


def test_uniform_field_known_answer():
    """omega = const -> q(s) = exp(-omega s), Q = exp(-omega N), rho_a = f_a."""
    s = diblock(3, [8, 8, 8], "cubic", [3.0], fA=0.3, chiN=10.0)
    o = O.Oracle(s)
    w = np.full((2, s.nr), 0.7)
    rho, q = o.density(w)
    assert abs(q[0] - np.exp(-0.7)) < 1e-13
    np.testing.assert_allclose(rho[0], 0.3, rtol=1e-13)
    np.testing.assert_allclose(rho[1], 0.7, rtol=1e-13)
    qf, qr = o.propagators(0)
    bgn, bds = chain_grid([0.3, 0.7], 0.01)
    svals = np.concatenate([[0.0], np.cumsum([bds[0]] * (bgn[1]) + [bds[1]] * (bgn[2] - bgn[1]))])
    np.testing.assert_allclose(qf[:, 0], np.exp(-0.7 * svals), rtol=1e-12)


@pytest.mark.parametrize("L,ds,steps", [(0.5, 0.01, 50), (0.25, 0.01, 26), (0.75, 0.01, 76), (0.39, 0.01, 40),
                                        (0.4, 0.005, 80), (0.6, 0.005, 120), (0.3, 0.005, 60), (0.001, 0.01, 2)])
def test_chain_grid_rule(L, ds, steps):
    """2*int(L/ds/2+0.5) steps per block, at least 2 (src/chain_mod.f90:140-157)."""
    bgn, bds = chain_grid([L], ds)
    assert bgn[-1] == steps
    assert abs(bds[0] * steps - L) < 1e-15
    b2 = np.zeros(2, np.int32)
    d2 = np.zeros(1)
    assert O.lib().orc_chain_grid(1, np.array([L]), ds, b2, d2) - 1 == steps


@pytest.mark.parametrize("dim,system,cp", [(1, "lamellar", [1.5]), (2, "square", [2.0]), (2, "rectangular", [2.0, 3.0]),
                                           (2, "hexagonal", [1.9]), (2, "oblique", [2.0, 2.5, 1.9]),
                                           (3, "cubic", [3.9]), (3, "tetragonal", [3.0, 4.0]),
                                           (3, "orthorhombic", [4.0, 8.0, 14.0]), (3, "hexagonal", [2.0, 3.0]),
                                           (3, "monoclinic", [2.0, 2.5, 3.0, 1.7])])
def test_unit_cell_host_matches_oracle(dim, system, cp):
    from pscf_b200.system import CRYSTAL_CODES
    G1, d1, n1 = make_unit_cell(dim, system, cp)
    G2, d2, n2 = O.unit_cell(dim, CRYSTAL_CODES[(dim, system)], cp)
    assert n1 == n2
    np.testing.assert_allclose(G1, G2, rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(d1, d2, rtol=1e-13, atol=1e-13)


def test_unit_cell_derivative_fd():
    """dGG(k) = d(b_i . b_j)/d cell_param_k by central differences."""
    for dim, system, cp in [(2, "hexagonal", [1.9]), (3, "orthorhombic", [4.0, 8.0, 14.0]),
                            (3, "monoclinic", [2.0, 2.5, 3.0, 1.7])]:
        G0, dGG, ncp = make_unit_cell(dim, system, cp)
        for k in range(ncp):
            h = 1e-6
            cpp = list(cp); cpp[k] += h
            cpm = list(cp); cpm[k] -= h
            Gp = make_unit_cell(dim, system, cpp)[0]
            Gm = make_unit_cell(dim, system, cpm)[0]
            fd = (Gp @ Gp.T - Gm @ Gm.T) / (2 * h)
            np.testing.assert_allclose(dGG[k], fd, rtol=1e-6, atol=1e-6)


def _ksq_bruteforce(dim, n, Gb):
    """Independent restatement of make_ksq / G_to_bz (src/grid_mod.f90:141-160, 225-283)."""
    n = list(n) + [1] * (3 - len(n))
    out = []
    rng = [range(1, -2, -1) if d < dim else [0] for d in range(3)]
    for i3 in range(n[2]):
        for i2 in range(n[1]):
            for i1 in range(n[0] // 2 + 1):
                best, bv = None, 1e10
                for a in rng[0]:
                    for b in rng[1]:
                        for c in rng[2]:
                            g = np.array([i1 + a * n[0], i2 + b * n[1], i3 + c * n[2]])[:dim]
                            v = g @ Gb[:dim, :dim]
                            q = float(v @ v)
                            if q < bv - 1e-8:
                                best, bv = g, q
                out.append(bv)
    return np.array(out)


@pytest.mark.parametrize("dim,ngrid,system,cp", [(2, [12, 12], "hexagonal", [1.9]), (2, [10, 6], "oblique", [2.0, 2.5, 1.9]),
                                                 (3, [6, 6, 4], "hexagonal", [2.0, 3.0]), (3, [8, 6, 4], "orthorhombic", [1., 2., 3.])])
def test_ksq_matches_bruteforce(dim, ngrid, system, cp):
    Gb = make_unit_cell(dim, system, cp)[0]
    got = O.make_ksq(dim, ngrid, Gb)
    np.testing.assert_allclose(got, _ksq_bruteforce(dim, ngrid, Gb), rtol=1e-14, atol=1e-13)


def test_groups_match_reference_tables():
    from fractions import Fraction as Fr
    g = json.load(open(os.path.join(HERE, "golden", "golden.json")))["groups"]
    for name, ref in g.items():
        mine = G.group(name)
        d = len(mine[0][0])
        refset = {(tuple(tuple(r["m"][i][:d]) for i in range(d)), tuple(Fr(x) % 1 for x in r["v"][:d])) for r in ref}
        assert set(mine) == refset, name


def test_symmetrize_projection():
    s = diblock(3, [8, 8, 8], "cubic", [3.0])
    f = smooth_field(s, 7, 1.0) + np.random.default_rng(0).normal(size=s.nr)
    p1 = G.symmetrize(f, "I m -3 m", [8, 8, 8])
    p2 = G.symmetrize(p1, "I m -3 m", [8, 8, 8])
    np.testing.assert_allclose(p1, p2, atol=1e-14)
    o = O.Oracle(s)
    M, t = G.grid_ops("I m -3 m", [8, 8, 8])
    o.set_symmetry(M, t)
    np.testing.assert_allclose(o.symmetrize(f), p1, atol=1e-14)
    with pytest.raises(ValueError):
        G.grid_ops("I a -3 d", [6, 6, 6])  # 1/4 translations need n divisible by 4
