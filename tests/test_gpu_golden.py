"""GPU engine vs the reference's golden outputs (through the C ABI)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from pscf_b200 import groups as G
from pscf_b200.engine import Engine, FP64
from tests.cases import diblock, lamellar_guess, omega_guess, rel_err, sphere_guess

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))


def test_lamellar_outfile_golden_gpu():
    g = GOLD["lamellar_outfile"]
    s = diblock(1, [32], "lamellar", g["cell_param"], fA=0.5, chiN=g["chi"][0])
    e = Engine([s])
    e.set_symmetry(0, "-1")
    w, rho, r = e.iterate_am(lamellar_guess(s)[None], error_max=1e-11, max_itr=500)
    r = r[0]
    assert r["converged"]
    for key, gk in [("f_helmholtz", "f_Helmholtz"), ("pressure", "pressure")]:
        assert abs(r[key] - g[gk][0]) < 1e-10, key
    assert abs(r["mu_chain"][0] - g["mu_chain"][0]) < 1e-10
    assert abs(r["stress"][0]) < 1e-10


def _bcc_systems(cells=None):
    out = []
    for i, g in enumerate(GOLD["bcc_sweep"]):
        cell = g["cell_param"] if cells is None else [cells[i]]
        out.append(diblock(3, [20, 20, 20], "cubic", cell, fA=g["block_length"][0], chiN=g["chi"][0]))
    return out


def test_bcc_sweep_golden_batched_gpu():
    """All 12 sweep points of the BCC fixture in one batched engine."""
    ss = _bcc_systems()
    e = Engine(ss)
    for i in range(len(ss)):
        e.set_symmetry(i, "I m -3 m")
    w0 = np.stack([sphere_guess(s, s.chains[0].block_length[0], width=0.05) for s in ss])
    w, rho, res = e.iterate_am(w0, error_max=1e-11, max_itr=800)
    for r, g in zip(res, GOLD["bcc_sweep"]):
        assert r["converged"]
        tol = 5e-11 + 2 * g["final_error"][0] + 1e-10
        assert abs(r["f_helmholtz"] - g["f_Helmholtz"][0]) < tol
        assert abs(r["mu_chain"][0] - g["mu_chain"][0]) < tol
        assert abs(r["pressure"] - g["pressure"][0]) < tol
        assert abs(r["stress"][0]) < 1e-9


def test_bcc_sweep_relaxed_cells_gpu():
    """Cell relaxation (stress -> 0) lands on the reference's relaxed cells."""
    ss = _bcc_systems([g["cell_param"][0] * 1.02 for g in GOLD["bcc_sweep"]])
    e = Engine(ss)
    for i in range(len(ss)):
        e.set_symmetry(i, "I m -3 m")
    w0 = np.stack([sphere_guess(s, s.chains[0].block_length[0], width=0.05) for s in ss])
    w, rho, res = e.iterate_am(w0, error_max=1e-11, max_itr=1500, domain=True)
    for r, g in zip(res, GOLD["bcc_sweep"]):
        assert r["converged"]
        assert abs(r["cell_param"][0] - g["cell_param"][0]) < 5e-10
        assert abs(r["f_helmholtz"] - g["f_Helmholtz"][0]) < 2e-10


@pytest.mark.parametrize("group,dim,ngrid,crystal,cell,fA", [
    ("I m -3 m", 3, [16, 16, 16], "cubic", [3.9], 0.25),
    ("p 6 m m", 2, [24, 24], "hexagonal", [1.9], 0.3),
    ("I a -3 d", 3, [16, 16, 16], "cubic", [3.7], 0.4),
    ("F d d d : 2", 3, [8, 16, 28], "orthorhombic", [1.0, 2.0, 3.5], 0.3),
])
def test_star_weighted_free_energy_and_stress_vs_oracle(group, dim, ngrid, crystal, cell, fA):
    s = diblock(dim, ngrid, crystal, cell, fA=fA, chiN=18.0)
    w = omega_guess(s, 17, 2.0)
    w = np.stack([G.symmetrize(w[a], group, ngrid) for a in range(2)])
    o = O.Oracle(s)
    M, t = G.grid_ops(group, ngrid)
    o.set_symmetry(M, t)
    rho_ref, q_ref = o.density(w)
    f_ref, p_ref = o.free_energy(w, rho_ref)
    st_ref = o.stress()
    e = Engine([s])
    e.set_symmetry(0, group)
    rho, q = e.density(w[None])
    assert rel_err(rho[0], rho_ref) < 1e-12
    st = e.scf_stress()[0, : len(st_ref)]
    np.testing.assert_allclose(st, st_ref, rtol=1e-10, atol=1e-12)
    f, p, mu = e.free_energy()
    assert abs(f[0] - f_ref) < 1e-11 and abs(p[0] - p_ref) < 1e-11


def test_symmetry_projection_keeps_symmetric_solution():
    """A symmetric initial field stays in the group's subspace during the solve."""
    s = diblock(3, [16, 16, 16], "cubic", [3.9], fA=0.25, chiN=20.0)
    e = Engine([s])
    e.set_symmetry(0, "I m -3 m")
    w0 = sphere_guess(s, 0.25, width=0.06)
    w, rho, r = e.iterate_am(w0[None], error_max=1e-9, max_itr=400)
    assert r[0]["converged"]
    for a in range(2):
        np.testing.assert_allclose(G.symmetrize(w[0, a], "I m -3 m", [16, 16, 16]), w[0, a], atol=1e-12)


def test_mixed_precision_matches_fp64_solution():
    """FP32 propagation until the residual nears the switch error (1e-3 by
    default), then FP64 to 1e-11: the converged free energy equals the FP64
    solve to 1e-10 per monomer."""
    from pscf_b200.engine import MIXED
    ss = _bcc_systems()[:4]
    w0 = np.stack([sphere_guess(s, s.chains[0].block_length[0], width=0.05) for s in ss])
    res = {}
    for prec in (FP64, MIXED):
        e = Engine(ss, prec)
        for i in range(len(ss)):
            e.set_symmetry(i, "I m -3 m")
        w, rho, r = e.iterate_am(w0, error_max=1e-11, max_itr=800)
        assert all(x["converged"] for x in r)
        res[prec] = r
    for a, b, g in zip(res[FP64], res[MIXED], GOLD["bcc_sweep"]):
        assert b["itr_fp32"] > 0
        assert abs(a["f_helmholtz"] - b["f_helmholtz"]) < 1e-10
        assert abs(b["f_helmholtz"] - g["f_Helmholtz"][0]) < 2e-10


@pytest.mark.parametrize("n_cut", [None, 100])
def test_newton_bcc_golden_batched_jacobian(n_cut):
    """iterate_NR on the engine: the 290 finite-difference Jacobian columns
    of the BCC fixture (146 stars) are one batched density call; with
    N_cut = 100 (the fixture's own setting) 198 columns are differenced and
    the 46 shortest-wavelength stars take the Debye tail."""
    from pscf_b200.basis import StarBasis
    from pscf_b200.newton import EngineProvider, iterate_nr
    g = GOLD["bcc_sweep"][0]
    s = diblock(3, [20, 20, 20], "cubic", g["cell_param"], fA=g["block_length"][0], chiN=g["chi"][0])
    basis = StarBasis("I m -3 m", [20, 20, 20])
    assert basis.n_star == int(g["N_star"][0])
    # start from a partly converged Anderson state, as the reference's
    # sweep starts from the previous point
    e = Engine([s])
    e.set_symmetry(0, "I m -3 m")
    w0, _, _ = e.iterate_am(sphere_guess(s, s.chains[0].block_length[0], width=0.05)[None], error_max=1e-3,
                            max_itr=200)
    prov = EngineProvider(s, "I m -3 m", max_batch=146)
    w, rho, r = iterate_nr(prov, basis, s, w0[0], error_max=1e-10, max_itr=40, n_cut=n_cut)
    assert r["converged"], r["error"]
    e.density(w[None])
    f, p, mu = e.free_energy()
    assert abs(f[0] - g["f_Helmholtz"][0]) < 2e-10
    assert abs(mu[0, 0] - g["mu_chain"][0]) < 2e-10


def test_mixed_shape_batches_concurrent():
    """Lamellae, cylinders and spheres as three engines driven concurrently
    give the same converged results as each solved on its own."""
    from pscf_b200 import guess
    from pscf_b200.batch import ShapeBatch, solve_batches
    lam = [diblock(1, [64], "lamellar", [1.7], fA=0.5, chiN=20.0), diblock(1, [64], "lamellar", [1.8], fA=0.45, chiN=22.0)]
    hexs = [diblock(2, [32, 32], "hexagonal", [1.9], fA=0.3, chiN=20.0)]
    bcc = [diblock(3, [16, 16, 16], "cubic", [1.95], fA=0.25, chiN=20.0)]
    mk = lambda: [ShapeBatch(lam, np.stack([guess.lamellar(s, s.chains[0].block_length[0]) for s in lam]), "-1"),
                  ShapeBatch(hexs, np.stack([guess.cylinders(s, 0.3) for s in hexs]), "p 6 m m"),
                  ShapeBatch(bcc, np.stack([guess.spheres_bcc(s, 0.25) for s in bcc]), "I m -3 m")]
    together = solve_batches(mk(), error_max=1e-9, max_itr=800, domain=True)
    alone = []
    for b in mk():
        _, _, r = b.engine.iterate_am(b.omega0, error_max=1e-9, max_itr=800, domain=True)
        alone.append(r)
    for rs1, rs2 in zip(together, alone):
        for r1, r2 in zip(rs1, rs2):
            assert r1["converged"] and r2["converged"]
            assert r1["f_helmholtz"] == r2["f_helmholtz"] and r1["itr"] == r2["itr"]
