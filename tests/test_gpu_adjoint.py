"""Adjoint of density(): central finite differences and the reference's
own gradient relation dlnQ/domega_m(r) = -rho_m(r) N / (phi N_r) (the
Simpson contour integral approximates this derivative to O(ds^2))."""
import numpy as np
import pytest

from pscf_b200.engine import Engine, FP64
from tests.cases import diblock, omega_guess, triblock

pytestmark = pytest.mark.gpu

CASES = [
    (1, [16], "lamellar", [1.6]),
    (2, [12, 12], "hexagonal", [1.8]),
    (3, [8, 8, 8], "cubic", [2.0]),
    (3, [16, 16, 16], "cubic", [2.0]),
    (3, [6, 10, 8], "orthorhombic", [1.5, 2.0, 2.5]),
]


def _loss(e, w, c, a):
    rho, q = e.density(w[None])
    return float((c * rho[0]).sum() + (a * np.log(q[0, :len(a)])).sum())


@pytest.mark.parametrize("dim,ngrid,crystal,cell", CASES)
def test_adjoint_matches_central_differences(dim, ngrid, crystal, cell):
    s = diblock(dim, ngrid, crystal, cell, fA=0.35, chiN=14.0, ds=0.05)
    rng = np.random.default_rng(7)
    w = omega_guess(s, 3, 2.0)
    c = rng.normal(size=(2, s.nr))
    a = np.array([0.7])
    e = Engine([s], FP64)
    e.density(w[None])
    g = e.density_adjoint(c[None], a[None])[0]
    h = 1e-5
    for _ in range(6):
        m, r = int(rng.integers(2)), int(rng.integers(s.nr))
        wp, wm = w.copy(), w.copy()
        wp[m, r] += h
        wm[m, r] -= h
        fd = (_loss(e, wp, c, a) - _loss(e, wm, c, a)) / (2 * h)
        assert abs(fd - g[m, r]) < 1e-6 * max(1.0, abs(fd)), (m, r, fd, g[m, r])


def test_adjoint_multiblock_chain_and_lnq():
    s = triblock(2, [10, 12], "rectangular", [1.6, 2.0], ds=0.05)
    rng = np.random.default_rng(11)
    w = omega_guess(s, 5, 1.5)
    c = rng.normal(size=(3, s.nr))
    a = np.array([-1.3])
    e = Engine([s], FP64)
    e.density(w[None])
    g = e.density_adjoint(c[None], a[None])[0]
    h = 1e-5
    for _ in range(6):
        m, r = int(rng.integers(3)), int(rng.integers(s.nr))
        wp, wm = w.copy(), w.copy()
        wp[m, r] += h
        wm[m, r] -= h
        fd = (_loss(e, wp, c, a) - _loss(e, wm, c, a)) / (2 * h)
        assert abs(fd - g[m, r]) < 1e-6 * max(1.0, abs(fd))


def test_lnq_gradient_equals_minus_phi_over_v():
    s = diblock(3, [16, 16, 16], "cubic", [2.0], fA=0.3, chiN=16.0, ds=0.01)
    w = omega_guess(s, 9, 2.0)
    e = Engine([s], FP64)
    rho, q = e.density(w[None])
    g = e.density_adjoint(np.zeros((1, 2, s.nr)), np.array([[1.0]]))[0]
    expect = -rho[0] * s.chains[0].length / (s.chains[0].phi * s.nr)
    err = np.max(np.abs(g - expect)) / np.max(np.abs(expect))
    assert err < 1e-4, err


def test_torch_autograd_function():
    import torch
    from pscf_b200.autograd import density
    s = diblock(3, [8, 8, 8], "cubic", [2.0], fA=0.35, chiN=14.0, ds=0.05)
    w = torch.tensor(omega_guess(s, 3, 2.0)[None], dtype=torch.float64, device="cuda", requires_grad=True)
    target = torch.full((s.nr,), 0.35, dtype=torch.float64, device="cuda")
    e = Engine([s], FP64)
    rho, lnq = density(w, e)
    loss = ((rho[0, 0] - target) ** 2).sum() + lnq.sum()
    loss.backward()
    g_auto = w.grad.detach().cpu().numpy()[0]
    rho_np = rho.detach().cpu().numpy()[0]
    G = np.zeros((2, s.nr))
    G[0] = 2 * (rho_np[0] - 0.35)
    g_ref = e.density_adjoint(G[None], np.array([[1.0]]))[0]
    np.testing.assert_allclose(g_auto, g_ref, rtol=1e-12, atol=1e-14)


def _loss_cell(e, s, w, cp, c, a):
    e.set_cell_param(0, list(cp))
    return _loss(e, w, c, a)


@pytest.mark.parametrize("dim,ngrid,crystal,cell", CASES)
def test_cell_gradient_matches_central_differences(dim, ngrid, crystal, cell):
    """dL/dcell from the adjoint equals central differences of L(cell)
    (the exact derivative of the discrete algorithm)."""
    s = diblock(dim, ngrid, crystal, cell, fA=0.35, chiN=14.0, ds=0.05)
    rng = np.random.default_rng(11)
    w = omega_guess(s, 4, 2.0)
    c = rng.normal(size=(2, s.nr))
    a = np.array([0.6])
    e = Engine([s], FP64)
    e.density(w[None])
    _, gc = e.density_adjoint(c[None], a[None], want_cell=True)
    for b in range(len(cell)):
        h = 1e-5 * cell[b]
        cp, cm = list(cell), list(cell)
        cp[b] += h
        cm[b] -= h
        fd = (_loss_cell(e, s, w, cp, c, a) - _loss_cell(e, s, w, cm, c, a)) / (2 * h)
        assert abs(fd - gc[0, b]) < 1e-6 * max(1.0, abs(fd)), (b, fd, gc[0, b])
    e.close()


def test_cell_gradient_with_star_weights_and_stress_relation():
    """With a space group set (star weights on the stress) the cell gradient
    is still the exact derivative, and for L = lnQ it matches the
    reference's stress formula, stress = -(phi/N) dlnQ/dcell, to the contour
    discretisation error."""
    s = diblock(3, [16, 16, 16], "cubic", [1.95], fA=0.3, chiN=16.0, ds=0.01)
    w = omega_guess(s, 6, 2.0)
    from pscf_b200 import groups as Gr
    w = np.stack([Gr.symmetrize(w[m], "I m -3 m", s.ngrid) for m in range(2)])
    e = Engine([s], FP64)
    e.set_symmetry(0, "I m -3 m")
    e.density(w[None])
    stress = e.scf_stress()[0, 0]
    _, gc = e.density_adjoint(np.zeros((1, 2, s.nr)), np.array([[1.0]]), want_cell=True)
    h = 1e-5 * 1.95
    lq = []
    for cp in (1.95 + h, 1.95 - h):
        e.set_cell_param(0, [cp])
        _, q = e.density(w[None])
        lq.append(np.log(q[0, 0]))
    fd = (lq[0] - lq[1]) / (2 * h)
    assert abs(fd - gc[0, 0]) < 1e-7 * max(1.0, abs(fd))
    phi_over_n = s.chains[0].phi / s.chains[0].length
    assert abs(stress - (-phi_over_n * gc[0, 0])) < 1e-3 * abs(stress), (stress, -phi_over_n * gc[0, 0])
    e.close()


def test_torch_autograd_cell_input():
    import torch
    from pscf_b200.autograd import density
    s = diblock(2, [12, 12], "hexagonal", [1.8], fA=0.35, chiN=14.0, ds=0.05)
    w = torch.tensor(omega_guess(s, 3, 2.0)[None], dtype=torch.float64, requires_grad=True)
    cell = torch.tensor([[1.8]], dtype=torch.float64, requires_grad=True)
    e = Engine([s], FP64)
    rho, lnq = density(w, e, cell)
    loss = ((rho[0, 0] - 0.35) ** 2).sum() + lnq.sum()
    loss.backward()
    rho_np = rho.detach().numpy()[0]
    G = np.zeros((2, s.nr))
    G[0] = 2 * (rho_np[0] - 0.35)
    e.set_cell_param(0, [1.8])
    e.density(w.detach().numpy())
    g_ref, gc_ref = e.density_adjoint(G[None], np.array([[1.0]]), want_cell=True)
    np.testing.assert_allclose(w.grad.numpy()[0], g_ref[0], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(cell.grad.numpy(), gc_ref, rtol=1e-12)
