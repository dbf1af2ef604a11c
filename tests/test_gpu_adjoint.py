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
