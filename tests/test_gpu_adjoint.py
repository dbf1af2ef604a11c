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


def test_gyroid_64_loss_gradients():
    """The gyroid workload (I a -3 d, 64^3, a = 3.7, f_A = 0.40, chi N = 16,
    ds = 0.005, FP64 forward): L = sum_r (phi_A - phi_target)^2 with a seeded
    smooth target (+-0.1 around f_A).  The fields are the workload's
    parametrisation omega_A = chiN phi_B + delta, omega_B = chiN phi_A - delta
    with delta the gyroid level-set profile plus noise, projected onto
    I a -3 d.  Gradients through torch.autograd (the adjoint) against
    central differences with h = 1e-6 (relative) for a, to 1e-6 relative;
    dL/dchi N is zero (see below); for omega at single grid points the
    five-point stencil with h = 1e-3 (relative), to 1e-6 relative: the loss
    change a one-point step causes is small against the densities' roundoff
    (about 1e-13 relative per point, summed over 64^3 points), so smaller
    steps measure that roundoff (1e-5: differences of 4e-6 relative), and
    the stencil keeps the truncation at O(h^4).  Loss differences are summed
    from the density difference, L(1) - L(2) = sum (phi1 - phi2)(phi1 + phi2
    - 2 phi_target), which keeps the roundoff of the two large sums out of
    the difference."""
    import torch
    from pscf_b200 import groups
    from pscf_b200.autograd import density
    s = diblock(3, [64, 64, 64], "cubic", [3.7], fA=0.40, chiN=16.0, ds=0.005)
    n = 64
    x = 2 * np.pi * np.arange(n) / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    Gy = (np.sin(X) * np.cos(Y) + np.sin(Y) * np.cos(Z) + np.sin(Z) * np.cos(X)).ravel()
    rng = np.random.default_rng(20261203 + 3)
    delta = -(np.abs(Gy) - np.abs(Gy).mean()) + rng.normal(0, 0.01, s.nr)
    delta = groups.symmetrize(delta, "I a -3 d", [n, n, n])
    phi = s.phi_monomer()
    # target: Gaussian-filtered N(0,1) (sigma = 2 cells), scaled to +-0.1 around f_A
    k = np.fft.fftfreq(n) * n
    KZ, KY, KX = np.meshgrid(k, k, k, indexing="ij")
    filt = np.exp(-0.5 * (2.0 * 2 * np.pi / n) ** 2 * (KX ** 2 + KY ** 2 + KZ ** 2))
    t = np.real(np.fft.ifftn(np.fft.fftn(rng.normal(size=(n, n, n))) * filt)).ravel()
    target = 0.40 + 0.1 * t / np.max(np.abs(t))
    e = Engine([s], FP64)

    def omega(chi):
        return np.stack([chi * phi[1] + delta, chi * phi[0] - delta])

    def phi_a(wv, a):
        e.set_cell_param(0, [a])
        rho, _ = e.density(wv[None])
        return rho[0, 0].copy()

    def dL(p1, p2):
        return float(((p1 - p2) * (p1 + p2 - 2.0 * target)).sum())

    chi_t = torch.tensor(16.0, dtype=torch.float64, requires_grad=True)
    d_t = torch.from_numpy(delta)
    wt = torch.stack([chi_t * phi[1] + d_t, chi_t * phi[0] - d_t])[None]
    wt.retain_grad()
    cell = torch.tensor([[3.7]], dtype=torch.float64, requires_grad=True)
    rho, _ = density(wt, e, cell)
    L = ((rho[0, 0] - torch.from_numpy(target)) ** 2).sum()
    L.backward()
    gw = wt.grad.numpy()[0]
    w = omega(16.0)
    ha = 1e-6 * 3.7
    fd_a = dL(phi_a(w, 3.7 + ha), phi_a(w, 3.7 - ha)) / (2 * ha)
    assert abs(fd_a - cell.grad.item()) < 1e-6 * abs(fd_a), (fd_a, cell.grad.item())
    # chi N enters omega as a uniform shift of each species' field, which
    # multiplies qf qr and Q by the same constant: phi, hence L, does not
    # depend on it.  The adjoint gives that zero (the per-species sums of
    # dL/domega vanish) and the central difference agrees within its noise.
    hc = 1e-6 * 16.0
    fd_chi = dL(phi_a(omega(16.0 + hc), 3.7), phi_a(omega(16.0 - hc), 3.7)) / (2 * hc)
    assert abs(chi_t.grad.item()) < 1e-10 * abs(fd_a), (chi_t.grad.item(), fd_a)
    assert abs(fd_chi) < 1e-6 * abs(fd_a), (fd_chi, fd_a)
    for m, r in [(0, 0), (1, 12345), (0, 200000), (1, 77777)]:
        hw = 1e-3 * abs(w[m, r])

        def at(k):
            wk = w.copy()
            wk[m, r] += k * hw
            return phi_a(wk, 3.7)

        fd = (8.0 * dL(at(1), at(-1)) - dL(at(2), at(-2))) / (12.0 * hw)
        assert abs(fd - gw[m, r]) < 1e-6 * abs(fd), (m, r, fd, gw[m, r])
    e.close()
