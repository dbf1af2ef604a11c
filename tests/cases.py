"""Seeded SCFT systems and fields shared by the tests (small sizes)."""
import numpy as np

from pscf_b200.system import Chain, System


def diblock(dim, ngrid, crystal, cell, fA=0.5, chiN=15.0, ds=0.01, b=(1.0, 1.0)):
    return System(dim=dim, ngrid=list(ngrid), crystal_system=crystal, cell_param=list(cell),
                  kuhn=list(b), chi=[[0.0, chiN], [chiN, 0.0]],
                  chains=[Chain([0, 1], [fA, 1.0 - fA])], ds=ds)


def triblock(dim, ngrid, crystal, cell, f=(0.3, 0.4, 0.3), chi=(30.0, 30.0, 60.0), ds=0.01):
    cab, cbc, cac = chi
    X = [[0, cab, cac], [cab, 0, cbc], [cac, cbc, 0]]
    return System(dim=dim, ngrid=list(ngrid), crystal_system=crystal, cell_param=list(cell),
                  kuhn=[1.0, 1.0, 1.0], chi=X, chains=[Chain([0, 1, 2], list(f))], ds=ds)


def smooth_field(system, seed, amp=1.0, modes=3):
    """Seeded smooth real field (sum of a few low Fourier modes)."""
    rng = np.random.default_rng(seed)
    n = system.n
    x = [np.arange(n[d]) / n[d] for d in range(3)]
    Z, Y, X = np.meshgrid(x[2], x[1], x[0], indexing="ij")
    f = np.zeros((n[2], n[1], n[0]))
    for _ in range(modes):
        k = rng.integers(-2, 3, size=3)
        for d in range(system.dim, 3):
            k[d] = 0
        ph = rng.uniform(0, 2 * np.pi)
        f += rng.normal() * np.cos(2 * np.pi * (k[0] * X + k[1] * Y + k[2] * Z) + ph)
    return amp * f.ravel()


def omega_guess(system, seed, amp=2.0):
    """omega_a = chi.phi_mon + alternating smooth perturbation + seeded noise."""
    rng = np.random.default_rng(seed)
    w0 = system.omega_uniform()
    d = smooth_field(system, seed, amp)
    w = np.zeros((system.n_monomer, system.nr))
    sgn = [1.0, -1.0, 0.5, -0.5]
    for a in range(system.n_monomer):
        w[a] = w0[a] + sgn[a] * d + 0.01 * rng.normal(size=system.nr)
    return w


def lamellar_guess(system, amp=5.0):
    n = system.n[0]
    x = np.arange(n) / n
    w0 = system.omega_uniform()
    w = np.zeros((2, n))
    w[0] = w0[0] + amp * np.cos(2 * np.pi * x)
    w[1] = w0[1] - amp * np.cos(2 * np.pi * x)
    return w


def bcc_guess(system, amp=6.0, sigma=0.3):
    """Gaussian A-rich spheres at the BCC sites (0,0,0), (1/2,1/2,1/2)."""
    n = system.n
    x = [np.arange(n[d]) / n[d] for d in range(3)]
    Z, Y, X = np.meshgrid(x[2], x[1], x[0], indexing="ij")
    g = np.zeros_like(X)
    for c in [(0, 0, 0), (0.5, 0.5, 0.5)]:
        for sx in (-1, 0, 1):
            for sy in (-1, 0, 1):
                for sz in (-1, 0, 1):
                    dx, dy, dz = X - c[0] - sx, Y - c[1] - sy, Z - c[2] - sz
                    g += np.exp(-(dx * dx + dy * dy + dz * dz) / (2 * sigma * sigma))
    g = g / g.max()
    g -= g.mean()
    w0 = system.omega_uniform()
    w = np.zeros((2, system.nr))
    w[0] = w0[0] - amp * g.ravel()
    w[1] = w0[1] + amp * g.ravel()
    return w


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


from pscf_b200.guess import BCC_SITES, site_density, omega_from_density  # noqa: E402


def sphere_guess(system, fA, sites=BCC_SITES, width=0.08, chiN=None):
    """omega from tanh-edged spheres at `sites` (pscf_b200.guess)."""
    return omega_from_density(system, site_density(system, fA, sites, width))
