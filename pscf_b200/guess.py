"""Seeded, phase-appropriate initial fields (host utility).

The reference reads its initial omega from a field file; these build the
equivalent starting fields for synthetic runs: a target A-monomer density
with sharp (tanh) domain boundaries around the sites of the phase, turned
into omega_A - omega_B = chi (1 - 2 rho_A) around the uniform values
chi . phi_mon (set_omega_uniform, src/scf_mod.fp.f90:724-750), plus seeded
Gaussian noise.
"""
from __future__ import annotations

import math

import numpy as np

BCC_SITES = [(0.0, 0.0, 0.0), (0.5, 0.5, 0.5)]
HEX_SITES = [(0.0, 0.0)]


def _bravais(system):
    dim = system.dim
    G, _, _ = system.unit_cell()
    return 2 * math.pi * np.linalg.inv(G[:dim, :dim]).T        # rows: Bravais vectors


def site_density(system, fA, sites, width=0.05):
    """rho_A = (1 - tanh((d - R)/w))/2, d the distance to the nearest site,
    R such that <rho_A> = fA, w = width * (cell volume)^(1/dim)."""
    n, dim = system.n, system.dim
    R = _bravais(system)
    axes = [np.arange(n[d]) / n[d] for d in range(dim)]
    grids = np.meshgrid(*axes[::-1], indexing="ij")[::-1]
    frac = np.stack([g.ravel() for g in grids], axis=1)
    dmin = np.full(frac.shape[0], np.inf)
    shifts = np.array(np.meshgrid(*[[-1, 0, 1]] * dim)).T.reshape(-1, dim)
    for c in sites:
        df = frac - np.array(c[:dim])
        df -= np.round(df)
        for sh in shifts:
            v = (df + sh) @ R
            dmin = np.minimum(dmin, np.sqrt((v * v).sum(axis=1)))
    scale = float(abs(np.linalg.det(R))) ** (1.0 / dim)
    w = width * scale
    lo, hi = 0.0, scale
    for _ in range(60):
        Rs = 0.5 * (lo + hi)
        m = np.mean(0.5 * (1 - np.tanh((dmin - Rs) / w)))
        lo, hi = (Rs, hi) if m < fA else (lo, Rs)
    return 0.5 * (1 - np.tanh((dmin - Rs) / w))


def omega_from_density(system, rho_a, noise=0.0, seed=0):
    chi = system.chi[0, 1]
    d = 0.5 * chi * (1.0 - 2.0 * rho_a)
    d -= d.mean()
    w0 = system.omega_uniform()
    rng = np.random.default_rng(seed)
    w = np.zeros((2, system.nr))
    w[0] = w0[0] + d + (rng.normal(0.0, noise, system.nr) if noise else 0.0)
    w[1] = w0[1] - d + (rng.normal(0.0, noise, system.nr) if noise else 0.0)
    return w


def lamellar(system, fA, noise=0.0, seed=0, width=0.05):
    """A layer of thickness fA d centred at x = 0."""
    n = system.n[0]
    x = np.arange(n) / n
    d = np.abs(x - np.round(x))
    L = fA / 2.0
    rho = 0.5 * (1 - np.tanh((d - L) / width))
    rho *= fA / rho.mean()
    return omega_from_density(system, np.clip(rho, 0, 1), noise, seed)


def cylinders(system, fA, noise=0.0, seed=0):
    return omega_from_density(system, site_density(system, fA, HEX_SITES), noise, seed)


def spheres_bcc(system, fA, noise=0.0, seed=0):
    return omega_from_density(system, site_density(system, fA, BCC_SITES), noise, seed)
