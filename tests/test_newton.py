"""Newton/Broyden iteration (iterate_NR restated) and the star basis.

The host logic runs here with the CPU oracle as the density provider; the
same loop drives the batched GPU engine in tests/test_gpu_golden.py."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from pscf_b200 import groups as G
from pscf_b200.basis import StarBasis
from pscf_b200.newton import iterate_nr
from tests.cases import diblock, lamellar_guess

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))


class OracleProvider:
    def __init__(self, system, group):
        self.o = O.Oracle(system)
        M, t = G.grid_ops(group, list(system.ngrid))
        self.o.set_symmetry(M, t)
        self.cell = list(system.cell_param)

    def __call__(self, omegas, cells=None, want_stress=False):
        B = omegas.shape[0]
        rho = np.zeros_like(omegas)
        q = np.zeros((B, 1))
        stress = np.zeros((B, len(self.cell))) if want_stress else None
        for b in range(B):
            c = list(cells[b]) if cells is not None else self.cell
            self.o.set_cell(c)
            rho[b], q[b] = self.o.density(omegas[b])
            if want_stress:
                stress[b] = self.o.stress()
        return dict(rho=rho, q=q, stress=stress)


@pytest.mark.parametrize("name,ngrid,nstar", [("-1", [32], 17), ("I m -3 m", [20, 20, 20], 146),
                                              ("p 6 m m", [24, 24], 61), ("I a -3 d", [16, 16, 16], 51)])
def test_star_basis_spans_symmetric_fields(name, ngrid, nstar):
    b = StarBasis(name, ngrid)
    if name in ("-1", "I m -3 m"):
        assert b.n_star == nstar          # N_star of the reference's fixtures
    f = G.symmetrize(np.random.default_rng(1).normal(size=int(np.prod(ngrid))), name, ngrid)
    np.testing.assert_allclose(b.to_grid(b.to_basis(f)), f, atol=1e-13)
    a = np.random.default_rng(2).normal(size=b.n_star)
    np.testing.assert_allclose(b.to_basis(b.to_grid(a)), a, atol=1e-12)


@pytest.mark.parametrize("domain", [False, True])
def test_newton_lamellar_golden(domain):
    g = GOLD["lamellar_outfile"]
    cell0 = g["cell_param"][0] * (1.03 if domain else 1.0)
    s = diblock(1, [32], "lamellar", [cell0], fA=0.5, chiN=g["chi"][0])
    basis = StarBasis("-1", [32])
    prov = OracleProvider(s, "-1")
    w, rho, r = iterate_nr(prov, basis, s, lamellar_guess(s), error_max=1e-11, max_itr=60, domain=domain)
    assert r["converged"]
    o = prov.o
    o.set_cell(r["cell_param"])
    rr, q = o.density(w)
    f, p = o.free_energy(w, rr)
    mu, _ = o.mu_phi()
    assert abs(f - g["f_Helmholtz"][0]) < 1e-10
    assert abs(mu[0] - g["mu_chain"][0]) < 1e-10
    if domain:
        assert abs(r["cell_param"][0] - g["cell_param"][0]) < 1e-9


@pytest.mark.parametrize("domain", [False, True])
def test_newton_lamellar_golden_n_cut(domain):
    """N_cut = 8 of 17 stars: finite differences for the first 8, the
    Debye tail beyond (response_pd_omega / debye_rsp,
    src/response_pd_mod.f90:91-180); Newton lands on the same golden state."""
    g = GOLD["lamellar_outfile"]
    cell0 = g["cell_param"][0] * (1.03 if domain else 1.0)
    s = diblock(1, [32], "lamellar", [cell0], fA=0.5, chiN=g["chi"][0])
    basis = StarBasis("-1", [32])
    prov = OracleProvider(s, "-1")
    w, rho, r = iterate_nr(prov, basis, s, lamellar_guess(s), error_max=1e-11, max_itr=80, domain=domain, n_cut=8)
    assert r["converged"]
    o = prov.o
    o.set_cell(r["cell_param"])
    rr, q = o.density(w)
    f, p = o.free_energy(w, rr)
    assert abs(f - g["f_Helmholtz"][0]) < 1e-10
    if domain:
        assert abs(r["cell_param"][0] - g["cell_param"][0]) < 1e-9


def test_debye_correlation_limits():
    """q -> 0: corrlt_ab = phi f_a f_b (g1 = g2 = 1); large q: the self term
    decays like 2/x."""
    from pscf_b200.newton import debye_correlation
    s = diblock(1, [32], "lamellar", [1.7], fA=0.3, chiN=15.0)
    c = debye_correlation(s, np.array([0.0, 1e6]))
    np.testing.assert_allclose(c[:, :, 0], [[0.09, 0.21], [0.21, 0.49]], rtol=1e-14)
    x = 0.3 * 1e6 / 6.0
    assert abs(c[0, 0, 1] - 0.09 * 2.0 * (x - 1.0) / x ** 2) < 1e-15


def test_newton_n_cut_zero_uses_the_debye_response_alone():
    """N_cut = 0 (N_corner = 0 in iterate_NR_startup,
    src/iterate_mod.fp.f90:200-225): no column is differenced, the Jacobian
    is the homogeneous melt's Debye response, and from the lamellar guess
    at chi N = 15 Newton settles on the disordered solution (uniform rho,
    F = the Flory-Huggins free energy), itself a solution of the SCF
    equations."""
    from pscf_b200.sweep import free_energy_fh
    g = GOLD["lamellar_outfile"]
    s = diblock(1, [32], "lamellar", [g["cell_param"][0]], fA=0.5, chiN=g["chi"][0])
    basis = StarBasis("-1", [32])
    prov = OracleProvider(s, "-1")
    batches = []
    inner = prov.__call__

    def counting(oms, cells=None, want_stress=False):
        batches.append(len(oms))
        return inner(oms, cells, want_stress)
    w, rho, r = iterate_nr(counting, basis, s, lamellar_guess(s), error_max=1e-11, max_itr=100, n_cut=0)
    assert r["converged"] and set(batches) <= {0, 1}
    assert np.ptp(rho, axis=1).max() < 1e-10
    o = prov.o
    rr, q = o.density(w)
    f, p = o.free_energy(w, rr)
    assert abs(f - free_energy_fh(s)) < 1e-9
