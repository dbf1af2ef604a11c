"""Graph-driven Anderson iterations (pscfg_am_param.graph_check > 0).

Each iteration -- density, stress, free energy, the Anderson sums, the
coefficient solve (src/iterate_mod.fp.f90:1349-1381), the mixing, the
projection and the cell update -- replays from one captured CUDA graph with
the per-instance control on the device; the host reads the status words every
graph_check iterations.  Everything is compared with the host-driven
iteration, which the oracle pins elsewhere.  The control kernels round as
the host loop does (no multiply-add contraction, the same lambda ramp), so
canonical runs on the k-space-table kernels give the host's iterates to the
last bits; the grand ensemble (exp of mu on the device) and the plane-kernel
grids (separable k-space factors from the device cell) agree to roundoff."""
import numpy as np
import pytest

from pscf_b200.engine import CHECKPOINT, Engine, EngineError, FP64, MIXED
from tests.cases import bcc_guess, diblock, lamellar_guess, omega_guess, rel_err

pytestmark = pytest.mark.gpu


def _solve(systems, w0, group=None, **kw):
    import copy
    systems = copy.deepcopy(systems)   # a domain solve writes the relaxed cell into its systems
    e = Engine(systems, FP64)
    if group:
        for i in range(len(systems)):
            e.set_symmetry(i, group)
    w, rho, res = e.iterate_am(w0, **kw)
    n = e.launch_count
    e.close()
    return w, rho, res, n


def test_fixed_iterations_match_host_bcc_with_cell():
    """BCC 16^3 (I m -3 m star weights, projection, cell relaxation): 12
    iterations driven by the host and by the graph give the same fields."""
    ss = [diblock(3, [16, 16, 16], "cubic", [1.95 + 0.02 * i], fA=0.25 + 0.01 * i, chiN=20.0 + i, ds=0.02)
          for i in range(3)]
    w0 = np.stack([bcc_guess(s, amp=6.0) for s in ss])
    kw = dict(error_max=1e-14, max_itr=11, n_hist=20, domain=True)
    w_h, rho_h, r_h, _ = _solve(ss, w0, "I m -3 m", **kw)
    w_g, rho_g, r_g, _ = _solve(ss, w0, "I m -3 m", graph_check=4, **kw)
    for a, b in zip(r_h, r_g):
        assert a["status"] == b["status"] == "maxiter" and a["itr"] == b["itr"] == 12
        assert abs(a["f_helmholtz"] - b["f_helmholtz"]) < 1e-13
        np.testing.assert_allclose(b["cell_param"], a["cell_param"], rtol=1e-14)
        np.testing.assert_allclose(b["stress"], a["stress"], rtol=1e-12, atol=1e-15)
    assert rel_err(w_g, w_h) < 1e-14 and rel_err(rho_g, rho_h) < 1e-14


def test_converged_solve_matches_host_bcc():
    ss = [diblock(3, [16, 16, 16], "cubic", [1.95], fA=0.25, chiN=20.0, ds=0.02),
          diblock(3, [16, 16, 16], "cubic", [1.97], fA=0.27, chiN=21.0, ds=0.02)]
    w0 = np.stack([bcc_guess(s, amp=6.0) for s in ss])
    kw = dict(error_max=1e-9, max_itr=300, n_hist=20, domain=True)
    _, _, r_h, n_h = _solve(ss, w0, "I m -3 m", **kw)
    _, _, r_g, n_g = _solve(ss, w0, "I m -3 m", graph_check=5, **kw)
    for a, b in zip(r_h, r_g):
        assert a["converged"] and b["converged"], (a, b)
        assert a["itr"] == b["itr"]
        assert abs(a["f_helmholtz"] - b["f_helmholtz"]) < 1e-12
        np.testing.assert_allclose(b["cell_param"], a["cell_param"], rtol=1e-13)
        np.testing.assert_allclose(b["mu_chain"][:1], a["mu_chain"][:1], rtol=1e-13)
    assert n_g > 0 and n_h > 0


def test_nan_instance_retired_and_staggered_finishes():
    """Lamellae converging after different numbers of iterations (the graph
    is rebuilt as they finish) and one NaN-injected instance retired as
    non-finite, as in the host-driven run."""
    ss = [diblock(1, [32], "lamellar", [1.7], fA=0.3 + 0.04 * i, chiN=12.0 + 2.0 * i) for i in range(6)]
    w0 = np.stack([lamellar_guess(s) for s in ss])
    w0[2, 0, 7] = np.nan
    kw = dict(error_max=1e-9, max_itr=400, domain=True)
    _, _, r_h, _ = _solve(ss, w0, **kw)
    _, _, r_g, _ = _solve(ss, w0, graph_check=2, **kw)
    assert r_g[2]["status"] == "nonfinite" and not r_g[2]["converged"]
    for a, b in zip(r_h, r_g):
        assert a["status"] == b["status"]
        if a["converged"]:
            assert a["itr"] == b["itr"]
            assert abs(a["f_helmholtz"] - b["f_helmholtz"]) < 1e-12
    assert len({r["itr"] for r in r_g if r["converged"]}) > 1


@pytest.mark.parametrize("ensemble", [0, 1])
def test_fixed_iterations_match_host_blend(ensemble):
    """Diblock + homopolymer + solvent, canonical and grand canonical (phi
    from the device Q inside the iteration), without cell relaxation."""
    from pscf_b200.system import Chain, Solvent, System
    chains = [Chain([0, 1], [0.4, 0.6], phi=0.7, mu=2.0), Chain([0], [0.5], phi=0.2, mu=1.5)]
    solvents = [Solvent(monomer=1, size=0.1, phi=0.1, mu=0.3)]
    s = System(dim=2, ngrid=[16, 16], crystal_system="hexagonal", cell_param=[1.7], kuhn=[1.0, 1.2],
               chi=[[0, 14.0], [14.0, 0]], chains=chains, solvents=solvents, ds=0.02, ensemble=ensemble)
    w0 = omega_guess(s, 31, 1.5)[None]
    kw = dict(error_max=1e-14, max_itr=9, domain=False)
    w_h, rho_h, r_h, _ = _solve([s], w0, **kw)
    w_g, rho_g, r_g, _ = _solve([s], w0, graph_check=3, **kw)
    a, b = r_h[0], r_g[0]
    tol = 1e-13 if ensemble == 0 else 1e-10
    assert a["itr"] == b["itr"] == 10
    assert abs(a["f_helmholtz"] - b["f_helmholtz"]) < tol and abs(a["pressure"] - b["pressure"]) < tol
    np.testing.assert_allclose(b["mu_chain"][:2], a["mu_chain"][:2], rtol=tol)
    np.testing.assert_allclose(b["q"][:2], a["q"][:2], rtol=tol)
    np.testing.assert_allclose(b["stress"][:1], a["stress"][:1], rtol=100 * tol, atol=1e-14)
    assert rel_err(w_g, w_h) < tol and rel_err(rho_g, rho_h) < tol


def test_plane_kernel_grid_fixed_iterations():
    """64^3 (the plane kernels; the graph computes their separable k-space
    factors on the device from the device cell, the host-driven sweep on the
    host in extended precision)."""
    s = diblock(3, [64, 64, 64], "cubic", [3.7], fA=0.4, chiN=16.0, ds=0.1)
    w0 = omega_guess(s, 3, 2.0)[None]
    kw = dict(error_max=1e-14, max_itr=3, domain=True)
    w_h, _, r_h, _ = _solve([s], w0, **kw)
    w_g, _, r_g, _ = _solve([s], w0, graph_check=2, **kw)
    assert r_h[0]["itr"] == r_g[0]["itr"] == 4
    assert abs(r_h[0]["f_helmholtz"] - r_g[0]["f_helmholtz"]) < 1e-11
    np.testing.assert_allclose(r_g[0]["cell_param"][:1], r_h[0]["cell_param"][:1], rtol=1e-11)
    assert rel_err(w_g, w_h) < 1e-11


def test_incremental_graph_run_and_refusals():
    ss = [diblock(1, [32], "lamellar", [1.7], fA=0.5, chiN=15.0) for _ in range(2)]
    w0 = np.stack([lamellar_guess(s) for s in ss])
    e = Engine(ss, FP64)
    e.am_begin(w0, error_max=1e-9, max_itr=400, graph_check=3)
    assert e.am_iterate(4) == 2
    _, _, mid = e.am_results(want_fields=False)
    assert all(r["status"] == "running" and r["itr"] == 4 for r in mid)
    while e.am_iterate(7) > 0:
        pass
    _, _, res = e.am_results(want_fields=False)
    assert all(r["converged"] for r in res)
    e.close()
    for prec in (MIXED, FP64 | CHECKPOINT):
        m = Engine(ss, prec)
        with pytest.raises(EngineError):
            m.iterate_am(w0, error_max=1e-9, max_itr=10, graph_check=2)
        m.close()
