"""Propagator checkpointing (PSCFG_CHECKPOINT): the engine keeps every K-th
slice of qf and qr (K = ceil(sqrt(Ns))) and two working segments instead of
the Ns + 1 slices of the reference's chain_grid_type%qf/qr
(src/chain_mod.f90:159-165), and recomputes each segment from its
checkpoint with the same step kernels for the density's Simpson sums, the
stress and the adjoint.  Everything is compared with the stored-slice
engine, which the oracle pins elsewhere."""
import numpy as np
import pytest

from pscf_b200.engine import CHECKPOINT, Engine, EngineError, FP32, FP64
from tests.cases import diblock, omega_guess, rel_err, triblock

pytestmark = pytest.mark.gpu

CASES = [
    (1, [32], "lamellar", [1.7], 0.005),
    (2, [24, 24], "hexagonal", [1.9], 0.01),
    (2, [64, 64], "hexagonal", [1.9], 0.01),
    (3, [16, 16, 16], "cubic", [3.9], 0.01),
    (3, [32, 32, 32], "cubic", [3.9], 0.01),
    (3, [64, 64, 64], "cubic", [3.7], 0.005),
]


def _pair(systems, prec=FP64):
    return Engine(systems, prec), Engine(systems, prec | CHECKPOINT)


@pytest.mark.parametrize("dim,ngrid,crystal,cell,ds", CASES)
def test_checkpointed_density_stress_free_energy(dim, ngrid, crystal, cell, ds):
    ss = [diblock(dim, ngrid, crystal, cell, fA=0.3 + 0.05 * i, chiN=15.0 + i, ds=ds) for i in range(2)]
    w = np.stack([omega_guess(s, 7 + i, 2.0) for i, s in enumerate(ss)])
    e, c = _pair(ss)
    rho, q = e.density(w)
    rho_c, q_c = c.density(w)
    assert rel_err(q_c[:, :1], q[:, :1]) < 1e-14
    assert rel_err(rho_c, rho) < 1e-13, rel_err(rho_c, rho)
    for i in range(2):
        qf, qr = e.propagators(i, 0)
        qf_c, qr_c = c.propagators(i, 0)
        assert qf_c.shape == qf.shape
        # same kernels; a segment's first step starts from the checkpoint in
        # global memory where the uninterrupted sweep fused it into the
        # previous step's last kernel: agreement to the last bits
        assert rel_err(qf_c, qf) < 1e-14 and rel_err(qr_c, qr) < 1e-14
    np.testing.assert_allclose(c.scf_stress(), e.scf_stress(), rtol=1e-12, atol=1e-15)
    f, p, _ = e.free_energy()
    f_c, p_c, _ = c.free_energy()
    np.testing.assert_allclose(f_c, f, rtol=1e-13)
    e.close()
    c.close()


def test_checkpointed_triblock_uneven_chains_and_fp32():
    """Three blocks (block changes inside segments) and FP32 propagation."""
    s = triblock(3, [8, 12, 20], "orthorhombic", [1.5, 3.0, 5.25], ds=0.02)
    w = omega_guess(s, 9, 2.0)[None]
    for prec, tol in ((FP64, 1e-13), (FP32, 1e-6)):
        e, c = _pair([s], prec)
        rho, q = e.density(w)
        rho_c, q_c = c.density(w)
        assert rel_err(rho_c, rho) < tol and rel_err(q_c[:, :1], q[:, :1]) < tol
        np.testing.assert_allclose(c.scf_stress(), e.scf_stress(), rtol=tol * 100, atol=1e-12)
        e.close()
        c.close()


@pytest.mark.parametrize("dim,ngrid,crystal,cell,fA,chiN,ds", [(1, [24], "lamellar", [1.6], 0.35, 14.0, 0.02),
                                                        (3, [16, 16, 16], "cubic", [2.0], 0.35, 14.0, 0.02),
                                                        (3, [64, 64, 64], "cubic", [3.7], 0.40, 16.0, 0.005)])
def test_checkpointed_adjoint_matches_stored(dim, ngrid, crystal, cell, fA, chiN, ds):
    """The last case is the gyroid workload's grid and contour (Ns = 200)."""
    s = diblock(dim, ngrid, crystal, cell, fA=fA, chiN=chiN, ds=ds)
    rng = np.random.default_rng(5)
    w = omega_guess(s, 3, 2.0)[None]
    G = rng.normal(size=(1, 2, s.nr))
    a = np.array([[0.7]])
    e, c = _pair([s])
    e.density(w)
    c.density(w)
    g, gc = e.density_adjoint(G, a, want_cell=True)
    g_c, gc_c = c.density_adjoint(G, a, want_cell=True)
    assert rel_err(g_c, g) < 1e-13, rel_err(g_c, g)
    np.testing.assert_allclose(gc_c, gc, rtol=1e-12, atol=1e-15)
    e.close()
    c.close()


def test_checkpointed_anderson_solve_and_memory():
    """A full Anderson solve with cell relaxation gives the stored-slice
    result, with the propagator memory reduced: C3-size 64^3 diblock at
    ds = 0.005 (Ns = 200, K = 15: 30 checkpoints + 32 working slices per
    chain instead of 402 slices)."""
    import torch
    from tests.cases import bcc_guess
    s = diblock(3, [16, 16, 16], "cubic", [1.95], fA=0.25, chiN=20.0, ds=0.02)
    w0 = bcc_guess(s, amp=6.0)[None]
    res = []
    for prec in (FP64, FP64 | CHECKPOINT):
        e = Engine([s], prec)
        e.set_symmetry(0, "I m -3 m")
        _, _, r = e.iterate_am(w0, error_max=1e-9, max_itr=300, domain=True)
        res.append(r[0])
        e.close()
    assert res[0]["converged"] and res[1]["converged"]
    assert abs(res[0]["f_helmholtz"] - res[1]["f_helmholtz"]) < 1e-10
    big = diblock(3, [64, 64, 64], "cubic", [3.7], fA=0.4, chiN=16.0, ds=0.005)
    used = []
    for prec in (FP64, FP64 | CHECKPOINT):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        e = Engine([big], prec)
        torch.cuda.synchronize()
        used.append(free0 - torch.cuda.mem_get_info()[0])
        e.close()
    slab = 2 * 201 * big.nr * 8
    assert used[0] - used[1] > 0.8 * (slab - 62 * big.nr * 8), used


def test_checkpointed_engine_refuses_the_response():
    s = diblock(1, [32], "lamellar", [1.7])
    c = Engine([s], FP64 | CHECKPOINT)
    c.density(omega_guess(s, 1, 2.0)[None])
    with pytest.raises(EngineError):
        c.response_raw(0, [0.0, 0.0, 0.0], 0.0, [0], np.zeros((1, s.nr)), [0], np.ones(1, dtype=complex))
    c.close()
