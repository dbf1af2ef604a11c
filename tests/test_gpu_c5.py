"""ABC triblock on the 64 x 128 x 224 grid (F d d d : 2 cell 4 : 8 : 14, the
mixed-precision workload): the GPU against the FP64 oracle on that exact
grid, so that the radix-7 extent 224 and the shared-memory plane kernels of
kernels3p.cuh are exercised at full size.

Reference routines: step_exp (src/step_mod.f90:146-176), chain_density,
scf_stress and free_energy (src/scf_mod.fp.f90:315-550, 834-886)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pscf_b200 import groups
from pscf_b200.engine import Engine, FP32, FP64
from tests.cases import rel_err, smooth_field, triblock

pytestmark = pytest.mark.gpu

GRID = [64, 128, 224]
CELL = [4.0, 8.0, 14.0]
GROUP = "F d d d : 2"


@pytest.fixture(scope="module", autouse=True)
def _oracle_threads():
    O.set_fft_threads(os.cpu_count() or 1)
    yield
    O.set_fft_threads(1)


def c5(ds):
    return triblock(3, GRID, "orthorhombic", CELL, ds=ds)


@pytest.fixture(scope="module")
def c5_omega():
    """omega_a = (chi phi)_a + N(0, 0.5^2) noise projected onto F d d d : 2."""
    s = c5(0.005)
    rng = np.random.default_rng(20261207)
    w0 = s.omega_uniform()
    w = np.zeros((3, s.nr))
    for a in range(3):
        w[a] = w0[a] + groups.symmetrize(rng.normal(0.0, 0.5, size=s.nr), GROUP, GRID)
    return w


def test_c5_single_step_parity():
    s = c5(0.005)
    o = O.Oracle(s)
    ksq = o.ksq()
    e = Engine([s], FP64)
    np.testing.assert_allclose(e.ksq(0), ksq, rtol=1e-14, atol=1e-12)
    w = 7.5 + smooth_field(s, 11, 3.0)
    q0 = 1.0 + 0.3 * smooth_field(s, 12, 1.0)
    ref = O.step(s, ksq, 1.0, 0.005, w, q0, 1)
    got = e.propagate(0, w, 1.0, 0.005, q0, 1)
    assert rel_err(got, ref) < 1e-12, rel_err(got, ref)
    e.close()


def test_c5_density_stress_free_energy(c5_omega):
    """ds = 0.1 (4 + 4 + 4 = 12 steps per chain, block changes at slices 4 and 8):
    every slice, rho, Q, stress and F against the oracle."""
    s = c5(0.1)
    w = c5_omega
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    st_ref = o.stress()
    f_ref, p_ref = o.free_energy(w, rho_ref)
    qf_ref, qr_ref = o.propagators(0)
    e = Engine([s], FP64)
    rho, q = e.density(w[None])
    assert rel_err(q[0, :1], q_ref) < 1e-12
    assert rel_err(rho[0], rho_ref) < 1e-12, rel_err(rho[0], rho_ref)
    qf, qr = e.propagators(0, 0)
    assert qf.shape == qf_ref.shape
    assert rel_err(qf, qf_ref) < 1e-12 and rel_err(qr, qr_ref) < 1e-12
    st = e.scf_stress()[0, : len(st_ref)]
    assert np.max(np.abs(st - st_ref)) < 1e-10 * max(1.0, np.max(np.abs(st_ref))), (st, st_ref)
    f, p, mu = e.free_energy()
    assert abs(f[0] - f_ref) < 1e-11 * max(1.0, abs(f_ref)) and abs(p[0] - p_ref) < 1e-11 * max(1.0, abs(p_ref))
    e.close()


def _density_path(monkeypatch, plane_p, w, prec=FP64):
    monkeypatch.setenv("PSCFG_PLANE_P", str(plane_p))
    e = Engine([c5(0.005)], prec)
    rho, q = e.density(w[None])
    st = e.scf_stress()[0, :3].copy()
    e.close()
    return rho[0], q[0, 0], st


def test_c5_plane_kernels_match_generic(monkeypatch, c5_omega):
    """Full contour (ds = 0.005, 200 steps per chain): the plane kernels
    against the run-time shaped kernels, which the oracle pins elsewhere."""
    rho_p, q_p, st_p = _density_path(monkeypatch, 1, c5_omega)
    rho_g, q_g, st_g = _density_path(monkeypatch, 0, c5_omega)
    assert abs(q_p / q_g - 1.0) < 1e-12
    assert rel_err(rho_p, rho_g) < 1e-12, rel_err(rho_p, rho_g)
    np.testing.assert_allclose(st_p, st_g, rtol=1e-10, atol=1e-12)


def test_c5_fp32_propagation_close(monkeypatch, c5_omega):
    """FP32 propagation with FP64 contour sums, against FP64."""
    rho_d, q_d, _ = _density_path(monkeypatch, 1, c5_omega, FP64)
    rho_s, q_s, _ = _density_path(monkeypatch, 1, c5_omega, FP32)
    assert abs(q_s / q_d - 1.0) < 1e-4
    assert rel_err(rho_s, rho_d) < 1e-4, rel_err(rho_s, rho_d)


def test_plane_kernels_64_cubed():
    """The same plane kernels at 64^3 (the default there) against the oracle."""
    from tests.cases import diblock, omega_guess
    s = diblock(3, [64, 64, 64], "cubic", [3.7], fA=0.4, chiN=16.0, ds=0.05)
    w = omega_guess(s, 21, 2.0)
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    st_ref = o.stress()
    e = Engine([s], FP64)
    rho, q = e.density(w[None])
    assert rel_err(q[0, :1], q_ref) < 1e-12
    assert rel_err(rho[0], rho_ref) < 1e-12, rel_err(rho[0], rho_ref)
    st = e.scf_stress()[0, : len(st_ref)]
    assert np.max(np.abs(st - st_ref)) < 1e-10 * max(1.0, np.max(np.abs(st_ref))), (st, st_ref)
    e.close()
