"""GPU engine vs the FP64 CPU oracle: single steps, density, stress, F."""
import numpy as np
import pytest

from oracle import oracle as O
from pscf_b200.engine import Engine, FP32, FP64
from tests.cases import diblock, omega_guess, rel_err, smooth_field, triblock

pytestmark = pytest.mark.gpu

STEP_CASES = [
    (1, [32], "lamellar", [1.7]),
    (1, [30], "lamellar", [1.3]),
    (1, [27], "lamellar", [1.4]),
    (2, [24, 24], "hexagonal", [1.9]),
    (2, [20, 14], "rectangular", [1.6, 2.1]),
    (2, [15, 12], "rectangular", [1.6, 2.1]),
    (3, [16, 16, 16], "cubic", [3.9]),
    (3, [20, 12, 14], "orthorhombic", [2.0, 2.5, 3.0]),
    (3, [9, 10, 8], "orthorhombic", [2.0, 2.5, 3.0]),
    (3, [32, 32, 32], "cubic", [3.9]),
    (3, [64, 64, 64], "cubic", [3.7]),
]


@pytest.mark.parametrize("dim,ngrid,crystal,cell", STEP_CASES)
def test_step_parity_fp64(dim, ngrid, crystal, cell):
    s = diblock(dim, ngrid, crystal, cell)
    e = Engine([s], FP64)
    o = O.Oracle(s)
    ksq = o.ksq()
    np.testing.assert_allclose(e.ksq(0), ksq, rtol=1e-14, atol=1e-12)
    w = 7.5 + smooth_field(s, 11, 3.0)
    q0 = 1.0 + 0.3 * smooth_field(s, 12, 1.0)
    for nsteps in ((1, 7) if s.nr <= 40000 else (1,)):
        ref = O.step(s, ksq, 1.0, 0.01, w, q0, nsteps)
        got = e.propagate(0, w, 1.0, 0.01, q0, nsteps)
        assert rel_err(got, ref) < 1e-12, (nsteps, rel_err(got, ref))


DENSITY_CASES = [
    (1, [32], "lamellar", [1.7], 0.5),
    (3, [32, 32, 32], "cubic", [1.95], 0.25),
    (2, [24, 24], "hexagonal", [1.9], 0.3),
    (3, [16, 16, 16], "cubic", [3.9], 0.25),
    (3, [12, 10, 14], "orthorhombic", [2.0, 2.5, 3.0], 0.4),
]


@pytest.mark.parametrize("dim,ngrid,crystal,cell,fA", DENSITY_CASES)
def test_density_stress_free_energy_fp64(dim, ngrid, crystal, cell, fA):
    s = diblock(dim, ngrid, crystal, cell, fA=fA, chiN=15.0, ds=0.05 if np.prod(ngrid) > 20000 else 0.01)
    w = omega_guess(s, 5, 2.0)
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    st_ref = o.stress()
    f_ref, p_ref = o.free_energy(w, rho_ref)
    e = Engine([s], FP64)
    rho, q = e.density(w[None])
    assert rel_err(q[0, :1], q_ref) < 1e-12
    assert rel_err(rho[0], rho_ref) < 1e-12
    qf_ref, qr_ref = o.propagators(0)
    qf, qr = e.propagators(0, 0)
    assert rel_err(qf, qf_ref) < 1e-12 and rel_err(qr, qr_ref) < 1e-12
    st = e.scf_stress()[0, : len(st_ref)]
    assert np.max(np.abs(st - st_ref)) < 1e-10 * max(1.0, np.max(np.abs(st_ref)))
    f, p, mu = e.free_energy()
    assert abs(f[0] - f_ref) < 1e-11 and abs(p[0] - p_ref) < 1e-11


def test_triblock_density_fp64():
    s = triblock(3, [8, 12, 20], "orthorhombic", [1.5, 3.0, 5.25], ds=0.02)
    w = omega_guess(s, 9, 2.0)
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    e = Engine([s], FP64)
    rho, q = e.density(w[None])
    assert rel_err(rho[0], rho_ref) < 1e-12
    assert rel_err(q[0, :1], q_ref) < 1e-12
    st = e.scf_stress()[0, :3]
    np.testing.assert_allclose(st, o.stress(), rtol=1e-10, atol=1e-12)


def test_batched_uneven_instances_fp64():
    """Instances with different f_A (uneven step counts), chi and cells."""
    systems = [diblock(3, [12, 12, 12], "cubic", [3.6 + 0.1 * i], fA=0.25 + 0.05 * i, chiN=14.0 + i)
               for i in range(4)]
    ws = np.stack([omega_guess(s, 40 + i, 1.5) for i, s in enumerate(systems)])
    e = Engine(systems, FP64)
    rho, q = e.density(ws)
    st = e.scf_stress()
    f, p, mu = e.free_energy()
    for i, s in enumerate(systems):
        o = O.Oracle(s)
        rr, qq = o.density(ws[i])
        assert rel_err(rho[i], rr) < 1e-12
        assert rel_err(q[i, :1], qq) < 1e-12
        assert abs(st[i, 0] - o.stress()[0]) < 1e-10 * max(1.0, abs(o.stress()[0]))
        fr, pr = o.free_energy(ws[i], rr)
        assert abs(f[i] - fr) < 1e-11


@pytest.mark.parametrize("dim,ngrid,crystal,cell", [(3, [16, 16, 16], "cubic", [3.9]),
                                                   (2, [64, 64], "hexagonal", [1.9])])
def test_density_fp32_close(dim, ngrid, crystal, cell):
    """FP32 propagation (FP64 sums) against the FP64 oracle; 64 x 64 runs the
    whole-sweep 2-D kernel in single precision."""
    s = diblock(dim, ngrid, crystal, cell, fA=0.3)
    w = omega_guess(s, 3, 2.0)
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    e = Engine([s], FP32)
    rho, q = e.density(w[None])
    assert rel_err(rho[0], rho_ref) < 2e-5
    assert rel_err(q[0, :1], q_ref) < 2e-5


def test_cluster_step_matches_five_launch_step(monkeypatch):
    """The one-launch cluster step (32^3) agrees with the five-launch
    compile-time-shaped step, for propagation, the full density and the
    adjoint (which stores the step intermediates)."""
    s = diblock(3, [32, 32, 32], "cubic", [1.95], fA=0.3, ds=0.05)
    w = 7.5 + smooth_field(s, 5, 3.0)
    q0 = 1.0 + 0.3 * smooth_field(s, 6, 1.0)
    wf = omega_guess(s, 8, 2.0)
    g = smooth_field(s, 9, 1.0)
    grad = np.stack([g, -0.5 * g])[None]
    out = []
    for flag in ("0", "1"):
        monkeypatch.setenv("PSCFG_CLUSTER_STEP", flag)
        e = Engine([s], FP64)
        a = e.propagate(0, w, 1.0, 0.01, q0, 3)
        r, q = e.density(wf[None])
        gw = e.density_adjoint(grad)
        out.append((a, r, q[:, :1], gw))
        e.close()
    for x, y in zip(out[0], out[1]):
        assert rel_err(x, y) < 1e-13


@pytest.mark.parametrize("n", [16, 32, 64])
def test_fixed_shape_kernels_match_generic(n, monkeypatch):
    """The compile-time-shaped 3-D step kernels agree with the run-time sized
    ones (same algebra, different transform order) to roundoff."""
    s = diblock(3, [n, n, n], "cubic", [3.9], fA=0.3)
    w = 7.5 + smooth_field(s, 5, 3.0)
    q0 = 1.0 + 0.3 * smooth_field(s, 6, 1.0)
    e1 = Engine([s], FP64)
    a = e1.propagate(0, w, 1.0, 0.01, q0, 3)
    monkeypatch.setenv("PSCFG_GENERIC_KERNELS", "1")
    e2 = Engine([s], FP64)
    b = e2.propagate(0, w, 1.0, 0.01, q0, 3)
    assert rel_err(a, b) < 1e-13
    for prec, tol in ((FP32, 2e-6),):
        monkeypatch.delenv("PSCFG_GENERIC_KERNELS")
        e3 = Engine([s], prec)
        c = e3.propagate(0, w, 1.0, 0.01, q0, 3)
        assert rel_err(c, a) < tol


@pytest.mark.parametrize("n", [16, 32])
def test_fixed_shape_density_and_stress_paths_agree(n, monkeypatch):
    """Register-column kernels (default), shared-memory kernels and the
    run-time sized kernels give the same density, Q and stress."""
    s = diblock(3, [n, n, n], "cubic", [1.95], fA=0.3, ds=0.05)
    w = omega_guess(s, 11, 2.0)
    out = []
    for env in ({}, {"PSCFG_SMEM_FFT": "1"}, {"PSCFG_GENERIC_KERNELS": "1"}):
        for k in ("PSCFG_SMEM_FFT", "PSCFG_GENERIC_KERNELS"):
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        e = Engine([s], FP64)
        rho, q = e.density(w[None])
        st = e.scf_stress()
        out.append((rho, q[:, :1], st[:, :1]))
        e.close()
    for o in out[1:]:
        assert rel_err(o[0], out[0][0]) < 1e-13
        assert rel_err(o[1], out[0][1]) < 1e-13
        assert abs(o[2][0, 0] - out[0][2][0, 0]) < 1e-11 * max(1.0, abs(out[0][2][0, 0]))


def _blend(ensemble):
    """AB diblock + A homopolymer + B-selective solvent (three species)."""
    from pscf_b200.system import Chain, Solvent, System
    chains = [Chain([0, 1], [0.4, 0.6], phi=0.7, mu=2.0), Chain([0], [0.5], phi=0.2, mu=1.5)]
    solvents = [Solvent(monomer=1, size=0.1, phi=0.1, mu=0.3)]
    return System(dim=2, ngrid=[16, 16], crystal_system="hexagonal", cell_param=[1.7], kuhn=[1.0, 1.2],
                  chi=[[0, 14.0], [14.0, 0]], chains=chains, solvents=solvents, ds=0.02, ensemble=ensemble)


@pytest.mark.parametrize("ensemble", [0, 1])
def test_solvent_and_ensemble_parity(ensemble):
    s = _blend(ensemble)
    w = omega_guess(s, 31, 1.5)
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    st_ref = o.stress()
    f_ref, p_ref = o.free_energy(w, rho_ref)
    mu_ref, phi_ref = o.mu_phi()
    e = Engine([s], FP64)
    rho, q = e.density(w[None])
    assert rel_err(rho[0], rho_ref) < 1e-12
    assert rel_err(q[0, :2], q_ref) < 1e-12
    st = e.scf_stress()[0, :1]
    np.testing.assert_allclose(st, st_ref, rtol=1e-10, atol=1e-12)
    f, p, mu = e.free_energy()
    assert abs(f[0] - f_ref) < 1e-11 and abs(p[0] - p_ref) < 1e-11
    np.testing.assert_allclose(mu[0, :2], mu_ref, rtol=1e-12)


def test_concurrent_engines_with_different_plane_sizes():
    """Engines of different grid shapes driven from separate host threads
    (small lamellar and large hexagonal plane kernels launched together)
    give the same densities as when run alone."""
    import threading
    lam = diblock(1, [64], "lamellar", [1.7], fA=0.4, ds=0.02)
    hexs = diblock(2, [64, 64], "hexagonal", [1.9], fA=0.3, ds=0.02)
    wl, wh = omega_guess(lam, 1, 2.0), omega_guess(hexs, 2, 2.0)
    ref = [Engine([lam], FP64).density(wl[None])[0], Engine([hexs], FP64).density(wh[None])[0]]
    engines = [Engine([lam], FP64), Engine([hexs], FP64)]
    outs = [[], []]
    errs = []

    def run(k, w):
        try:
            for _ in range(40):
                outs[k].append(engines[k].density(w[None])[0])
        except Exception as ex:      # surfaced below
            errs.append(ex)

    th = [threading.Thread(target=run, args=(0, wl)), threading.Thread(target=run, args=(1, wh))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for k in range(2):
        for r in outs[k]:
            assert rel_err(r, ref[k]) < 1e-14


def test_sweep_graph_replay_matches_direct_launches(monkeypatch):
    """The 3-D sweep replayed from a captured CUDA graph gives bit-identical
    propagators to direct launches, on first capture and on replay, and an
    Anderson run (whose active instance set shrinks) agrees too."""
    s = diblock(3, [32, 32, 32], "cubic", [1.95], fA=0.3, ds=0.02)
    ws = np.stack([omega_guess(s, 20 + i, 2.0) for i in range(3)])
    out = {}
    for flag in ("0", "1"):
        monkeypatch.setenv("PSCFG_NO_GRAPHS", flag)
        e = Engine([s, s, s], FP64)
        r1, q1 = e.density(ws)
        r2, q2 = e.density(ws[::-1].copy())
        _, _, res = e.iterate_am(ws, error_max=1e-6, max_itr=40)
        out[flag] = (r1, q1, r2, q2, [x["f_helmholtz"] for x in res], [x["itr"] for x in res])
        e.close()
    a, b = out["0"], out["1"]
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x, y)
    assert a[4] == b[4] and a[5] == b[5]


@pytest.mark.parametrize("n,choices", [(32, ("4", "2", "1")), (16, ("8", "4", "2", "1"))])
def test_sweep_planes_per_cta_agree(n, choices, monkeypatch):
    """The register sweep with any number of x-y planes per CTA (chosen by
    launch size: fewer planes for few instances) gives the same densities,
    Q, stress and free energy: to roundoff against the most planes per CTA
    (whose column pass transforms the real columns kx = 0 and n/2 together
    as one complex column), bit-identical among the others (every row and
    column by the same arithmetic whatever CTA holds it)."""
    s = diblock(3, [n, n, n], "cubic", [1.95 * n / 32], fA=0.3, ds=0.02)
    ws = np.stack([omega_guess(s, 30 + i, 2.0) for i in range(2)])
    out = {}
    for p in choices:
        monkeypatch.setenv("PSCFG_PLANES", p)
        e = Engine([s, s], FP64)
        rho, q = e.density(ws)
        st = e.scf_stress()
        fh, fp, _ = e.free_energy()
        out[p] = (rho, q, st, fh, fp)
        e.close()
    ref = out[choices[0]]
    for p in choices[1:]:
        for x, y in zip(out[p], ref):
            assert np.max(np.abs(x - y)) <= 1e-12 * max(1.0, np.max(np.abs(y))), p
    for p in choices[2:]:
        for x, y in zip(out[p], out[choices[1]]):
            assert np.array_equal(x, y), p


@pytest.mark.parametrize("ngrid,crystal,cell", [([12, 20, 28], "orthorhombic", [1.5, 2.0, 2.5]),
                                                ([16, 30, 14], "orthorhombic", [1.6, 2.4, 1.4]),
                                                ([24, 24, 24], "cubic", [2.0])])
def test_line_pass_step_matches_plane_step(ngrid, crystal, cell, monkeypatch):
    """The line-pass 3-D step (any even n1 with 2,3,5,7-smooth extents; used
    where the x-y plane does not fit shared memory) agrees with the
    whole-plane kernels: propagation, density, stress, and the FP32 path."""
    s = diblock(3, ngrid, crystal, cell, fA=0.3, ds=0.05)
    w = omega_guess(s, 12, 2.0)
    wf = 7.0 + smooth_field(s, 13, 2.0)
    q0 = 1.0 + 0.3 * smooth_field(s, 14, 1.0)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("PSCFG_LINE_STEP", flag)
        e = Engine([s], FP64)
        p = e.propagate(0, wf, 1.0, 0.01, q0, 3)
        rho, q = e.density(w[None])
        st = e.scf_stress()[0, :len(cell)]
        e.close()
        e32 = Engine([s], FP32)
        rho32, _ = e32.density(w[None])
        e32.close()
        out[flag] = (p, rho, q[:, :1], st, rho32)
    a, b = out["0"], out["1"]
    assert rel_err(a[0], b[0]) < 1e-13
    assert rel_err(a[1], b[1]) < 1e-13 and rel_err(a[2], b[2]) < 1e-13
    assert np.max(np.abs(a[3] - b[3])) < 1e-11 * max(1.0, np.max(np.abs(b[3])))
    assert rel_err(a[4], b[4]) < 1e-5


def test_large_plane_density_uses_line_passes():
    """A grid whose x-y plane does not fit the shared memory of the
    whole-plane kernels (256 x 128 spectral plane, 528 KB) runs on the line
    passes and matches the oracle's propagators and density."""
    s = diblock(3, [256, 128, 4], "orthorhombic", [4.0, 3.0, 0.5], fA=0.4, chiN=12.0, ds=0.1)
    w = omega_guess(s, 15, 2.0)
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    e = Engine([s], FP64)
    rho, q = e.density(w[None])
    assert rel_err(q[0, :1], q_ref) < 1e-12
    assert rel_err(rho[0], rho_ref) < 1e-12
    qf_ref, _ = o.propagators(0)
    qf, _ = e.propagators(0, 0)
    assert rel_err(qf, qf_ref) < 1e-12
    e.close()


ROUGH_CASES = [(3, [64, 64, 64], "cubic", [3.7]), (3, [32, 32, 32], "cubic", [3.9]), (3, [16, 16, 16], "cubic", [3.9]),
               (2, [64, 64], "hexagonal", [1.9])]


@pytest.mark.parametrize("dim,ngrid,crystal,cell", ROUGH_CASES)
@pytest.mark.parametrize("path", ["default", "PSCFG_PLANE_P=0", "PSCFG_GENERIC_KERNELS=1", "PSCFG_SMEM_FFT=1"])
def test_rough_fields_all_kernel_paths(monkeypatch, dim, ngrid, crystal, cell, path):
    """White-noise omega and q (every wave vector up to the Nyquist ones
    carries weight): single steps and a density against the oracle, for
    each kernel family of the grid."""
    if path != "default":
        k, v = path.split("=")
        monkeypatch.setenv(k, v)
    s = diblock(dim, ngrid, crystal, cell, fA=0.4, chiN=15.0, ds=0.05)
    rng = np.random.default_rng(99)
    w = s.omega_uniform()[:, None] + rng.normal(0.0, 1.0, (2, s.nr))
    q0 = 1.0 + 0.3 * rng.normal(size=s.nr)
    o = O.Oracle(s)
    ksq = o.ksq()
    e = Engine([s], FP64)
    ref = O.step(s, ksq, 1.0, 0.05, w[0], q0, 2)
    got = e.propagate(0, w[0], 1.0, 0.05, q0, 2)
    assert rel_err(got, ref) < 1e-12, ("step", rel_err(got, ref))
    rho_ref, q_ref = o.density(w)
    rho, q = e.density(w[None])
    assert rel_err(q[0, :1], q_ref) < 1e-12
    assert rel_err(rho[0], rho_ref) < 1e-12, ("density", rel_err(rho[0], rho_ref))
    e.close()


def test_measured_planes_per_cta():
    """The register sweep's planes per CTA are measured before the first
    sweep of each (grid, precision, class of field counts) -- one timed
    trial sweep per candidate -- and every density comes from the chosen
    count: repeated calls are bit-identical."""
    ss = [diblock(3, [32, 32, 32], "cubic", [3.9], fA=0.25 + 0.02 * i, chiN=20.0, ds=0.02) for i in range(3)]
    w = np.stack([omega_guess(s, 40 + i, 2.0) for i, s in enumerate(ss)])
    e = Engine(ss, FP64)
    outs = [e.density(w)[0] for _ in range(5)]
    p = e.sweep_planes(2 * len(ss))
    e.close()
    assert p in (1, 2, 4, -1), p                                     # -1: the cluster step
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


def test_cluster_sweep_matches_oracle(monkeypatch):
    """The thread-block-cluster sweep (one launch per sweep, kernels3x.cuh),
    forced with PSCFG_PLANES=-1, against the oracle on white-noise fields,
    and the densities of two engines that chose by measurement agree with
    it to roundoff."""
    s = diblock(3, [32, 32, 32], "cubic", [3.9], fA=0.4, chiN=15.0, ds=0.05)
    rng = np.random.default_rng(17)
    w = s.omega_uniform()[:, None] + rng.normal(0.0, 1.0, (2, s.nr))
    rho_ref, q_ref = O.Oracle(s).density(w)
    monkeypatch.setenv("PSCFG_PLANES", "-1")
    e = Engine([s, s], FP64)
    rho, q = e.density(np.stack([w, w]))
    e.close()
    for i in range(2):
        assert rel_err(q[i, :1], q_ref) < 1e-12
        assert rel_err(rho[i], rho_ref) < 1e-12, rel_err(rho[i], rho_ref)
    monkeypatch.delenv("PSCFG_PLANES")
    e = Engine([s, s], FP64)
    rho2, _ = e.density(np.stack([w, w]))
    e.close()
    assert rel_err(rho2, rho) < 1e-13


@pytest.mark.parametrize("dim,ngrid,crystal,cell", [(2, [12, 12], "square", [1.8]),
                                                   (3, [16, 16, 16], "cubic", [2.2])])
def test_system_at_the_limits(dim, ngrid, crystal, cell):
    """Every array bound of the C ABI at its maximum (include/pscf_gpu.h:
    4 monomers, 4 chains, an 8-block chain, 4 solvents): density, Q, Q_s,
    stress, free energy and mu against the oracle."""
    from pscf_b200.system import Chain, Solvent, System
    chi = np.array([[0, 12.0, 18.0, 9.0], [12.0, 0, 14.0, 20.0], [18.0, 14.0, 0, 11.0], [9.0, 20.0, 11.0, 0]])
    chains = [Chain([0, 1, 2, 3, 0, 1, 2, 3], [0.15, 0.1, 0.2, 0.1, 0.1, 0.15, 0.1, 0.1], phi=0.5),
              Chain([1], [0.4], phi=0.15), Chain([2, 3], [0.3, 0.3], phi=0.15), Chain([3, 0, 2], [0.2, 0.3, 0.25], phi=0.1)]
    solvents = [Solvent(monomer=m, size=0.05 + 0.05 * m, phi=0.025) for m in range(4)]
    s = System(dim=dim, ngrid=ngrid, crystal_system=crystal, cell_param=cell, kuhn=[1.0, 1.1, 0.9, 1.2], chi=chi,
               chains=chains, solvents=solvents, ds=0.02)
    w = omega_guess(s, 23, 1.5)
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    st_ref = o.stress()
    f_ref, p_ref = o.free_energy(w, rho_ref)
    mu_ref, _ = o.mu_phi()
    e = Engine([s], FP64)
    rho, q = e.density(w[None])
    assert rel_err(rho[0], rho_ref) < 1e-12
    assert rel_err(q[0, :len(q_ref)], q_ref) < 1e-12
    np.testing.assert_allclose(e.scf_stress()[0, :1], st_ref, rtol=1e-10, atol=1e-12)
    f, p, mu = e.free_energy()
    assert abs(f[0] - f_ref) < 1e-11 and abs(p[0] - p_ref) < 1e-11
    np.testing.assert_allclose(mu[0, :4], mu_ref[:4], rtol=1e-12)
    e.close()


def test_batch_with_a_solvent_only_instance():
    """Ragged batch: an instance without chains (two solvents) next to a
    diblock + solvent instance in one engine; densities, stress and free
    energy against the oracle (the chainless instance has no propagators,
    no stress and no sweep fields)."""
    from pscf_b200.system import Chain, Solvent, System
    kw = dict(dim=2, ngrid=[12, 12], crystal_system="square", cell_param=[1.8], kuhn=[1.0, 1.0],
              chi=[[0, 2.0], [2.0, 0]], ds=0.02)
    a = System(chains=[], solvents=[Solvent(0, 1.0, phi=0.6), Solvent(1, 0.5, phi=0.4)], **kw)
    b = System(chains=[Chain([0, 1], [0.4, 0.6], phi=0.8)], solvents=[Solvent(1, 0.3, phi=0.2)], **kw)
    ws = [omega_guess(a, 3, 0.5), omega_guess(b, 4, 1.0)]
    e = Engine([a, b], FP64)
    rho, q = e.density(np.stack(ws))
    st = e.scf_stress()
    f, p, _ = e.free_energy()
    for i, s in enumerate((a, b)):
        o = O.Oracle(s)
        rho_ref, q_ref = o.density(ws[i])
        assert rel_err(rho[i], rho_ref) < 1e-12, i
        f_ref, p_ref = o.free_energy(ws[i], rho_ref)
        assert abs(f[i] - f_ref) < 1e-11 and abs(p[i] - p_ref) < 1e-11, i
        np.testing.assert_allclose(st[i, :1], o.stress(), rtol=1e-10, atol=1e-13)
    e.close()
