#!/usr/bin/env python
"""Benchmark: MDE contour steps/s and converged SCFT solves/s on one node.

Default workload (--config c5; the largest single-GPU configuration): an
ABC linear triblock, block fractions 0.3/0.4/0.3, b = 1 for every block,
chi_AB N = chi_BC N = 30, chi_AC N = 60, orthorhombic cell with aspect
1 : 2 : 3.5 (a = 4, 8, 14), space group F d d d : 2, on a 64 x 128 x 224
grid with ds = 0.005 (60 + 80 + 60 contour steps).  Initial fields: the
uniform values chi.phi plus seeded N(0, 0.5^2) noise per monomer, projected
onto F d d d : 2 (seed 20261203 + 5 + instance).  Anderson mixing, 20
history vectors, cell relaxed by the stress, to 1e-10.  The solve legs
use the engine's two stabilisers for starts far from a solution (lambda
cap and history restart; the reference's iterate_AM diverges from this
random start).

--config c2: a batch of B instances of the BCC sphere phase, I m -3 m on a
32^3 grid: AB diblock f_A = 0.25, chi N = 20, ds = 0.01 (26 + 76 steps),
cubic cell a = 3.9, Anderson with cell relaxation to 1e-10, initial fields
from tanh-edged sphere densities at the BCC sites (edge width 0.05 a,
radius such that <rho_A> = f_A) plus seeded N(0, 0.01) noise (seed
20261203 + 1 + instance).  Diffuse Gaussians of width 0.3 a do not seed
the sphere phase at chi N = 20 (Anderson mixing then converges to the
disordered state).  The default run reports this workload (64 instances)
as a nested object of the C5 line.

One bench step = one Anderson iteration of the whole batch: density
(forward and backward MDE sweeps, Simpson contour integrals), stress,
deviations, Gram matrix and mixing, all on the device.  `value` counts the
MDE steps (one step_exp of one chain in one direction) processed per second
over the timed steps.  The propagator slabs (5.9 GB per C5 instance, 53 MB
per C2 instance x 64) exceed the 126 MB L2, so no L2 flush is inserted.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config c5|c2] [--batch B]
  python bench.py --impl reference   (CPU reference arm: the FP64 oracle)

Under torchrun every rank solves its own batch on its own GPU (instances
are independent: weak scaling, no data-path collective); the elapsed time
is the max over ranks.
"""
from __future__ import annotations

import argparse
import copy
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_HIST = 20
ERROR_MAX = 1e-10

# --- C2: BCC 32^3 ---------------------------------------------------------
N_GRID = 32
CELL = 3.9
F_A = 0.25
CHI_N = 20.0
DS = 0.01
SEED = 20261203 + 1
WORKLOAD_C2 = ("BCC I m -3 m 32^3 AB diblock fA=0.25 chiN=20 ds=0.01 a=3.9, Anderson n_hist=20 "
               "with cell relaxation to 1e-10")

# --- C5: ABC triblock, F d d d : 2, 64 x 128 x 224 -------------------------
C5_GRID = [64, 128, 224]
C5_CELL = [4.0, 8.0, 14.0]
C5_DS = 0.005
C5_GROUP = "F d d d : 2"
C5_SEED = 20261203 + 5
WORKLOAD_C5 = ("ABC triblock 0.3/0.4/0.3 chiN_AB=chiN_BC=30 chiN_AC=60, F d d d : 2 orthorhombic "
               "64x128x224 cell 4:8:14, ds=0.005, seeded N(0,0.5^2) fields, Anderson n_hist=20 "
               "with cell relaxation to 1e-10")
# Anderson stabilisers of the C5 solves (pscfg_am_param.mix_max / restart)
C5_AM = dict(mix_max=0.3, restart=3.0)


def make_system():
    from pscf_b200.system import Chain, System
    return System(dim=3, ngrid=[N_GRID] * 3, crystal_system="cubic", cell_param=[CELL],
                  kuhn=[1.0, 1.0], chi=[[0.0, CHI_N], [CHI_N, 0.0]],
                  chains=[Chain([0, 1], [F_A, 1.0 - F_A])], ds=DS)


def make_c5_system():
    from pscf_b200.system import Chain, System
    X = [[0.0, 30.0, 60.0], [30.0, 0.0, 30.0], [60.0, 30.0, 0.0]]
    return System(dim=3, ngrid=list(C5_GRID), crystal_system="orthorhombic", cell_param=list(C5_CELL),
                  kuhn=[1.0, 1.0, 1.0], chi=X, chains=[Chain([0, 1, 2], [0.3, 0.4, 0.3])], ds=C5_DS)


def c5_omega(system, inst):
    """chi.phi + N(0, 0.5^2) noise per monomer, projected onto F d d d : 2."""
    from pscf_b200 import groups
    rng = np.random.default_rng(C5_SEED + inst)
    w0 = system.omega_uniform()
    out = np.zeros((3, system.nr))
    for a in range(3):
        out[a] = w0[a] + groups.symmetrize(rng.normal(0.0, 0.5, size=system.nr), C5_GROUP, C5_GRID)
    return out


def initial_omega(system, inst):
    n = system.n[0]
    a = system.cell_param[0]
    x = np.arange(n) / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    d = np.full(X.shape, np.inf)
    for c in [(0.0, 0.0, 0.0), (0.5, 0.5, 0.5)]:
        dx, dy, dz = X - c[0], Y - c[1], Z - c[2]
        dx, dy, dz = dx - np.round(dx), dy - np.round(dy), dz - np.round(dz)
        d = np.minimum(d, a * np.sqrt(dx * dx + dy * dy + dz * dz))
    w = 0.05 * a
    lo, hi = 0.0, a
    for _ in range(60):
        R = 0.5 * (lo + hi)
        m = np.mean(0.5 * (1 - np.tanh((d - R) / w)))
        lo, hi = (R, hi) if m < F_A else (lo, R)
    rho_a = 0.5 * (1 - np.tanh((d - R) / w))
    delta = 0.5 * CHI_N * (1.0 - 2.0 * rho_a)
    delta -= delta.mean()
    rng = np.random.default_rng(SEED + inst)
    w0 = system.omega_uniform()
    out = np.zeros((2, system.nr))
    out[0] = w0[0] + delta.ravel() + rng.normal(0.0, 0.01, system.nr)
    out[1] = w0[1] - delta.ravel() + rng.normal(0.0, 0.01, system.nr)
    return out


class Workload:
    """One benchmark configuration: systems, initial fields, group."""

    def __init__(self, name, batch, rank):
        self.name = name
        if name == "c5":
            self.systems = [make_c5_system() for _ in range(batch)]
            self.omega0 = np.stack([c5_omega(self.systems[i], rank * batch + i) for i in range(batch)])
            self.group, self.workload, self.am = C5_GROUP, WORKLOAD_C5, dict(C5_AM)
        else:
            self.systems = [make_system() for _ in range(batch)]
            self.omega0 = np.stack([initial_omega(self.systems[i], rank * batch + i) for i in range(batch)])
            self.group, self.workload, self.am = "I m -3 m", WORKLOAD_C2, {}
        self.batch = batch
        self.cell0 = [list(s.cell_param) for s in self.systems]

    def engine(self, precision):
        from pscf_b200.engine import Engine
        e = Engine([copy.deepcopy(s) for s in self.systems], precision)
        for i in range(self.batch):
            e.set_cell_param(i, self.cell0[i])
            e.set_symmetry(i, self.group)
        return e


def c4_batches(seed_base):
    """The mixed batch: 96 lamellae (64 points, group -1), 96 hexagonal
    cylinders (p 6 m m, 64 x 64), 64 BCC spheres (I m -3 m, 32^3); AB diblocks
    with f_A ~ U[0.2, 0.5], chiN ~ U[12, 30], ds = 0.01; starting cells from
    strong-segregation scaling (chiN/20)^(1/6) times d = 1.7, a_hex = 1.9,
    a_bcc = 1.95 (half the 3.9 of the single-instance workload, which lies
    beyond the sphere phase's cell at these chiN)."""
    from pscf_b200 import guess
    from pscf_b200.batch import ShapeBatch
    from pscf_b200.system import Chain, System
    rng = np.random.default_rng(seed_base)
    out = []
    for kind, count in (("lam", 96), ("hex", 96), ("bcc", 64)):
        systems, omegas = [], []
        for i in range(count):
            fA = float(rng.uniform(0.2, 0.5))
            chiN = float(rng.uniform(12.0, 30.0))
            sc = (chiN / 20.0) ** (1.0 / 6.0)
            chi = [[0.0, chiN], [chiN, 0.0]]
            ch = [Chain([0, 1], [fA, 1.0 - fA])]
            if kind == "lam":
                s = System(1, [64], "lamellar", [1.7 * sc], [1.0, 1.0], chi, ch, DS)
                w = guess.lamellar(s, fA, noise=0.01, seed=seed_base + i)
            elif kind == "hex":
                s = System(2, [64, 64], "hexagonal", [1.9 * sc], [1.0, 1.0], chi, ch, DS)
                w = guess.cylinders(s, fA, noise=0.01, seed=seed_base + i)
            else:
                s = System(3, [32, 32, 32], "cubic", [1.95 * sc], [1.0, 1.0], chi, ch, DS)
                w = guess.spheres_bcc(s, fA, noise=0.01, seed=seed_base + i)
            systems.append(s)
            omegas.append(w)
        group = {"lam": "-1", "hex": "p 6 m m", "bcc": "I m -3 m"}[kind]
        out.append(ShapeBatch(systems, np.stack(omegas), group))
    return out


def bytes_per_step(system, wq=8, ww=8):
    """Algorithmic HBM bytes of one MDE step: read q(s), write q(s +- ds),
    read the block's omega: N_r (2 w_q + w_omega)."""
    return system.nr * (2 * wq + ww)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "", 1).isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU legs (the oracle): cpu_baseline of our arm, and the reference arm.  Both
# call cpu_mde_rate with one step per thread per round, so the two are the
# same measurement.
# ---------------------------------------------------------------------------
def cpu_mde_rate(config, nthreads, rounds):
    """MDE steps/s of the FP64 oracle's step_exp on the workload's grid: each
    round runs one step of an independent field on each of nthreads threads
    (ctypes releases the GIL; the oracle's transforms run serially within a
    thread).  Returns (rate, seconds, steps)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    O.set_fft_threads(1)
    if config == "c5":
        s = make_c5_system()
        w = c5_omega(s, 0)
    else:
        s = make_system()
        w = initial_omega(s, 0)
    o = O.Oracle(s)
    ksq = o.ksq()
    q0 = np.ones(s.nr)
    ds = s.ds
    total = 0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(nthreads) as ex:
        for _ in range(rounds):
            futs = [ex.submit(O.step, s, ksq, 1.0, ds, w[0], q0, 1) for _ in range(nthreads)]
            for f in futs:
                f.result()
            total += nthreads
    dt = time.perf_counter() - t0
    o.close()
    return total / dt, dt, total


def cpu_sample_text(config, nthreads, steps, dt):
    grid = "64x128x224" if config == "c5" else "32^3"
    return (f"{nthreads} threads, each running step_exp of the FP64 C oracle on an independent field of the "
            f"{grid} grid, one step per thread per round: {steps} steps in {dt:.1f} s (the reference "
            f"Fortran/FFTW cannot be built here)")


def run_reference(args, rank):
    """Reference arm: the reference is Fortran/FFTW and cannot be built in
    this image (no Fortran compiler, no FFTW); the FP64 C restatement of
    its propagator (oracle/) stands in, on all host threads.  Each step is
    one round of cpu_mde_rate (one step per thread)."""
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    cpu_mde_rate(args.config, nthreads, args.warmup)
    rate, secs, total_steps = cpu_mde_rate(args.config, nthreads, args.steps)
    s = make_c5_system() if args.config == "c5" else make_system()
    line = {
        "impl": "reference", "metric": "MDE steps/s", "value": rate, "unit": "MDE steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_C5 if args.config == "c5" else WORKLOAD_C2, "grid": list(s.n),
                   "contour_steps_per_chain": s.contour_steps()},
        "cpu_baseline": {"value": rate, "unit": "MDE steps/s", "cores": nthreads, "kind": "port",
                         "sample": cpu_sample_text(args.config, nthreads, total_steps, secs)},
        "e2e": {"value": rate, "unit": "MDE steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def reduce_max_sum(vals, ops, dev, world):
    """All-reduce of a few scalars with per-entry ops ('max' or 'sum')."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return [float(v) for v in vals]
    out = []
    for v, op in zip(vals, ops):
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        out.append(float(t.item()))
    return out


def timed_iterations(e, wl, steps, warmup, stream, barrier, sample_clocks, local_rank):
    """Warm-up and timed Anderson iterations of one engine (CUDA events on
    its stream).  Returns (seconds, MDE steps, profile, launches, clocks)."""
    import torch
    e.am_begin(wl.omega0, error_max=ERROR_MAX, max_itr=100000, n_hist=N_HIST, domain=True, **wl.am)
    for _ in range(warmup):
        e.am_iterate(1)
    barrier()
    sampler = ClockSampler(local_rank) if sample_clocks else None
    if sampler:
        sampler.start()
    l0 = e.launch_count
    e.set_profiling(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        e.am_iterate(1)
    ev1.record(stream)
    barrier()
    clocks = sampler.stop() if sampler else None
    prof = e.profile()
    e.set_profiling(False)
    return ev0.elapsed_time(ev1) / 1e3, prof["steps"], prof, e.launch_count - l0, clocks


def roofline(system, prof, steps_done, peak, peak_kind, wq, kernel):
    bstep = bytes_per_step(system, wq=wq)
    sweep_s = prof["sweep_ms"] / 1e3
    achieved = steps_done * bstep / sweep_s / 1e9 if sweep_s > 0 else None
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
            "traffic": None, "kernel": kernel, "bytes_per_step": bstep,
            "sweep_ms": prof["sweep_ms"], "steps": steps_done}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from pscf_b200.engine import FP64

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    B = args.batch if args.batch else (1 if args.config == "c5" else 64)
    wl = Workload(args.config, B, rank)
    e = wl.engine(FP64)
    stream = torch.cuda.ExternalStream(e.stream, device=dev)

    # ---- timed Anderson iterations -------------------------------------
    secs, steps_done, prof, launches, clocks = timed_iterations(e, wl, args.steps, args.warmup, stream, barrier,
                                                                True, local_rank)
    elapsed, total_steps = reduce_max_sum([secs, steps_done], ["max", "sum"], dev, world)
    value = total_steps / elapsed

    # ---- end to end, converged solves, the nested workloads -------------
    e2e_value, e2e_bytes = e2e_leg(e, wl, args, stream, barrier, dev, world)
    run_solve = (args.config == "c2" and not args.no_solve) or args.c5_solve
    solve = solve_legs(e, wl, stream, barrier, dev, world) if run_solve else None
    e.close()
    mixed_iter = fp32_iteration_leg(wl, args, barrier, dev, world, local_rank, elapsed / args.steps,
                                    steps_done / (prof["sweep_ms"] / 1e3))
    nested = {}
    if args.config == "c5" and not args.no_c2:
        nested["c2_bcc32_x64"] = c2_leg(args, rank, world, barrier, dev, local_rank)
    if not args.no_c4:
        nested["mixed_shape_batch"] = c4_leg(rank, world, barrier, dev, args.c4_graph_check)

    if rank != 0:
        return
    s0 = wl.systems[0]
    peak, peak_kind = measured_peaks()
    kernel = ("MDE step: k3p_final_fwd + k3p_zconv x2 + k3p_mid (kernels3p.cuh, 64x128x224)" if args.config == "c5"
              else "MDE step: k3r_final_fwd + k3s_zconv x2 + k3r_inv_mid (kernels3c.cuh, 32^3)")
    cpu = None
    if world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        rate, dt, nst = cpu_mde_rate(args.config, nthreads, 2)
        cpu = {"value": rate, "unit": "MDE steps/s", "cores": nthreads, "kind": "port",
               "sample": cpu_sample_text(args.config, nthreads, nst, dt)}
    line = {
        "metric": "MDE steps/s", "value": value, "unit": "MDE steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.workload, "batch_per_gpu": B, "grid": list(s0.n),
                   "contour_steps_per_chain": s0.contour_steps(), "parallelism": f"instances x{world}",
                   "l2": "inputs larger than L2 (propagator slabs %.1f GB per GPU)"
                         % (B * 2 * (s0.contour_steps() + 1) * s0.nr * 8 / 1e9)},
    }
    if solve is not None:
        if args.config == "c5":
            line["c5_solve"] = solve
        else:
            line.update(solve)
    if "mixed_precision" in line:
        line["mixed_precision"].update(mixed_iter)
    else:
        line["mixed_precision"] = mixed_iter
    line.update({
        "e2e": {"value": e2e_value, "unit": "MDE steps/s", "api": "pscfg_density + pscfg_stress (host buffers)",
                "h2d_bytes_per_step": e2e_bytes[0], "d2h_bytes_per_step": e2e_bytes[1]},
        "roofline": roofline(s0, prof, steps_done, peak, peak_kind, 8, kernel),
        "phase_ms": {k: prof[k] for k in ("sweep_ms", "contour_ms", "stress_ms")},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
    })
    line.update(nested)
    print(json.dumps(line), flush=True)


def fp32_iteration_leg(wl, args, barrier, dev, world, local_rank, fp64_iter_s, fp64_sweep_rate):
    """The same Anderson iterations with FP32 propagation (FP64 contour sums,
    mixing and stress): per-iteration time against FP64, the ceiling of any
    mixed-precision speed-up on this workload."""
    import torch
    from pscf_b200.engine import FP32
    e32 = wl.engine(FP32)
    s32 = torch.cuda.ExternalStream(e32.stream, device=dev)
    steps = max(3, min(args.steps, 10))
    secs, n32, p32, _, _ = timed_iterations(e32, wl, steps, 3, s32, barrier, False, local_rank)
    e32.close()
    secs, = reduce_max_sum([secs], ["max"], dev, world)
    it32 = secs / steps
    return {"fp64_iteration_ms": 1e3 * fp64_iter_s, "fp32_iteration_ms": 1e3 * it32,
            "per_iteration_speedup_fp32": fp64_iter_s / it32,
            "fp64_sweep_steps_per_s": fp64_sweep_rate, "fp32_sweep_steps_per_s": n32 / (p32["sweep_ms"] / 1e3)}


def solve_legs(e, wl, stream, barrier, dev, world):
    """Full solves of the batch from its initial fields and cells: FP64 (in
    engine e), then mixed FP32 -> FP64 in a second engine.  Reports the
    mixed solve's error against the FP64 one: |dF|, max |d phi| and
    max |d stress|."""
    import torch
    from pscf_b200.engine import MIXED
    B = wl.batch
    for i in range(B):
        e.set_cell_param(i, wl.cell0[i])
    max_itr = 4000
    barrier()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    e.am_begin(wl.omega0, error_max=ERROR_MAX, max_itr=max_itr, n_hist=N_HIST, domain=True, **wl.am)
    while e.am_iterate(8) > 0:
        pass
    ev3.record(stream)
    barrier()
    solve_s = ev2.elapsed_time(ev3) / 1e3
    _, rho64, res = e.am_results(want_fields=True)
    conv = sum(1 for r in res if r["converged"])
    itrs = [r["itr"] for r in res]

    em = wl.engine(MIXED)
    streamm = torch.cuda.ExternalStream(em.stream, device=dev)
    barrier()
    ev6, ev7 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev6.record(streamm)
    em.am_begin(wl.omega0, error_max=ERROR_MAX, max_itr=max_itr, n_hist=N_HIST, domain=True,
                switch_error=1e-6 if wl.name == "c5" else 0.0, **wl.am)
    while em.am_iterate(8) > 0:
        pass
    ev7.record(streamm)
    barrier()
    mixed_s = ev6.elapsed_time(ev7) / 1e3
    _, rhom, resm = em.am_results(want_fields=True)
    em.close()
    convm = sum(1 for r in resm if r["converged"])
    both = [(a, b) for a, b in zip(res, resm) if a["converged"] and b["converged"]]
    dF = max((abs(a["f_helmholtz"] - b["f_helmholtz"]) for a, b in both), default=float("nan"))
    dst = max((max(abs(x - y) for x, y in zip(a["stress"], b["stress"])) for a, b in both), default=float("nan"))
    dphi = float(np.max(np.abs(rho64 - rhom))) if both else float("nan")
    itr32 = float(np.mean([r["itr_fp32"] for r in resm]))
    itrm = float(np.mean([r["itr"] for r in resm]))
    solve_s, conv, mixed_s, convm, dF, dphi, dst = reduce_max_sum(
        [solve_s, conv, mixed_s, convm, dF, dphi, dst], ["max", "sum", "max", "sum", "max", "max", "max"], dev, world)
    rate64 = conv / solve_s
    ratem = convm / mixed_s
    return {
        "solves_per_s": rate64, "solve_seconds": solve_s, "solves_converged": int(conv),
        "solve_iterations": {"min": int(min(itrs)), "max": int(max(itrs)), "mean": float(np.mean(itrs))},
        "mixed_precision": {"solves_per_s": ratem, "speedup_vs_fp64": (ratem / rate64) if rate64 > 0 else None,
                            "seconds": mixed_s, "solves_converged": int(convm),
                            "mean_iterations": itrm, "mean_fp32_iterations": itr32,
                            "switch_error": 1e-6 if wl.name == "c5" else 1e-3,
                            "max_abs_dF_vs_fp64": dF, "max_abs_dphi_vs_fp64": dphi,
                            "max_abs_dstress_vs_fp64": dst},
        "f_helmholtz": {"min": float(min(r["f_helmholtz"] for r in res)),
                        "max": float(max(r["f_helmholtz"] for r in res))},
        "cell_param": [r["cell_param"] for r in res][:4],
    }


def e2e_leg(e, wl, args, stream, barrier, dev, world):
    """MDE steps/s through the C ABI (pscfg_density + pscfg_stress) with
    pinned host buffers: host->device fields and device->host densities,
    Q and stress inside the timed region.  Returns (value, (h2d, d2h))."""
    import ctypes as C
    import torch
    omega0 = wl.omega0
    B = wl.batch
    w_pin = torch.from_numpy(omega0.copy()).pin_memory()
    rho_pin = torch.empty_like(w_pin).pin_memory()
    q = np.zeros((B, 4))
    lib = e.lib
    dp = C.POINTER(C.c_double)
    wp = C.cast(w_pin.data_ptr(), dp)
    rp = C.cast(rho_pin.data_ptr(), dp)
    stress = np.zeros((B, 6))
    for _ in range(2):
        e._check(lib.pscfg_density(e._h, wp, rp, q.ctypes.data_as(dp), None))
    barrier()
    n_e2e = max(2, min(args.steps, 5))
    ev4, ev5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev4.record(stream)
    for _ in range(n_e2e):
        e._check(lib.pscfg_density(e._h, wp, rp, q.ctypes.data_as(dp), None))
        e._check(lib.pscfg_stress(e._h, stress.ctypes.data_as(dp)))
    ev5.record(stream)
    barrier()
    e2e_s, = reduce_max_sum([ev4.elapsed_time(ev5) / 1e3], ["max"], dev, world)
    value = world * n_e2e * e.steps_per_density / e2e_s
    return value, (int(omega0.nbytes), int(omega0.nbytes + q.nbytes + stress.nbytes))


def c2_leg(args, rank, world, barrier, dev, local_rank):
    """The BCC 32^3 batch of 64: MDE steps/s of timed Anderson iterations
    (FP64, and FP32 propagation for the sweep rate), converged solves/s
    FP64 and mixed."""
    import torch
    from pscf_b200.engine import FP64
    wl = Workload("c2", 64, rank)
    e = wl.engine(FP64)
    stream = torch.cuda.ExternalStream(e.stream, device=dev)
    steps = 10
    secs, nsteps, prof, launches, _ = timed_iterations(e, wl, steps, 3, stream, barrier, False, local_rank)
    elapsed, total = reduce_max_sum([secs, nsteps], ["max", "sum"], dev, world)
    peak, peak_kind = measured_peaks()
    out = {"workload": WORKLOAD_C2, "batch_per_gpu": 64, "value": total / elapsed, "unit": "MDE steps/s",
           "ms_per_step": 1e3 * elapsed / steps, "steps": steps,
           "roofline": roofline(wl.systems[0], prof, nsteps, peak, peak_kind, 8,
                                "MDE step: k3r_final_fwd + k3s_zconv x2 + k3r_inv_mid (kernels3c.cuh, 32^3)"),
           "sweep_steps_per_s_fp64": nsteps / (prof["sweep_ms"] / 1e3),
           "planes_per_cta": e.sweep_planes(2 * len(wl.systems))}
    if not args.no_solve:
        out.update(solve_legs(e, wl, stream, barrier, dev, world))
    e.close()
    mi = fp32_iteration_leg(wl, args, barrier, dev, world, local_rank, elapsed / steps,
                            out["sweep_steps_per_s_fp64"])
    out.setdefault("mixed_precision", {}).update(mi)
    return out


def c4_leg(rank, world, barrier, dev, graph_check=0):
    """Concurrent solve of the mixed-shape batch (one engine and stream per
    grid shape), wall clock; graph_check > 0 runs the iterations from
    captured graphs with the Anderson step on the device."""
    import torch
    import torch.distributed as dist
    from pscf_b200.batch import solve_batches
    batches = c4_batches(20261203 + 3 + 1000 * rank)
    barrier()
    t0 = time.perf_counter()
    results = solve_batches(batches, error_max=1e-9, max_itr=1000, n_hist=20, domain=True,
                            graph_check=graph_check)
    torch.cuda.synchronize()
    c4_s = time.perf_counter() - t0
    nconv = sum(1 for rs in results for r in rs if r["converged"])
    ninst = sum(len(rs) for rs in results)
    tc = torch.tensor([c4_s, float(nconv), float(ninst)], dtype=torch.float64, device=dev)
    if world > 1:
        for k, op in ((0, dist.ReduceOp.MAX), (1, dist.ReduceOp.SUM), (2, dist.ReduceOp.SUM)):
            x = tc[k:k + 1].clone()
            dist.all_reduce(x, op=op)
            tc[k] = x[0]
    out = {"instances": int(tc[2].item()), "converged": int(tc[1].item()), "seconds": float(tc[0].item()),
           "solves_per_s": float(tc[1].item()) / float(tc[0].item()),
           "per_shape_converged": [sum(1 for r in rs if r["converged"]) for rs in results],
           "graph_check": graph_check,
           "note": "wall clock of concurrent engines (one host thread and stream per grid shape)"}
    for b in batches:
        b.engine.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c5", choices=["c5", "c2"])
    ap.add_argument("--batch", type=int, default=0, help="instances per GPU (default: 1 for c5, 64 for c2)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-c2", action="store_true", help="skip the nested BCC 32^3 x 64 leg")
    ap.add_argument("--no-c4", action="store_true", help="skip the mixed-shape batch leg")
    ap.add_argument("--c4-graph-check", type=int, default=0,
                    help="mixed-shape batch: iterations per host check of the graph-driven Anderson loop "
                         "(0: host-driven iterations)")
    ap.add_argument("--no-solve", action="store_true",
                    help="time the Anderson iterations only (no full FP64 / mixed solves; profiling runs)")
    ap.add_argument("--ds", type=float, default=0.0,
                    help="contour step override (profiling runs on a short contour; same kernels per step)")
    ap.add_argument("--c5-solve", action="store_true",
                    help="also run the full FP64 and mixed-precision solves of the C5 workload (minutes)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.ds > 0:
        global DS, C5_DS
        DS = C5_DS = args.ds
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
