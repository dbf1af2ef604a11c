#!/usr/bin/env python
"""Benchmark: MDE contour steps/s and converged SCFT solves/s on one node.

Workload (per GPU): a batch of B instances of the BCC sphere phase,
space group I m -3 m on a 32^3 grid: AB diblock f_A = 0.25, chi N = 20,
b_A = b_B = 1, ds = 0.01 (26 + 76 contour steps), cubic cell a = 3.9,
Anderson mixing with 20 history vectors, cell relaxed by the stress, to a
residual of 1e-10.  Initial fields from sphere densities at the BCC sites:
rho_A = (1 - tanh((d - R)/w))/2 with d the distance to the nearest site,
edge width w = 0.05 a and R set so that <rho_A> = f_A (a density swing of
1.0), omega_A - omega_B = chiN (1 - 2 rho_A) around the uniform values
chiN phi_B, chiN phi_A, plus seeded N(0, 0.01) noise (seed
20261203 + 1 + instance).  Diffuse Gaussians of width 0.3 a do not seed the
sphere phase at chiN = 20 (Anderson mixing then converges to the
disordered state); the sharp profile converges to BCC from the starting
cell a = 3.9 (relaxed cell 1.9232, F = 2.6145888805).

One bench step = one Anderson iteration of the whole batch: density
(forward and backward MDE sweeps, Simpson contour integrals), stress,
deviations, Gram matrix and mixing, all on the device.  `value` counts the
MDE steps (one step_exp of one chain in one direction) processed per second
over the timed steps.  The batch's propagator slabs (about 53 MB per
instance) exceed the 126 MB L2, so no L2 flush is inserted.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B]
  python bench.py --impl reference   (CPU reference arm: the FP64 oracle)

Under torchrun every rank solves its own batch on its own GPU (instances
are independent: weak scaling, no data-path collective); the elapsed time
is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 32
CELL = 3.9
F_A = 0.25
CHI_N = 20.0
DS = 0.01
N_HIST = 20
ERROR_MAX = 1e-10
SEED = 20261203 + 1
WORKLOAD = ("BCC I m -3 m 32^3 AB diblock fA=0.25 chiN=20 ds=0.01 a=3.9, Anderson n_hist=20 "
            "with cell relaxation to 1e-10")


def make_system():
    from pscf_b200.system import Chain, System
    return System(dim=3, ngrid=[N_GRID] * 3, crystal_system="cubic", cell_param=[CELL],
                  kuhn=[1.0, 1.0], chi=[[0.0, CHI_N], [CHI_N, 0.0]],
                  chains=[Chain([0, 1], [F_A, 1.0 - F_A])], ds=DS)


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


def ncu_traffic_per_step():
    """DRAM bytes per MDE step of the sweep kernels from the committed ncu
    summary (profiles/mde_step_bcc32_fp64.md, line 'traffic_bytes_per_step:')."""
    path = os.path.join(ROOT, "profiles", "mde_step_bcc32_fp64.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_step:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# CPU legs (the oracle): cpu_baseline of our arm, and the reference arm
# ---------------------------------------------------------------------------
def cpu_mde_rate(nthreads, nsteps_per_thread, min_seconds=0.0):
    """MDE steps/s of the FP64 oracle's step_exp on the 32^3 C2 grid, one
    field per thread (ctypes releases the GIL), repeated in rounds of
    nsteps_per_thread steps per thread until min_seconds have passed.
    Returns (rate, seconds)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    s = make_system()
    o = O.Oracle(s)
    ksq = o.ksq()
    w = initial_omega(s, 0)
    q0 = np.ones(s.nr)
    O.step(s, ksq, 1.0, 0.01, w[0], q0, 1)   # load / warm
    total = 0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(nthreads) as ex:
        while total == 0 or time.perf_counter() - t0 < min_seconds:
            futs = [ex.submit(O.step, s, ksq, 1.0, 0.01, w[0], q0, nsteps_per_thread) for _ in range(nthreads)]
            for f in futs:
                f.result()
            total += nthreads * nsteps_per_thread
    dt = time.perf_counter() - t0
    return total / dt, dt


def run_reference(args, rank):
    """Reference arm: the reference is Fortran/FFTW and cannot be built in
    this image (no Fortran compiler, no FFTW); the FP64 C restatement of
    its propagator (oracle/) stands in, on all host threads."""
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    per, step_seconds = 2, 5.0
    for _ in range(args.warmup):
        cpu_mde_rate(nthreads, per, step_seconds)
    secs = 0.0
    total_steps = 0
    for _ in range(args.steps):
        r, dt = cpu_mde_rate(nthreads, per, step_seconds)
        secs += dt
        total_steps += r * dt
    value = total_steps / secs
    s = make_system()
    line = {
        "impl": "reference", "metric": "MDE steps/s", "value": value, "unit": "MDE steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": [N_GRID] * 3, "contour_steps_per_chain": s.contour_steps()},
        "cpu_baseline": {"value": value, "unit": "MDE steps/s", "cores": nthreads, "kind": "port",
                         "sample": f"each step: {nthreads} threads running step_exp of the FP64 C oracle on the 32^3 "
                                   f"grid for >= {step_seconds:.0f} s (the reference Fortran/FFTW cannot be "
                                   f"built here)"},
        "e2e": {"value": value, "unit": "MDE steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from pscf_b200.engine import Engine, FP64

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    B = args.batch
    systems = [make_system() for _ in range(B)]
    omega0 = np.stack([initial_omega(systems[i], rank * B + i) for i in range(B)])
    e = Engine(systems, FP64)
    for i in range(B):
        e.set_symmetry(i, "I m -3 m")
    stream = torch.cuda.ExternalStream(e.stream, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- timed Anderson iterations -------------------------------------
    e.am_begin(omega0, error_max=ERROR_MAX, max_itr=10000, n_hist=N_HIST, domain=True)
    for _ in range(args.warmup):
        e.am_iterate(1)
    barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    l0 = e.launch_count
    e.set_profiling(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        e.am_iterate(1)
    ev1.record(stream)
    barrier()
    clocks = sampler.stop()
    prof = e.profile()
    e.set_profiling(False)
    launches = e.launch_count - l0
    ms = ev0.elapsed_time(ev1)
    steps_done = prof["steps"]
    t = torch.tensor([ms / 1e3, float(steps_done)], dtype=torch.float64, device=dev)
    if world > 1:
        tmax = t[0:1].clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        tsum = t[1:2].clone()
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        elapsed, total_steps = float(tmax.item()), float(tsum.item())
    else:
        elapsed, total_steps = ms / 1e3, float(steps_done)
    value = total_steps / elapsed

    # ---- converged solves/s, mixed precision, end to end, mixed shapes ----
    solve = None if args.no_solve else solve_legs(e, systems, omega0, B, stream, barrier, dev, world)
    e2e_value, e2e_bytes = e2e_leg(e, omega0, B, args, stream, barrier, dev, world)
    c4 = None if args.no_c4 else c4_leg(rank, world, barrier, dev)

    if rank != 0:
        return
    s0 = systems[0]
    bstep = bytes_per_step(s0)
    peak, peak_kind = measured_peaks()
    sweep_s = prof["sweep_ms"] / 1e3
    achieved = steps_done * bstep / sweep_s / 1e9 if sweep_s > 0 else None
    traffic = ncu_traffic_per_step()
    cpu = None
    if world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        rate, dt = cpu_mde_rate(nthreads, 4, 10.0)
        cpu = {"value": rate, "unit": "MDE steps/s", "cores": nthreads, "kind": "port",
               "sample": f"{nthreads} threads running step_exp of the FP64 C oracle on the 32^3 grid, "
                         f"{round(rate * dt)} steps in {dt:.1f} s"}
    line = {
        "metric": "MDE steps/s", "value": value, "unit": "MDE steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch_per_gpu": B, "grid": [N_GRID] * 3,
                   "contour_steps_per_chain": s0.contour_steps(), "parallelism": f"instances x{world}",
                   "l2": "inputs larger than L2 (propagator slabs %.1f GB per GPU)" % (B * 2 * 103 * s0.nr * 8 / 1e9)},
    }
    if solve is not None:
        line.update(solve)
    line.update({
        "e2e": {"value": e2e_value, "unit": "MDE steps/s", "api": "pscfg_density + pscfg_stress (host buffers)",
                "h2d_bytes_per_step": e2e_bytes[0], "d2h_bytes_per_step": e2e_bytes[1]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                     "traffic": traffic, "kernel": "MDE step (sweep kernels)",
                     "bytes_per_step": bstep, "sweep_ms": prof["sweep_ms"], "steps": steps_done},
        "phase_ms": {k: prof[k] for k in ("sweep_ms", "contour_ms", "stress_ms")},
        "mixed_shape_batch": c4,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
    })
    print(json.dumps(line), flush=True)


def solve_legs(e, systems, omega0, B, stream, barrier, dev, world):
    """Full solves of the batch from the starting cell: FP64, then mixed
    FP32 -> FP64 in a second engine.  Returns the JSON keys of both."""
    import torch
    import torch.distributed as dist
    from pscf_b200.engine import Engine, MIXED
    for i in range(B):                     # back to the starting cell a = 3.9
        e.set_cell_param(i, [CELL])
    barrier()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    e.am_begin(omega0, error_max=ERROR_MAX, max_itr=2000, n_hist=N_HIST, domain=True)
    while e.am_iterate(8) > 0:
        pass
    ev3.record(stream)
    barrier()
    solve_s = ev2.elapsed_time(ev3) / 1e3
    _, _, res = e.am_results(want_fields=False)
    conv = sum(1 for r in res if r["converged"])
    itrs = [r["itr"] for r in res]
    fvals = [r["f_helmholtz"] for r in res]
    cells = [r["cell_param"][0] for r in res]
    ts = torch.tensor([solve_s, float(conv)], dtype=torch.float64, device=dev)
    if world > 1:
        smax = ts[0:1].clone()
        dist.all_reduce(smax, op=dist.ReduceOp.MAX)
        csum = ts[1:2].clone()
        dist.all_reduce(csum, op=dist.ReduceOp.SUM)
        solve_s_all, conv_all = float(smax.item()), float(csum.item())
    else:
        solve_s_all, conv_all = solve_s, float(conv)

    em = Engine(systems, MIXED)
    for i in range(B):
        em.set_symmetry(i, "I m -3 m")
    streamm = torch.cuda.ExternalStream(em.stream, device=dev)
    barrier()
    ev6, ev7 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev6.record(streamm)
    em.am_begin(omega0, error_max=ERROR_MAX, max_itr=2000, n_hist=N_HIST, domain=True)
    while em.am_iterate(8) > 0:
        pass
    ev7.record(streamm)
    barrier()
    mixed_s = ev6.elapsed_time(ev7) / 1e3
    _, _, resm = em.am_results(want_fields=False)
    convm = sum(1 for r in resm if r["converged"])
    dF = max(abs(a["f_helmholtz"] - b["f_helmholtz"]) for a, b in zip(res, resm))
    itr32 = float(np.mean([r["itr_fp32"] for r in resm]))
    tm = torch.tensor([mixed_s, float(convm), dF], dtype=torch.float64, device=dev)
    if world > 1:
        for k, op in ((0, dist.ReduceOp.MAX), (1, dist.ReduceOp.SUM), (2, dist.ReduceOp.MAX)):
            x = tm[k:k + 1].clone()
            dist.all_reduce(x, op=op)
            tm[k] = x[0]
    em.close()
    mixed_rate = float(tm[1].item()) / float(tm[0].item())
    return {
        "solves_per_s": conv_all / solve_s_all, "solve_seconds": solve_s_all, "solves_converged": int(conv_all),
        "solve_iterations": {"min": int(min(itrs)), "max": int(max(itrs)), "mean": float(np.mean(itrs))},
        "mixed_precision": {"solves_per_s": mixed_rate, "speedup_vs_fp64": mixed_rate / (conv_all / solve_s_all),
                            "max_abs_dF_vs_fp64": float(tm[2].item()), "mean_fp32_iterations": itr32,
                            "solves_converged": int(tm[1].item())},
        "f_helmholtz": {"min": float(min(fvals)), "max": float(max(fvals))},
        "cell_param": {"min": float(min(cells)), "max": float(max(cells))},
    }


def e2e_leg(e, omega0, B, args, stream, barrier, dev, world):
    """MDE steps/s through the C ABI (pscfg_density + pscfg_stress) with
    pinned host buffers: host->device fields and device->host densities,
    Q and stress inside the timed region.  Returns (value, (h2d, d2h))."""
    import ctypes as C
    import torch
    import torch.distributed as dist
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
    e2e_s = ev4.elapsed_time(ev5) / 1e3
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    value = world * n_e2e * e.steps_per_density / float(te.item())
    return value, (int(omega0.nbytes), int(omega0.nbytes + q.nbytes + stress.nbytes))


def c4_leg(rank, world, barrier, dev):
    """Concurrent solve of the mixed-shape batch (one engine and stream per
    grid shape), wall clock."""
    import torch
    import torch.distributed as dist
    from pscf_b200.batch import solve_batches
    batches = c4_batches(20261203 + 3 + 1000 * rank)
    barrier()
    t0 = time.perf_counter()
    results = solve_batches(batches, error_max=1e-9, max_itr=1000, n_hist=20, domain=True)
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
           "note": "wall clock of concurrent engines (one host thread and stream per grid shape)"}
    for b in batches:
        b.engine.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the mixed-shape batch leg")
    ap.add_argument("--no-solve", action="store_true",
                    help="time the Anderson iterations only (no full FP64 / mixed solves; profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
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
