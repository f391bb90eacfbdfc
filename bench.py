#!/usr/bin/env python
"""bench.py -- steps/s of sma-dft's advected (adv) time step at 256^3 on B200.

Metric (the reference's headline path): steps/s at 256^3 adv, mixed precision (FP32 fields,
FP64 spectral state, update and reductions) against the plain FP64 GPU step, with the
relative L2 error of psi against FP64 stated.  Workload: adv/cosAdvTrackMult.cpp-style step,
256x256x256, dx = lambda0/8, dt = 0.01, nu = 1, eps = -0.75, alpha = 1, beta = 2, gamma = 1;
synthetic seeded IC (smectic layers with 4 focal-conic-like perturbations, built in numpy by
make_ic).  dt = 0.01 rather than the configuration's 0.02: at dx = lambda0/8 the scheme
diverges at 0.02 (the reference build does too); the cost of a step does not depend on dt.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  The path does not shard (one simulation per GPU,
"replicas only"): every rank runs its own replica, value = all ranks' steps / max time.
``--impl reference`` times the reference's own loop body (oracle/_ref/adv_ref: the
reference sources compiled with single-rank MPI / FFTW-r2r shims) on the host cores, for the
same K steps after W untimed ones; it never loads the product library.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "sma-dft_b200"))

METRIC = "steps/s at 256^3 adv: mixed-prec vs FP64 GPU, at stated L2 err vs FP64"
N = 256
# dt = 0.01: with dx = lambda0/8 and this initial condition the adv scheme diverges (psi
# non-finite before step 1000, FP64 and FP32 alike) at dt = 0.02; 0.01 runs 10^4 steps.
# The cost of a step does not depend on dt.
CFG = dict(nw=8.0, dt=0.01, eps=-0.75, nu=1.0, alpha=1.0, beta=2.0, gamma=1.0)
ERR_STEPS = 10000   # steps after which the FP32 psi is compared with the FP64 psi
F_ADV = 32          # compulsory full-field transfers per adv step (single-sweep stages)
# the kernel the roofline object describes, its key in pass_kernels and its ncu summary
DOMINANT_PASS = "x_dct3"
DOMINANT_PROFILE = "r2r_rd_x_pass_dct3_256cube_fp32.md"
DOMINANT_KERNEL = ("r2r_rd_kernel<float,256,x,DCT-III> plain inverse pass along x (the largest share of the adv "
                   "step's device time); algorithmic bytes per launch = 2 x 4 B x 256^3, 6-field ring")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of one GPU, polled through NVML every
    2 ms on a host thread (reads only; no setting of the GPU is touched).

    ``mark(t0, t1)`` keeps the samples taken inside the timed region (host wall clock); a
    timed region of a few tens of milliseconds still holds a dozen samples.  The GPU is found
    by the UUID torch reports for the CUDA device, so it is the right one under
    CUDA_VISIBLE_DEVICES.
    """

    INTERVAL_S = 0.002
    NAMES = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
             ("sw_power_cap", 0x4))

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.samples: list[tuple[float, int, int]] = []
        self.window = (0.0, float("inf"))
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        self._nvml = pynvml
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def __enter__(self):
        try:
            h = self._handle()
            nv = self._nvml
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))

            def poll():
                while not self._stop.is_set():
                    try:
                        mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((time.time(), int(mhz), int(rs)))
                    except Exception:
                        pass
                    time.sleep(self.INTERVAL_S)
            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5.0:
                time.sleep(0.001)
        except Exception:
            self._thread = None
        return self

    def mark(self, t0: float, t1: float):
        self.window = (t0, t1)

    def __exit__(self, *a):
        self._stop.set()
        if self._thread is not None:
            self._thread.join(timeout=2.0)
        if self._nvml is not None:
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self) -> dict:
        lo, hi = self.window
        inside = [(mhz, rs) for ts, mhz, rs in self.samples if lo <= ts <= hi]
        reasons = sorted({nm for _, rs in inside for nm, bit in self.NAMES if rs & bit})
        return {"sm_mhz": statistics.median([m for m, _ in inside]) if inside else None,
                "sm_max_mhz": self.max_mhz, "reasons": reasons, "samples": len(inside),
                "interval_ms": 1000 * self.INTERVAL_S, "source": "NVML"}


def cpu_reference_run(steps: int, psi0: np.ndarray, threads: int):
    """Run the shimmed reference adv loop at 256^3; returns (steps/s, seconds, kind, sample).

    The reference's own sources (adv/cosAdvTrackMult.cpp) compiled with the single-rank MPI /
    FFTW-r2r shim (oracle/_ref/adv_ref), timed by the reference's own wall clock around its
    loop; where that build is absent, the FP64 oracle port of the same loop."""
    import oracle
    shape = (N, N, N)
    if oracle.reference_available("adv"):
        with tempfile.TemporaryDirectory() as wd:
            t0 = time.time()
            _, _, out = oracle.run_reference("adv", shape, steps, psi0=psi0, workdir=wd,
                                             threads=threads, **{k: v for k, v in CFG.items()
                                                                 if k in ("nw", "dt", "eps", "nu")})
            wall = time.time() - t0
        m = re.search(r"Finished in ([0-9.eE+-]+) seconds \[Wall Clock\]", out)
        secs = float(m.group(1)) if m else wall
        return steps / secs, secs, "reference", (
            f"{steps} steps of the reference adv loop body at 256^3 (adv/cosAdvTrackMult.cpp, "
            f"single-rank shim, FFTW replaced by the oracle FP64 r2r, {threads} OpenMP threads), "
            f"timed by its own wall clock")
    o = oracle.Oracle(oracle.ADV, shape, **{k: v for k, v in CFG.items()})
    o.set_psi(psi0)
    t0 = time.perf_counter()
    o.step(steps)
    secs = time.perf_counter() - t0
    return steps / secs, secs, "port", f"{steps} steps of the FP64 oracle adv step at 256^3, {threads} threads"


def _mix64(z):
    """SplitMix64 finaliser (Steele, Lea, Flood 2014) on uint64 arrays (wrapping arithmetic)."""
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _uniform(seed: int, ctr):
    """Uniform in [0, 1) from (seed, counter): the counter-based stream of the product's IC
    builders (csrc/ic.cpp), so host and library make identical noise."""
    x = _mix64(np.uint64(seed) ^ _mix64(np.asarray(ctr, dtype=np.uint64)))
    return (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def make_ic(shape=(N, N, N), A=1.328, count=4, rmin=3.0, rmax=6.0, noise=1e-3, seed=20240601):
    """Config 3's synthetic initial condition, built on the host in numpy: smectic layers
    A cos(q0 z) over the smectic half x < L/2 (tanh envelope of width 2 lambda0) with `count`
    radial focal perturbations (radius rmin..rmax lambda0, centres uniform in the smectic
    half, blended over one wavelength), plus seeded uniform noise.  The same construction as
    smadft_ic_conics (node positions x_i = i dx, as adv/cosAdvTrackMult.cpp:500-536 writes its
    layers); both arms of the benchmark use this array, so the reference arm never loads the
    product library."""
    nw, q0 = CFG["nw"], 1.0
    nx, ny, nz = shape
    dx = 2.0 * np.pi / (q0 * nw)
    Lx, Ly, Lz = nx * dx, ny * dx, nz * dx
    lam0 = 2.0 * np.pi / q0
    base = 0x5A5A0000 + 16 * np.arange(count, dtype=np.uint64)
    cx = _uniform(seed, base + np.uint64(0)) * 0.5 * Lx
    cy = _uniform(seed, base + np.uint64(1)) * Ly
    cz = _uniform(seed, base + np.uint64(2)) * Lz
    R = (rmin + (rmax - rmin) * _uniform(seed, base + np.uint64(3))) * lam0
    x = (np.arange(nx) * dx)[:, None, None]
    y = (np.arange(ny) * dx)[None, :, None]
    z = (np.arange(nz) * dx)[None, None, :]
    layer = np.cos(q0 * z) * np.ones((nx, ny, 1))
    for c in range(count):
        d = np.sqrt((x - cx[c]) * (x - cx[c]) + (y - cy[c]) * (y - cy[c]) + (z - cz[c]) * (z - cz[c]))
        w = 0.5 * (1.0 - np.tanh((d - R[c]) / lam0))
        layer = w * np.cos(q0 * d) + (1.0 - w) * layer
    env = 0.5 * (1.0 - np.tanh((x - 0.5 * Lx) / (2.0 * lam0)))
    psi = A * layer * env
    if noise != 0.0:
        psi = psi + noise * (2.0 * _uniform(seed, np.arange(nx * ny * nz, dtype=np.uint64)).reshape(shape) - 1.0)
    return np.ascontiguousarray(psi)


def bench_config(world: int) -> dict:
    """The workload both arms run (identical in both JSON lines)."""
    return {"workload": "adv 256^3 time step (cosAdvTrackMult-style)",
            "grid": [N, N, N], "dt": CFG["dt"], "dx": "lambda0/8", "nu": CFG["nu"], "eps": CFG["eps"],
            "ic": "smectic layers + 4 seeded focal perturbations (radius 3-6 lambda0), noise 1e-3, seed 20240601",
            "parallelism": f"replicas x{world}",
            "l2_flush": "inputs larger than L2 (about 1 GB of fields touched per step)"}


def run_reference_arm(args, rank, world):
    """The reference's own loop body on the host cores: W untimed steps in one process, then
    the K timed steps in a second one (the reference times its loop with its own wall clock),
    all host threads.  Rank 0 alone runs and prints; other ranks exit without work."""
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    psi0 = make_ic()
    if args.warmup > 0:
        cpu_reference_run(args.warmup, psi0, threads)
    sps, secs, kind, sample = cpu_reference_run(args.steps, psi0, threads)
    line = {
        "metric": METRIC, "value": sps, "unit": "steps/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(world),
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(torch, dist, values, device):
    """Element-wise maximum of a list of floats over all ranks (one all-reduce on `device`:
    "cuda" under NCCL, "cpu" under gloo)."""
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def partition_by_cost(costs, world: int, rank: int):
    """Indices of the runs rank `rank` takes: greedy, largest cost first, each to the least
    loaded rank (no collective; every rank computes the same split)."""
    load = [0.0] * world
    mine = []
    for idx in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda w: (load[w], w))
        load[r] += costs[idx]
        if r == rank:
            mine.append(idx)
    return sorted(mine)


def timed_steps(torch, solver, steps: int, dist, world, sampler=None):
    """Device time of `steps` loop bodies on the solver's stream, max over ranks."""
    stream = torch.cuda.ExternalStream(solver.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = solver.launches
    t0 = time.time()
    ev0.record(stream)
    solver.step(steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    if sampler is not None:
        sampler.mark(t0, time.time())
    ms = ev0.elapsed_time(ev1)
    launches = solver.launches - l0
    if world > 1:
        ms = max_over_ranks(torch, dist, [ms], "cuda")[0]
        dist.barrier()
    return ms, launches


def profile_traffic(name: str):
    """dram__bytes_read.sum + dram__bytes_write.sum per launch, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            m = re.search(r"traffic_per_launch_bytes\s*=\s*([0-9]+)", f.read())
        return int(m.group(1)) if m else None
    except OSError:
        return None


def pass_roofline(torch, smadft, peak):
    """Average launch time of the plain axis passes of a 256^3 FP32 field, forward (DCT-II)
    and inverse (DCT-III) kinds along each axis.

    The passes run through a ring of 6 fields (384 MiB, well above the 126 MB L2): launch r
    reads field r mod 6 and writes field r+1 mod 6, so every launch reads a field that was
    last written five launches earlier.  Algorithmic bytes per launch = one field read + one
    field written = 2 x 4 B x 256^3.  Times are CUDA events on the context's stream.
    """
    ring = 6
    p = smadft.params(smadft.ADV, (N, N, N), precision=smadft.FP32, **CFG)
    with smadft.Solver(p) as s:
        bufs = [torch.randn((N, N, N), device="cuda", dtype=torch.float32) for _ in range(ring)]
        torch.cuda.synchronize()
        stream = torch.cuda.ExternalStream(s.stream)
        out = {}
        for axis, name in ((2, "z"), (1, "y"), (0, "x")):
            for kind, kname in ((0, "dct2"), (1, "dct3")):
                for r in range(ring):
                    s.r2r_pass_device(bufs[r].data_ptr(), bufs[(r + 1) % ring].data_ptr(), axis, kind)
                reps = 10 * ring
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                ev0.record(stream)
                for r in range(reps):
                    s.r2r_pass_device(bufs[r % ring].data_ptr(), bufs[(r + 1) % ring].data_ptr(), axis, kind)
                ev1.record(stream)
                torch.cuda.synchronize()
                us = 1000.0 * ev0.elapsed_time(ev1) / reps
                gbs = 2.0 * 4 * N ** 3 / (us * 1e-6) / 1e9
                out[f"{name}_{kname}"] = {"us": round(us, 2), "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
                # refill: repeated unnormalised passes grow the values by about 2N each
                for bft in bufs:
                    bft.normal_()
                torch.cuda.synchronize()
        return out


def sweep_params(smadft):
    """Config 4: 48 runs, 12 each of 64^3 / 96^3 / 128^3 / 160^3, noadv and adv alternating,
    eps ~ U[-0.85, -0.65], gamma in {0.8, 1.0, 1.2}, FP32 fields (FP64 state and reductions),
    seeded per run (seed 20240601 + run)."""
    rng = np.random.default_rng(20240601)
    runs = []
    for r in range(48):
        n = (64, 96, 128, 160)[r % 4]
        model = smadft.NOADV if (r // 4) % 2 == 0 else smadft.ADV
        kw = dict(eps=float(rng.uniform(-0.85, -0.65)), gamma=(0.8, 1.0, 1.2)[r % 3],
                  dt=0.05 if model == smadft.NOADV else 0.01)
        runs.append((model, n, kw, 20240601 + r))
    return runs


def run_batch_sweep(torch, smadft, steps, rank, world, dist):
    """Config 4 through smadft_batch: this rank's share of the 48 runs (greedy by cost
    N^3 F, F = 6 noadv / 32 adv), each autotuned, then `steps` batch steps timed with CUDA
    events on the batch stream (members of one model and grid are stepped as groups with
    pooled fields).  Beside it: the same runs as an FP64 batch (each run's relative L2 error of
    psi against its FP64 twin after `steps` steps), and 200 steps of the same FP32 runs stepped
    one context after another and as an ungrouped batch, for comparison."""
    runs = sweep_params(smadft)
    mine = partition_by_cost([n ** 3 * (6 if model == smadft.NOADV else 32) for model, n, _, _ in runs], world, rank)

    def plist_for(prec):
        out = []
        for i in sorted(mine):
            model, n, kw, _ = runs[i]
            out.append(smadft.params(model, (n, n, n), precision=prec, **kw))
        return out

    ics = []
    for i, p in zip(sorted(mine), plist_for(smadft.FP32)):
        seed = runs[i][3]
        if p.model == smadft.NOADV:
            ics.append(smadft.ic_interface(p, A=1.328, bump=0.0, noise=1e-3, seed=seed))
        else:
            ics.append(smadft.ic_conics(p, A=1.328, count=4, rmin=1.0, rmax=2.0, noise=1e-3, seed=seed))

    def timed(b, nsteps):
        stream = torch.cuda.ExternalStream(b.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b.sync()
        torch.cuda.synchronize()
        e0.record(stream)
        b.step(nsteps)
        e1.record(stream)
        b.sync()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    out = {}
    with smadft.Batch(plist_for(smadft.FP32)) as b:
        for m, psi in zip(b.members, ics):
            m.set_psi(psi)
        tuned = {}
        for m in b.members:
            rep = m.autotune(2)
            tuned[rep["chosen"]] = tuned.get(rep["chosen"], 0) + 1
        groups = b.groups
        b.step(3)
        ms_batch = timed(b, steps)
        psi32 = [m.get("psi") for m in b.members]
    with smadft.Batch(plist_for(smadft.FP64)) as b:
        for m, psi in zip(b.members, ics):
            m.set_psi(psi)
        b.step(3 + steps)
        b.sync()
        psi64 = [m.get("psi") for m in b.members]
    errs = [float(np.linalg.norm(a - c) / np.linalg.norm(c)) for a, c in zip(psi32, psi64)]
    finite = all(bool(np.all(np.isfinite(a))) for a in psi32)
    cmp_steps = min(steps, 200)
    # the same FP32 runs, one context after another (each on its own graph), and as an
    # ungrouped batch (each member's own kernels as graph branches)
    with smadft.Batch(plist_for(smadft.FP32)) as b:
        for m, psi in zip(b.members, ics):
            m.set_psi(psi)
            m.step(3)
        b.sync()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for m in b.members:
            m.step(cmp_steps)
        for m in b.members:
            m.sync()
        ms_solo = 1000.0 * (time.perf_counter() - t0)
    os.environ["SMADFT_BATCH_GROUP"] = "0"
    try:
        with smadft.Batch(plist_for(smadft.FP32)) as b:
            for m, psi in zip(b.members, ics):
                m.set_psi(psi)
            b.step(3)
            ms_ungrouped = timed(b, cmp_steps)
    finally:
        del os.environ["SMADFT_BATCH_GROUP"]
    bytes_per_step = sum(4.0 * n ** 3 * (6 if model == smadft.NOADV else 32)
                         for i, (model, n, _, _) in enumerate(runs) if i in set(mine))
    if world > 1:
        ms_batch, ms_solo, ms_ungrouped = max_over_ranks(torch, dist, [ms_batch, ms_solo, ms_ungrouped], "cuda")
        c = torch.tensor([float(finite)], device="cuda")
        dist.all_reduce(c, op=dist.ReduceOp.MIN)
        finite = bool(c.item())
    total = len(runs) * steps
    out = {"runs": len(runs), "runs_on_rank0": len(psi32), "steps": steps,
           "grids": "12 each of 64^3, 96^3, 128^3, 160^3; noadv/adv alternating; FP32",
           "groups_rank0": groups,
           "aggregate_steps_per_s": total / (ms_batch / 1000.0),
           "ms_per_batch_step": ms_batch / steps,
           "hbm_frac_rank0": bytes_per_step / (ms_batch / steps * 1e-3) / 1e9 / peaks()[0],
           "sequential_aggregate_steps_per_s": len(runs) * cmp_steps / (ms_solo / 1000.0),
           "ungrouped_batch_aggregate_steps_per_s": len(runs) * cmp_steps / (ms_ungrouped / 1000.0),
           "comparison_steps": cmp_steps,
           "rel_l2_err_vs_fp64": {"max": max(errs), "median": float(np.median(errs)),
                                  "per_run": [float(f"{e:.3e}") for e in errs]},
           "autotuned_paths_rank0": tuned, "finite": finite,
           "timing": "CUDA events on the batch stream (sequential: host wall clock), max over ranks"}
    return out


def run_adjoint_c5(torch, smadft, steps):
    """Config 5: the adjoint of the adv step at 128^3, dt = 0.02, checkpoints every 50 steps
    over `steps` steps, FP32 forward + adjoint, with the FP64 adjoint and a central
    difference of the FP64 forward (eps and nu) beside it.  The loss is the mean tracked
    interface position (bump tracker along x), so the initial condition is the x-normal
    interface with a bump (config 3's focal-conic field has no interface).  Times are host
    wall clock around one smadft_adjoint call (which synchronises), allocations included."""
    n, K = 128, 50
    kw = dict(CFG)
    kw["dt"] = 0.02
    track = dict(axis=0, mode=smadft.TRACK_BUMP, hi=0.6, lo=0.1)
    psi0 = smadft.ic_interface(smadft.params(smadft.ADV, (n, n, n), **kw), A=1.328, bump=0.5 * 2 * np.pi,
                               noise=1e-3, seed=20240601)
    out = {"config": f"adv {n}^3, dt=0.02, {steps} steps, checkpoints every {K}; interface IC (x-normal, bump); "
                     "loss = mean bump-tracked interface position (lambda0)"}
    grads = {}
    for prec, name in ((smadft.FP32, "fp32"), (smadft.FP64, "fp64")):
        p = smadft.params(smadft.ADV, (n, n, n), precision=prec, **kw)
        with smadft.Solver(p) as s:
            s.set_psi(psi0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g = s.adjoint(steps, checkpoint_every=K, **track)
            out[f"adjoint_{name}_ms"] = 1000.0 * (time.perf_counter() - t0)
        with smadft.Solver(p) as s:
            s.set_psi(psi0)
            s.step(3)
            s.sync()
            t0 = time.perf_counter()
            s.step(steps)
            s.sync()
            out[f"forward_{name}_ms"] = 1000.0 * (time.perf_counter() - t0)
        grads[name] = g
    names = ("eps", "alpha", "beta", "gamma", "nu")
    out["grad_fp32"] = {k: grads["fp32"][k] for k in names}
    out["grad_fp64"] = {k: grads["fp64"][k] for k in names}
    out["found_columns"] = grads["fp64"]["found"]
    out["max_rel_err_fp32_vs_fp64"] = max(abs(grads["fp32"][k] - grads["fp64"][k]) / abs(grads["fp64"][k])
                                          for k in names)
    d32, d64 = grads["fp32"]["psi0"], grads["fp64"]["psi0"]
    out["psi0_rel_l2_fp32_vs_fp64"] = float(np.linalg.norm(d32 - d64) / np.linalg.norm(d64))

    def loss(**over):
        kk = dict(kw)
        kk.update(over)
        with smadft.Solver(smadft.params(smadft.ADV, (n, n, n), **kk)) as s:
            s.set_psi(psi0)
            s.step(steps)
            idx, pos = s.track(**track)
        m = (idx >= 0) & np.isfinite(pos)
        return pos[m].mean() / kk["nw"], int(m.sum())
    h = 1e-7
    fd = {}
    for k in ("eps", "nu"):
        jp, fp = loss(**{k: kw[k] + h})
        jm, fm = loss(**{k: kw[k] - h})
        fd[k] = {"fd": (jp - jm) / (2 * h), "same_found_set": fp == fm == grads["fp64"]["found"],
                 "rel_err_fp64_adjoint": abs(grads["fp64"][k] - (jp - jm) / (2 * h)) / abs((jp - jm) / (2 * h))}
    out["central_difference_h1e-7"] = fd
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import smadft
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    if not os.path.exists(smadft.LIB_PATH):
        smadft.build()
    psi0 = make_ic()
    peak, peak_kind = peaks()
    res = {}
    launches_fp32 = 0
    clocks = {}
    solvers = {}
    tuned = {}
    for prec, name in ((smadft.FP32, "fp32"), (smadft.FP64, "fp64")):
        p = smadft.params(smadft.ADV, (N, N, N), precision=prec, device=local_rank, **CFG)
        s = solvers[name] = smadft.Solver(p)
        s.set_psi(psi0)
        tuned[name] = s.autotune(3)["chosen"]      # kernel path per grid and precision
        s.step(args.warmup)
        s.sync()
        if name == "fp32":
            with ClockSampler(local_rank) as cs:
                ms, launches = timed_steps(torch, s, args.steps, dist, world, cs)
            clocks = cs.summary()
            launches_fp32 = launches
        else:
            ms, _ = timed_steps(torch, s, args.steps, dist, world)
        res[name] = {"ms": ms, "psi": s.get("psi")}

    def rel_err(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    err_timed = rel_err(res["fp32"]["psi"], res["fp64"]["psi"])
    # both runs continue (untimed) to ERR_STEPS steps for the error the target is stated at
    done = args.warmup + args.steps
    err, err_steps = err_timed, done
    if args.err_steps > done:
        for s in solvers.values():
            s.step(args.err_steps - done)
        err = rel_err(solvers["fp32"].get("psi"), solvers["fp64"].get("psi"))
        err_steps = args.err_steps
    for s in solvers.values():
        s.close()
    ms_step = res["fp32"]["ms"] / args.steps
    ms_step64 = res["fp64"]["ms"] / args.steps
    value = world * args.steps / (res["fp32"]["ms"] / 1000.0)

    # end to end through the public API with host buffers: per step, psi (FP64, pinned host)
    # goes up, one loop body runs, psi comes back (smadft_step_host)
    p = smadft.params(smadft.ADV, (N, N, N), precision=smadft.FP32, device=local_rank, **CFG)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        host = torch.from_numpy(psi0.copy()).pin_memory()
        hn = host.numpy()
        for _ in range(2):
            s.step_host(hn, 1)
        e2e_steps = max(3, min(args.steps, 10))
        stream = torch.cuda.ExternalStream(s.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(e2e_steps):
            s.step_host(hn, 1)
        ev1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = ev0.elapsed_time(ev1)
        if world > 1:
            e2e_ms = max_over_ranks(torch, dist, [e2e_ms], "cuda")[0]
    e2e_value = world * e2e_steps / (e2e_ms / 1000.0)

    sweep = run_batch_sweep(torch, smadft, args.sweep_steps, rank, world, dist) if args.sweep_steps > 0 else None
    passes = pass_roofline(torch, smadft, peak) if rank == 0 else {}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    adjoint = run_adjoint_c5(torch, smadft, args.adjoint_steps) if args.adjoint_steps > 0 else None

    algo_bytes = 4.0 * N ** 3 * F_ADV
    achieved_step = algo_bytes / (ms_step * 1e-3) / 1e9
    cpu = {}
    try:
        threads = os.cpu_count() or 1
        sps, secs, kind, sample = cpu_reference_run(4, psi0, threads)
        cpu = {"value": sps, "unit": "steps/s", "cores": threads, "kind": kind, "sample": sample}
    except Exception as e:  # reported, not fatal
        cpu = {"value": None, "unit": "steps/s", "cores": 0, "kind": "port", "sample": f"failed: {e}"}
    # the dominant kernel of the step (largest share of its device time in the committed
    # launch list): the plain inverse (DCT-III) pass along z
    dom = passes.get(DOMINANT_PASS, {})
    config = bench_config(world)
    config.update({
        "fp32_ms_per_step": round(ms_step, 4), "fp64_ms_per_step": round(ms_step64, 4),
        "speedup_vs_fp64": round(ms_step64 / ms_step, 3), "rel_l2_err_vs_fp64": err, "err_after_steps": err_steps,
        "precision": "FP32 fields and transforms; FP64 spectral state, time update and reductions",
        "kernel_path": tuned.get("fp32")})
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config,
        "roofline": {"bound": "hbm", "achieved": dom.get("gbs"), "peak": peak, "unit": "GB/s",
                     "frac": dom.get("frac"), "traffic": profile_traffic(DOMINANT_PROFILE),
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "kernel": DOMINANT_KERNEL,
                     "step_frac": round(achieved_step / peak, 4)},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 8 * N ** 3,
                "d2h_bytes_per_step": 8 * N ** 3},
        "gpu_launches": launches_fp32,
        "clocks": clocks,
        "fp64_steps_per_s": world * args.steps / (res["fp64"]["ms"] / 1000.0),
        "rel_l2_err_after_timed_steps": err_timed,
        "step_roofline": {"achieved": achieved_step, "peak": peak, "unit": "GB/s", "frac": achieved_step / peak,
                          "basis": "4 B x 256^3 x 32 compulsory field transfers per adv step"},
        "pass_kernels": passes,
        "batch_sweep": sweep,
        "adjoint": adjoint,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_kernel_only(args):
    """A few launches of one kernel family for profiling (ncu): no timing, no JSON.

    pass-z | pass-y | pass-x: one plain axis pass (kind --kind) on a 256^3 field (2 fields held).
    r2r3d: one plain 3-D DCT-III (the plane kernel for z and y where it applies, then x).
    step: loop bodies of the adv model (all its kernels).
    comp-step: loop bodies of the compressible model past its relaxation switch.
    batch-step: config 4's 48-run FP32 batch, one eager body and `reps` graph-replayed bodies.
    """
    import torch
    import smadft
    prec = smadft.FP64 if args.precision == "fp64" else smadft.FP32
    n = args.shape
    p = smadft.params(smadft.ADV, (n, n, n), precision=prec, **CFG)
    with smadft.Solver(p) as s:
        if args.kernel_only.startswith("pass"):
            dt = torch.float32 if prec == smadft.FP32 else torch.float64
            x = torch.randn((n, n, n), device="cuda", dtype=dt)
            y = torch.empty_like(x)
            torch.cuda.synchronize()
            axis = {"pass-z": 2, "pass-y": 1, "pass-x": 0}[args.kernel_only]
            for _ in range(args.reps):
                s.r2r_pass_device(x.data_ptr(), y.data_ptr(), axis, args.kind)
        elif args.kernel_only == "r2r3d":
            dt = torch.float32 if prec == smadft.FP32 else torch.float64
            x = torch.randn((n, n, n), device="cuda", dtype=dt)
            y = torch.empty_like(x)
            torch.cuda.synchronize()
            for _ in range(args.reps):
                s.r2r3d_device(x.data_ptr(), y.data_ptr(), (1, 1, 1))
        elif args.kernel_only == "step":
            p2 = smadft.params(smadft.ADV, (n, n, n), **CFG)
            s.set_psi(smadft.ic_conics(p2, A=1.328, count=4, rmin=3.0, rmax=6.0, seed=1))
            s.step(args.reps)
        s.sync()
    if args.kernel_only == "batch-step":
        # config 4's 48 FP32 runs (grouped batch): set-up, one eager body, then `reps` graph bodies
        plist = [smadft.params(model, (nn, nn, nn), precision=smadft.FP32, **kw)
                 for model, nn, kw, _ in sweep_params(smadft)]
        with smadft.Batch(plist) as b:
            for m, p2 in zip(b.members, plist):
                m.set_psi(smadft.ic_interface(p2, A=1.328, bump=0.0, noise=1e-3, seed=1))
            b.step(1)
            b.step(args.reps)
            b.sync()
    if args.kernel_only == "comp-step":
        pc = smadft.params(smadft.COMP, (n, n, n), precision=prec, divv_switch=1)
        x = np.arange(n)[:, None, None]
        z = np.arange(n)[None, None, :] * 2 * np.pi / 8
        with smadft.Solver(pc) as s:
            s.set_psi(1.3 * np.cos(z) * 0.5 * (1 - np.tanh((x - n / 2) / 4.0)) * np.ones((1, n, 1)))
            s.step(1)
            s.step(args.reps)
            s.sync()
    print(f"kernel-only {args.kernel_only} {n}^3 {args.precision} x{args.reps}: done")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sweep-steps", type=int, default=2000,
                    help="steps of the 48-run batched sweep (config 4: 2000; 0: skip)")
    ap.add_argument("--err-steps", type=int, default=ERR_STEPS,
                    help="steps after which the FP32 error against FP64 is reported (0: after the timed steps)")
    ap.add_argument("--kernel-only", choices=["pass-z", "pass-y", "pass-x", "r2r3d", "step", "comp-step", "batch-step"],
                    default=None,
                    help="launch one kernel family a few times (for profilers) and exit")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--adjoint-steps", type=int, default=500,
                    help="steps of the 128^3 adv adjoint measurement (0: skip)")
    ap.add_argument("--shape", type=int, default=N)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--kind", type=int, default=0, choices=[0, 1, 2, 3],
                    help="kernel-only passes: 0 DCT-II, 1 DCT-III, 2 DST-II, 3 DST-III")
    args = ap.parse_args()
    if args.kernel_only:
        return run_kernel_only(args)
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
