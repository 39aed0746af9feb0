"""Throughput benchmark of the B200 force evaluation + leapfrog step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Default workload (``bh_collision_1m``): plain Barnes-Hut on two Plummer
spheres of 500k particles (a = 1, M = 1/2 each, centres 10 apart on x,
relative velocity 0.3 on y), eps = 0.01, theta = 0.7, leapfrog KDK at
dt = 1e-3 — one step = one kick-drift-force-kick of all N particles.
Metric: particle-steps/s (N x steps / device time).

Other workloads (parity configs, selectable): ``allpairs_plummer_16k``,
``allpairs_precision_262k``, ``ensemble_4096`` and ``bh_matched_10m`` (the
same collision at N = 10M).  Multi-GPU sharding (strong scaling, `scaling`
"strong"): ``allpairs_sharded_262k`` splits one all-pairs system by targets
over the ranks with an NCCL all-gather of the packed sources every step;
``ensemble_4096_sharded`` splits the 4096 systems over the ranks by cost.

`matched_accuracy` (Barnes-Hut workloads, skipped with --no-matched): on the
initial state, the rms relative force error against the FP64 direct sum on
4096 seeded targets is measured over a theta grid for the monopole and the
quadrupole walk under the reference's opening test and under the offset test;
each method is then timed at the largest theta whose error is at most 1e-3;
the relative opening test (G M (2h)^2 / d^4 <= alpha max(|a_old|, rms |a_old|)
with the reference's test at theta 1.0 as the safety bound) is swept over
alpha the same way.  "plain" is the monopole walk with the reference's test,
"chosen" the fastest method.  ``bh_matched_10m`` adds the plain walk at theta 0.5 and the learned
correction at theta 1.0 under both opening tests (network trained on 2^22
cell-target pairs of the 1M collision).

Timing: W untimed warm-up steps; then K steps, each a 1-step device-resident
advance bracketed by CUDA events recorded by the library on its own stream;
a 256 MiB buffer is written between timed steps to flush the 126 MB L2.
Under torchrun (N > 1) every rank of the Barnes-Hut and all-pairs workloads
advances its own replica (no data-path collective: "replicas only"), the step
time is the max over ranks and `value` sums the ranks' particle-steps; the
sharded workloads divide one job instead.

`e2e`: the same metric through the reference-facing plugin call
n_body_sim_pro_barnes_hut_compute_acceleration_cuda(view, ...) on pinned host
arrays inside a host leapfrog loop: every step copies positions + masses to
the device and accelerations back.

`cpu_baseline` / `--impl reference`: the reference engine compiled from its
own sources (oracle/_ref) timed on this host's cores on the same initial
conditions (a bounded sample of steps).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "bh_collision_1m": dict(n=1_000_000, algorithm="barnes_hut", theta=0.7, eps=0.01, dt=1e-3,
                            ic="collision", steps=10, order=1),
    "allpairs_plummer_16k": dict(n=16384, algorithm="all_pairs", eps=0.01, dt=1e-3,
                                 ic="plummer", steps=3),
    "allpairs_precision_262k": dict(n=262144, algorithm="all_pairs", eps=1e-3, dt=1e-4,
                                    ic="uniform_log_mass", steps=3),
    "ensemble_4096": dict(n=None, algorithm="ensemble", systems=4096, lo=32, hi=4096, eps=0.01,
                          dt=1e-3, ic="ensemble", steps=1000),
    "bh_matched_10m": dict(n=10_000_000, algorithm="barnes_hut", theta=0.5, eps=0.01, dt=1e-3,
                           ic="collision", steps=3, order=1, matched=True, correction=True),
    # one system split by targets over the ranks (strong scaling; NCCL all-gather per step)
    "allpairs_sharded_262k": dict(n=262144, algorithm="all_pairs_sharded", eps=1e-3, dt=1e-4,
                                  ic="uniform_log_mass", steps=3),
    # the 4096 systems split over the ranks by cost (strong scaling; no collective)
    "ensemble_4096_sharded": dict(n=None, algorithm="ensemble", systems=4096, lo=32, hi=4096,
                                  eps=0.01, dt=1e-3, ic="ensemble", steps=1000, sharded=True),
}

# Matched-accuracy study: the largest opening angle of this grid whose rms
# relative force error (FP64 direct sum on 4096 seeded targets, initial state)
# stays at or below RMS_TARGET, per method.
RMS_TARGET = 1e-3
THETA_GRID = (0.4, 0.45, 0.5, 0.525, 0.55, 0.575, 0.6, 0.625, 0.65, 0.675, 0.7, 0.725, 0.75, 0.8,
              0.9, 1.0)

# DRAM bytes (read + write) per launch of the dominant kernel from one ncu
# capture of exactly this configuration (the file under profiles/ gives the command).
PROFILED_TRAFFIC = {
    ("bh_collision_1m", 0.7, 1, "lists", 16): (
        30_559_232, "profiles/walk_lists_kernel_bh_collision_1m.md"),
    ("allpairs_plummer_16k", None, 1, "lists", 16): (
        296_960, "profiles/allpairs_force_paired_kernel_plummer_16k.md"),
}

FP32_LANES_PER_SM = 128  # FFMA lanes per Blackwell SM
FLOPS_PAIR = 20          # standard convention per softened pair interaction
FLOPS_QUAD = 58          # monopole + trace-free quadrupole per accepted cell
MLP_FLOPS = 2 * (10 * 64 + 64 * 64 + 64 * 3)  # 9,856: one forward pass of the 10-64-64-3 network


# ---------------------------------------------------------------------------
# initial conditions (numpy; statistically the reference's Plummer preset,
# src/c/generation/presets.c:144-202, not its RNG stream)
# ---------------------------------------------------------------------------

def plummer_block(rng, n, a, mass, centre):
    u = 1.0 - rng.random(n)
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pos = r[:, None] * d + np.asarray(centre)
    sigma = np.sqrt(mass / (6.0 * np.sqrt(a * a + r * r)))
    vel = rng.standard_normal((n, 3)) * sigma[:, None]
    vel -= vel.mean(axis=0)
    return pos, vel, np.full(n, mass / n)


def initial_conditions(kind, n, seed=42):
    rng = np.random.default_rng(seed)
    if kind == "plummer":
        return plummer_block(rng, n, 1.0, 1.0, (0.0, 0.0, 0.0))
    if kind == "collision":
        h = n // 2
        p1, v1, m1 = plummer_block(rng, h, 1.0, 0.5, (-5.0, 0.0, 0.0))
        p2, v2, m2 = plummer_block(rng, n - h, 1.0, 0.5, (5.0, 0.0, 0.0))
        v1[:, 1] -= 0.15
        v2[:, 1] += 0.15
        return np.vstack([p1, p2]), np.vstack([v1, v2]), np.concatenate([m1, m2])
    if kind == "uniform_log_mass":
        pos = rng.random((n, 3))
        m = 10.0 ** rng.uniform(-3.0, 0.0, n)
        return pos, np.zeros((n, 3)), m / m.sum()
    raise ValueError(kind)


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def _one_shot(self):
        """A single query, for timed regions shorter than the sampling period."""
        try:
            out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                  "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                 timeout=10)
            self.out.extend(line.strip() for line in out.stdout.splitlines() if line.strip())
        except (OSError, subprocess.TimeoutExpired):
            pass

    def summary(self):
        if not self.out:
            self._one_shot()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for name, flag in zip(names, f[4:8]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def fp32_peak_tflops(sm_count, mhz):
    return sm_count * FP32_LANES_PER_SM * 2 * mhz * 1e6 / 1e12


def dist_setup(gpus, backend="nccl"):
    """One process per GPU under torchrun (RANK / WORLD_SIZE / LOCAL_RANK from the
    environment); `backend` "gloo" runs the same host logic on CPU processes."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _device_sync():
    import torch

    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()


def barrier_sync(world):
    _device_sync()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        _device_sync()


def max_over_ranks(value, world):
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# reference arm / CPU baseline (the reference engine compiled from its sources)
# ---------------------------------------------------------------------------

def reference_steps(wl, pos, vel, mass, steps, threads):
    """Time `steps` leapfrog steps of the reference engine on this host:
    n_body_sim_pro_integrator_advance with its Barnes-Hut (or OpenMP AVX all-pairs)
    force function.  Returns seconds per step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if not O.ref_available():
        raise RuntimeError("oracle/_ref not built")
    os.environ["OMP_NUM_THREADS"] = str(threads)
    R = O.ref()
    p = O.Particles.zeros(mass.shape[0])
    p.x[:], p.y[:], p.z[:] = pos.T
    p.vx[:], p.vy[:], p.vz[:] = vel.T
    p.m[:] = mass
    g = O.Gravity()
    R.n_body_sim_pro_gravity_init(C.byref(g), 1.0, wl["eps"])
    err = O.Error()
    v = p.view()
    ctx = None
    if wl["algorithm"] == "barnes_hut":
        ctx = R.n_body_sim_pro_barnes_hut_tree_create(C.byref(err))
        R.n_body_sim_pro_barnes_hut_tree_set_theta(ctx, wl["theta"])
        fn = R.n_body_sim_pro_barnes_hut_compute_acceleration
    else:
        fn = R.n_body_sim_pro_gravity_compute_acceleration_openmp_avx512
    force = C.cast(fn, C.c_void_p)
    if fn(C.byref(v), C.byref(g), ctx, C.byref(err)) != 0:  # initial forces
        raise RuntimeError(err.message)
    t0 = time.perf_counter()
    for _ in range(steps):
        rc = R.n_body_sim_pro_integrator_advance(C.byref(v), C.byref(g), 1, wl["dt"], force, ctx,
                                                 C.byref(err))
        if rc != 0:
            raise RuntimeError(err.message)
    dt = (time.perf_counter() - t0) / steps
    if ctx is not None:
        R.n_body_sim_pro_barnes_hut_tree_destroy(ctx)
    return dt


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, wl, world, rank, local):
    import torch

    import n_body_sim_pro_b200 as nb

    n = wl["n"]
    pos, vel, mass = initial_conditions(wl["ic"], n, seed=42 + rank)
    g = nb.gravity_init(1.0, wl["eps"])
    algo = nb.Algorithm.BARNES_HUT if wl["algorithm"] == "barnes_hut" else nb.Algorithm.ALL_PAIRS
    ctx = nb.CudaContext(theta=wl.get("theta", 0.7), multipole_order=wl.get("order", 1),
                         leaf_capacity=wl.get("leaf"))
    ctx.set_walk(0 if wl.get("walk") == "stackless" else 1)
    system = nb.ParticleSystem.from_arrays(pos, vel, mass)
    ctx.upload(system)
    ctx.compute_acceleration(g, algo)
    q0, pe0 = ctx.diagnostics(g, potential=True) if n <= 2_000_000 else (ctx.diagnostics(g), None)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")

    for _ in range(args.warmup):
        ctx.advance(g, wl["dt"], 1, algo)
    barrier_sync(world)
    launches0 = nb.kernel_launches()
    step_ms, walk_ms, stats_acc, phases = [], [], [], []
    torch.cuda.nvtx.range_push("timed_steps")  # profilers can select the timed launches
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            ctx.advance(g, wl["dt"], 1, algo)
            t = ctx.timings()
            step_ms.append(t["total_ms"])
            walk_ms.append(t["walk_ms"])
            phases.append(t)
            st = ctx.stats()
            st["walk_restarts"] = ctx.walk_restarts()
            stats_acc.append(st)
    torch.cuda.nvtx.range_pop()
    launches = nb.kernel_launches() - launches0
    barrier_sync(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)

    # accuracy of the final state: forces vs the FP64 device oracle on 4096 targets
    ctx.compute_acceleration(g, algo)
    final = nb.ParticleSystem.zeros(n)
    ctx.download(final)
    targets = np.random.default_rng(7).choice(n, min(4096, n), replace=False)
    ref = ctx.reference_acceleration(g, targets)
    acc = final.acc()[targets]
    rms = float(np.sqrt(np.sum((acc - ref) ** 2) / np.sum(ref ** 2)))
    max_rel = float(np.max(np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)))
    drift = None
    if pe0 is not None:
        q1, pe1 = ctx.diagnostics(g, potential=True)
        drift = float(abs((q1[0] + pe1) - (q0[0] + pe0)) / abs(q0[0] + pe0))

    # dominant kernel roofline
    peaks, peak_kind = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    clk = clocks.summary()
    mhz_load = clk["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    peak_max = fp32_peak_tflops(sm_count, peaks.get("sm_max_mhz", 1965.0))
    if wl["algorithm"] == "barnes_hut":
        approx = np.mean([s["accepted_approximations"] for s in stats_acc])
        exact = np.mean([s["exact_interactions"] for s in stats_acc])
        flops = FLOPS_PAIR * exact + (FLOPS_PAIR if wl.get("order", 1) == 1 else FLOPS_QUAD) * approx
        kernel_ms = float(np.mean(walk_ms))
        kernel = "walk_kernel"
        interactions = approx + exact
    else:
        flops = FLOPS_PAIR * float(n) * float(n)
        kernel_ms = float(np.mean(walk_ms)) if np.mean(walk_ms) > 0 else total_ms / args.steps
        kernel = "allpairs_force_kernel"
        interactions = float(n) * n
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    try:
        probe = nb.measure_fp32_peak()
    except nb.CudaError:
        probe = None
    roofline = {"bound": "fp32", "kernel": kernel, "achieved": round(achieved, 3),
                "probe": probe,
                "peak": round(peak_max, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak_max, 4),
                "frac_at_load_clock": round(achieved / fp32_peak_tflops(sm_count, mhz_load), 4),
                "peak_kind": f"FP32 = {sm_count} SMs x 128 lanes x 2 x {peaks.get('sm_max_mhz', 1965.0)} MHz "
                             f"(sm_max_mhz of {peak_kind} MEASURED_PEAKS.json)",
                "flops_per_launch": flops, "launch_ms": round(kernel_ms, 4),
                "traffic": None}
    measured = PROFILED_TRAFFIC.get((args.workload, wl.get("theta"), wl.get("order", 1),
                                     wl.get("walk", "lists"), wl.get("leaf", 16)))
    if measured is not None:
        roofline["traffic"] = measured[0]
        roofline["traffic_source"] = measured[1]
    stages = None
    if wl["algorithm"] == "barnes_hut" and phases:
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        nodes = float(stats_acc[-1]["node_count"])
        # the moments pass: the monopole walk's reads each particle once and
        # writes 64 B per node (FP64 moments, the walk's float4, opening
        # terms), reading 52 (record, level, children's moments); the
        # quadrupole pass reads the particles twice, writes 156 and reads 108
        quad = wl.get("order", 1) == 2
        mom_bytes = (32.0 * n + 264.0 * nodes) if quad else (16.0 * n + 116.0 * nodes)
        stages = {}
        for name, key, nbytes in (
                ("bounds", "bounds_ms", 32.0 * n),
                ("keys", "keys_ms", 36.0 * n),
                ("sort", "sort_ms", 8 * 24.0 * n),
                ("moments", "moments_ms", mom_bytes),
                ("integrate", "integrate_ms", 36.0 * n + 24.0 * n + 120.0 * n)):
            ms = float(np.mean([ph[key] for ph in phases]))
            gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else None
            stages[name] = {"ms": round(ms, 4), "algorithmic_bytes": nbytes,
                            "gbs": round(gbs, 1) if gbs else None,
                            "frac_of_hbm": round(gbs / hbm, 4) if gbs else None}
        stages["_note"] = (f"HBM peak {hbm} GB/s ({peak_kind} MEASURED_PEAKS.json); bytes: "
                           "bounds 32/particle, keys 24+12, sort 8 passes x (12+12), moments "
                           + ("2 x 16 per particle + 264 per node" if quad else
                              "16 per particle + 116 per node")
                           + ", integrate scatter 36 + kick-drift 24 + 120 per particle")

    # e2e through the plugin call on pinned host arrays
    e2e = None
    if rank == 0 or world > 1:
        e2e = run_e2e(nb, wl, pos, vel, mass, min(args.steps, 5), algo, ctx)

    ctx.close()
    matched = None
    if wl["algorithm"] == "barnes_hut" and not args.no_matched:
        matched = matched_study(nb, torch, wl, system, g, min(args.steps, 5), 3, flush,
                                with_correction=wl.get("correction", False))
    value = world * n * args.steps / (total_ms * 1e-3)
    split = None
    if wl["algorithm"] == "barnes_hut":  # particle-cell and particle-particle terms apart
        per_s = world * args.steps / (total_ms * 1e-3)
        split = {"particle_cell_per_s": approx * per_s, "particle_particle_per_s": exact * per_s}
    return dict(value=value, total_ms=total_ms, rms=rms, max_rel=max_rel, drift=drift,
                roofline=roofline, clocks=clk, launches=launches, e2e=e2e,
                interactions_per_s=world * interactions * args.steps / (total_ms * 1e-3),
                interactions_split=split,
                stats=stats_acc[-1], timings=ctx_timings_summary(step_ms, walk_ms, phases),
                matched=matched, stages=stages)


def rms_at_targets(nb, ctx, g, n, targets, ref):
    ctx.compute_acceleration(g, nb.Algorithm.BARNES_HUT)
    acc = ctx.download_accelerations()[targets]
    return float(np.sqrt(np.sum((acc - ref) ** 2) / np.sum(ref ** 2)))


def timed_steps(nb, torch, system, g, wl, theta, order, steps, warmup, flush, correction=None,
                opening=0, alpha=0.0, leaf=16):
    """Device-timed 1-step advances from `system` (re-uploaded) at (theta, order, opening,
    relative tolerance alpha, bucket capacity)."""
    ctx = nb.CudaContext(theta=theta, multipole_order=order, opening=opening,
                         leaf_capacity=leaf)
    ctx.set_correction(correction)
    ctx.set_relative_opening(alpha)
    ctx.upload(system)
    for _ in range(warmup):
        ctx.advance(g, wl["dt"], 1, nb.Algorithm.BARNES_HUT)
    ms = []
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        ctx.advance(g, wl["dt"], 1, nb.Algorithm.BARNES_HUT)
        ms.append(ctx.timings()["total_ms"])
    ctx.close()
    return wl["n"] * steps / (sum(ms) * 1e-3), float(np.mean(ms))


OPENINGS = {"reference": 0, "offset": 1}
# relative opening test (G M (2h)^2 / d^4 <= alpha max(|a_old|, rms |a_old|)) over the
# reference test at theta 1.0: the alphas of its sweep
ALPHA_GRID = (0.001, 0.0015, 0.002, 0.0025, 0.003, 0.0035, 0.004, 0.0045, 0.005, 0.0055, 0.006,
              0.007, 0.01)


def matched_study(nb, torch, wl, system, g, steps, warmup, flush, with_correction=False):
    """Plain Barnes-Hut (monopole, the reference's opening test, 16-particle
    buckets) vs the chosen method — the fastest of {monopole, quadrupole} x
    {reference, offset opening test}, the monopole walk with 32-particle buckets,
    and the relative test over the reference test at theta 1.0 with 16- and
    32-particle buckets — each at the largest theta (alpha) of its grid meeting
    RMS_TARGET, all timed; optionally the learned correction at theta 1.0
    (trained on 2^22 pairs of the 1M collision) under either opening test and
    the plain walk at theta 0.5."""
    n = wl["n"]
    targets = np.random.default_rng(11).choice(n, min(4096, n), replace=False)
    ctx = nb.CudaContext(theta=0.5)
    ctx.upload(system)
    ref = ctx.reference_acceleration(g, targets)
    table = {}
    for oname, opening in OPENINGS.items():
        ctx.set_opening(opening)
        for order in (1, 2):
            ctx.set_multipole_order(order)
            rows = []
            for th in THETA_GRID:
                ctx.theta = th
                rows.append((th, rms_at_targets(nb, ctx, g, n, targets, ref)))
            table[(order, oname)] = rows
    ctx.set_opening(0)
    ctx.set_multipole_order(1)
    ctx.set_leaf_capacity(32)
    table_leaf32 = []
    for th in THETA_GRID:
        ctx.theta = th
        table_leaf32.append((th, rms_at_targets(nb, ctx, g, n, targets, ref)))
    ctx.set_leaf_capacity(16)
    # relative test: each alpha evaluated twice, the second walk reading the
    # first one's accelerations as a_old (as in a run, where a_old is the
    # previous step's)
    ctx.set_opening(0)
    ctx.set_multipole_order(1)
    ctx.theta = 1.0
    rel_rows = {}
    for leaf in (16, 32):
        ctx.set_leaf_capacity(leaf)
        rows = []
        for alpha in ALPHA_GRID:
            ctx.set_relative_opening(alpha)
            ctx.compute_acceleration(g, nb.Algorithm.BARNES_HUT)
            rows.append((alpha, rms_at_targets(nb, ctx, g, n, targets, ref)))
        rel_rows[leaf] = rows
    ctx.set_relative_opening(0.0)
    ctx.close()
    out = {"rms_target": RMS_TARGET, "oracle": "FP64 device direct sum, 4096 seeded targets, "
           "initial state",
           "sweep": {f"order{o}_{on}": [[t, round(r, 6)] for t, r in rows]
                     for (o, on), rows in table.items()}}
    out["sweep"]["order1_reference_leaf32"] = [[t, round(r, 6)] for t, r in table_leaf32]
    for leaf, rows in rel_rows.items():
        out["sweep"][f"order1_relative_alpha_theta1.0_leaf{leaf}"] = [[a, round(r, 6)]
                                                                      for a, r in rows]
    methods = {}
    for (order, oname), rows in table.items():
        ok = [t for t, r in rows if r <= RMS_TARGET]
        if not ok:
            continue
        th = max(ok)
        v, ms = timed_steps(nb, torch, system, g, wl, th, order, steps, warmup, flush,
                            opening=OPENINGS[oname])
        methods[(order, oname)] = {"theta": th, "multipole_order": order, "opening": oname,
                                   "leaf_capacity": 16, "rms": dict(rows)[th], "value": v,
                                   "ms_per_step": round(ms, 4)}
    ok = [t for t, r in table_leaf32 if r <= RMS_TARGET]
    if ok:
        th = max(ok)
        v, ms = timed_steps(nb, torch, system, g, wl, th, 1, steps, warmup, flush, leaf=32)
        methods[(1, "reference", 32)] = {"theta": th, "multipole_order": 1,
                                         "opening": "reference", "leaf_capacity": 32,
                                         "rms": dict(table_leaf32)[th], "value": v,
                                         "ms_per_step": round(ms, 4)}
    for leaf, rows in rel_rows.items():
        ok = [a for a, r in rows if r <= RMS_TARGET]
        if not ok:
            continue
        alpha = max(ok)
        v, ms = timed_steps(nb, torch, system, g, wl, 1.0, 1, steps, warmup, flush, alpha=alpha,
                            leaf=leaf)
        methods[(1, "relative", leaf)] = {"theta": 1.0, "multipole_order": 1,
                                          "opening": "reference", "relative_alpha": alpha,
                                          "leaf_capacity": leaf, "rms": dict(rows)[alpha],
                                          "value": v, "ms_per_step": round(ms, 4)}
    out["methods"] = list(methods.values())
    out["plain"] = methods.get((1, "reference"))
    out["chosen"] = max(methods.values(), key=lambda m: m["value"]) if methods else None
    if out["plain"] and out["chosen"]:
        out["chosen_over_plain"] = round(out["chosen"]["value"] / out["plain"]["value"], 3)
    if with_correction:
        v, ms = timed_steps(nb, torch, system, g, wl, 0.5, 1, steps, warmup, flush)
        out["plain_theta_0.5"] = {"theta": 0.5, "rms": dict(table[(1, "reference")])[0.5],
                                  "value": v, "ms_per_step": round(ms, 4)}
        pos1, vel1, mass1 = initial_conditions("collision", 1_000_000, seed=42)
        system1 = nb.ParticleSystem.from_arrays(pos1, vel1, mass1)
        corrected = {}
        for oname, opening in OPENINGS.items():
            with nb.CudaContext(theta=1.0, opening=opening) as c1, \
                    nb.CudaCorrection(seed=11) as corr:
                c1.upload(system1)
                t0 = time.time()
                corr.generate(c1, g, theta=1.0, samples=1 << 22, seed=3)
                tl, vl = corr.train(epochs=8, batch=1024, learning_rate=1e-3)
                train_s = time.time() - t0
                cctx = nb.CudaContext(theta=1.0, opening=opening)
                cctx.set_correction(corr)
                cctx.upload(system)
                rms_c = rms_at_targets(nb, cctx, g, n, targets, ref)
                evals = cctx.corrected_cells()  # network evaluations of that walk
                walk_ms = cctx.timings()["walk_ms"]
                cctx.close()
                v, ms = timed_steps(nb, torch, system, g, wl, 1.0, 1, steps, warmup, flush,
                                    correction=corr, opening=opening)
            corrected[oname] = {
                "theta": 1.0, "opening": oname, "rms": rms_c, "value": v,
                "ms_per_step": round(ms, 4),
                "uncorrected_rms_at_theta_1.0": dict(table[(1, oname)])[1.0],
                "network": {"evaluations_per_walk": evals, "flop_per_evaluation": MLP_FLOPS,
                            "walk_ms": round(walk_ms, 4),
                            "tensor_tflops_in_walk": round(evals * MLP_FLOPS / (walk_ms * 1e-3)
                                                           / 1e12, 3) if walk_ms > 0 else None},
                "training": {"pairs": 1 << 22, "from": "collision N=1M", "epochs": 8,
                             "final_validation_loss": float(vl[-1]),
                             "seconds": round(train_s, 2)}}
        out["corrected_theta_1.0"] = corrected
    return out


def ensemble_ic(wl, seed=42, systems=None):
    """Systems of round(exp(U(ln lo, ln hi))) Plummer particles (a = 1, M = 1), each
    from its own seeded stream, concatenated (only `systems`, when given)."""
    sizes, blocks = [], []
    keep = set(range(wl["systems"])) if systems is None else set(systems)
    for k in range(wl["systems"]):
        rng = np.random.default_rng([seed, k])
        n = int(np.clip(np.rint(np.exp(rng.uniform(np.log(wl["lo"]), np.log(wl["hi"])))),
                        wl["lo"], wl["hi"]))
        if k not in keep:
            continue
        blocks.append(plummer_block(rng, n, 1.0, 1.0, (0.0, 0.0, 0.0)))
        sizes.append(n)
    pos = np.vstack([b[0] for b in blocks])
    vel = np.vstack([b[1] for b in blocks])
    mass = np.concatenate([b[2] for b in blocks])
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    return pos, vel, mass, offsets


def ensemble_sizes(wl, seed=42):
    """The system sizes ensemble_ic draws, without generating the particles."""
    out = []
    for k in range(wl["systems"]):
        rng = np.random.default_rng([seed, k])
        out.append(int(np.clip(np.rint(np.exp(rng.uniform(np.log(wl["lo"]),
                                                           np.log(wl["hi"])))),
                               wl["lo"], wl["hi"])))
    return out


def run_ensemble(args, wl, world, rank, local):
    import torch

    import n_body_sim_pro_b200 as nb

    if wl.get("sharded"):  # one ensemble, its systems split over the ranks by cost
        from n_body_sim_pro_b200 import shard

        mine = shard.assign_systems(ensemble_sizes(wl), world)[rank]
        pos, vel, mass, offsets = ensemble_ic(wl, seed=42, systems=mine)
    else:  # an independent replica per rank
        pos, vel, mass, offsets = ensemble_ic(wl, seed=42 + rank)
    n = mass.shape[0]
    sizes = np.diff(offsets.astype(np.int64))
    g = nb.gravity_init(1.0, wl["eps"])
    system = nb.ParticleSystem.from_arrays(pos, vel, mass)
    ens = nb.CudaEnsemble()
    ens.upload(system, offsets)
    ens.autotune(g, wl["dt"])
    launches0 = None
    for _ in range(args.warmup):
        ens.advance(g, wl["dt"], 1)
    barrier_sync(world)
    launches0 = nb.kernel_launches()
    torch.cuda.nvtx.range_push("timed_steps")
    with ClockSampler(local) as clocks:
        ms = ens.advance(g, wl["dt"], args.steps)
    torch.cuda.nvtx.range_pop()
    launches = nb.kernel_launches() - launches0
    barrier_sync(world)
    total_ms = max_over_ranks(ms, world)
    info = ens.info()
    # baseline: one launch sequence per system and step, on a 2-step sample
    base_steps = 2
    ens.upload(system, offsets)
    base_ms = ens.advance(g, wl["dt"], base_steps, one_launch_per_system=True)
    baseline = {"value": n * base_steps / (base_ms * 1e-3), "unit": "particle-steps/s",
                "sample": f"{base_steps} steps, per-system all-pairs launches "
                          f"({int(nb.kernel_launches())} launches so far)"}
    interactions = float(np.sum(sizes.astype(np.float64) ** 2))
    peaks, peak_kind = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    peak_max = fp32_peak_tflops(sm_count, peaks.get("sm_max_mhz", 1965.0))
    flops = FLOPS_PAIR * interactions * (args.steps + 1)  # + the initial force pass
    achieved = flops / (total_ms * 1e-3) / 1e12
    clk = clocks.summary()
    roofline = {"bound": "fp32", "kernel": "ensemble_kernel", "achieved": round(achieved, 3),
                "peak": round(peak_max, 2), "unit": "TFLOP/s", "frac": round(achieved / peak_max, 4),
                "peak_kind": f"FP32 = {sm_count} SMs x 128 lanes x 2 x {peaks.get('sm_max_mhz')} MHz "
                             f"({peak_kind})", "flops_per_launch": flops,
                "launch_ms": round(total_ms, 3), "traffic": None}
    ens.close()
    if wl.get("sharded"):
        n_all = max_over_ranks(float(sum(ensemble_sizes(wl))), world)
        value = n_all * args.steps / (total_ms * 1e-3)
        interactions = float(sum(float(v) ** 2 for v in ensemble_sizes(wl))) / world
    else:
        value = world * n * args.steps / (total_ms * 1e-3)
    return dict(value=value, total_ms=total_ms, rms=None, max_rel=None, drift=None,
                roofline=roofline, clocks=clk, launches=launches, e2e=None,
                interactions_per_s=world * interactions * args.steps / (total_ms * 1e-3),
                stats={"systems": int(len(sizes)), "particles": int(n),
                       "ensemble": info, "one_launch_per_system": baseline},
                timings={"advance_ms": round(ms, 3)})


def run_sharded_allpairs(args, wl, world, rank, local):
    """One all-pairs system split by targets over the ranks (strong scaling):
    each step is shard_begin (kick-drift-pack), an NCCL all-gather of the
    packed sources (16 bytes per particle) and shard_end (forces + kick)."""
    import torch

    import n_body_sim_pro_b200 as nb
    from n_body_sim_pro_b200 import shard

    n = wl["n"]
    pos, vel, mass = initial_conditions(wl["ic"], n, seed=42)  # the same system on every rank
    first, count = shard.split(n, world)[rank]
    g = nb.gravity_init(1.0, wl["eps"])
    ctx = nb.CudaContext()
    part = nb.ParticleSystem.from_arrays(pos[first:first + count], vel[first:first + count],
                                         mass[first:first + count])
    device = torch.device("cuda", local)
    sim = shard.ShardedAllPairs(part, g, shard.CudaShardBackend(ctx), device)
    sim.compute_forces()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
    for _ in range(args.warmup):
        sim.step(wl["dt"], 1)
    barrier_sync(world)
    launches0 = nb.kernel_launches()
    step_ms, force_ms = [], []
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed_steps")
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            ev0.record()
            sim.step(wl["dt"], 1)
            ev1.record()
            ev1.synchronize()
            step_ms.append(ev0.elapsed_time(ev1))
            force_ms.append(ctx.timings()["walk_ms"])
    torch.cuda.nvtx.range_pop()
    launches = nb.kernel_launches() - launches0
    barrier_sync(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)

    # accuracy of the final state on rank 0: the full system gathered, FP64 oracle
    sim.compute_forces()
    mine = nb.ParticleSystem.zeros(count)
    sim.download(mine)
    rows = np.zeros((sim.capacity, 7))
    rows[:count] = np.stack([mine.x, mine.y, mine.z, part.m, mine.ax, mine.ay, mine.az], 1)
    local_rows = torch.from_numpy(rows).to(device)
    if world > 1:
        import torch.distributed as dist

        every = torch.empty((world * sim.capacity, 7), dtype=torch.float64, device=device)
        dist.all_gather_into_tensor(every, local_rows)
        every = every.cpu().numpy()
    else:
        every = rows
    rms = max_rel = None
    if rank == 0:
        full = np.concatenate([every[r * sim.capacity: r * sim.capacity + c]
                               for r, c in enumerate(sim.counts)])
        state = nb.ParticleSystem.from_arrays(full[:, :3], np.zeros((n, 3)), full[:, 3])
        targets = np.random.default_rng(7).choice(n, min(4096, n), replace=False)
        with nb.CudaContext() as oracle_ctx:
            oracle_ctx.upload(state)
            ref = oracle_ctx.reference_acceleration(g, targets)
        acc = full[targets, 4:7]
        rms = float(np.sqrt(np.sum((acc - ref) ** 2) / np.sum(ref ** 2)))
        max_rel = float(np.max(np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)))

    peaks, peak_kind = measured_peaks()
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    peak_max = fp32_peak_tflops(sm_count, peaks.get("sm_max_mhz", 1965.0))
    kernel_ms = float(np.mean(force_ms))
    flops = FLOPS_PAIR * float(count) * float(n)
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    roofline = {"bound": "fp32", "kernel": "allpairs_force_kernel (this rank's targets)",
                "achieved": round(achieved, 3), "peak": round(peak_max, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak_max, 4),
                "peak_kind": f"FP32 = {sm_count} SMs x 128 lanes x 2 x "
                             f"{peaks.get('sm_max_mhz', 1965.0)} MHz ({peak_kind})",
                "flops_per_launch": flops, "launch_ms": round(kernel_ms, 4), "traffic": None,
                "all_gather_bytes_per_step": 16 * world * sim.capacity}
    ctx.close()
    return dict(value=n * args.steps / (total_ms * 1e-3), total_ms=total_ms, rms=rms,
                max_rel=max_rel, drift=None, roofline=roofline, clocks=clocks.summary(),
                launches=launches, e2e=None,
                interactions_per_s=float(n) * n * args.steps / (total_ms * 1e-3),
                stats={"particles": n, "ranks": world, "slice": count,
                       "slice_capacity": sim.capacity},
                timings={"step_ms_mean": round(float(np.mean(step_ms)), 4),
                         "force_ms_mean": round(kernel_ms, 4)})


def ctx_timings_summary(step_ms, walk_ms, phases=()):
    out = {"step_ms_mean": round(float(np.mean(step_ms)), 4),
           "walk_ms_mean": round(float(np.mean(walk_ms)), 4)}
    for key in ("bounds_ms", "keys_ms", "sort_ms", "build_ms", "moments_ms", "integrate_ms"):
        if phases:
            out[key.replace("_ms", "_ms_mean")] = round(float(np.mean([p[key] for p in phases])), 4)
    return out


def run_e2e(nb, wl, pos, vel, mass, steps, algo, ctx):
    import torch

    n = wl["n"]
    alloc = lambda k: torch.empty(k, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    s = nb.ParticleSystem.zeros(n, allocator=alloc)
    s.x[:], s.y[:], s.z[:] = pos.T
    s.vx[:], s.vy[:], s.vz[:] = vel.T
    s.m[:] = mass
    g = nb.gravity_init(1.0, wl["eps"])
    c2 = nb.CudaContext(theta=wl.get("theta", 0.7), multipole_order=wl.get("order", 1))
    # the plugin function itself through its C ABI (the ctypes stub a host binds):
    # one view over the pinned arrays, accelerations written in place
    import ctypes as C

    plugin = getattr(nb.library(), "n_body_sim_pro_barnes_hut_compute_acceleration_cuda"
                     if algo == nb.Algorithm.BARNES_HUT
                     else "n_body_sim_pro_gravity_compute_acceleration_cuda")
    view, err = s.view(), nb.Error()

    def force(*_):
        if plugin(C.byref(view), C.byref(g), c2.handle, C.byref(err)) != nb.Status.OK:
            raise nb.CudaError(err.status, err.message.decode(errors="replace"))

    h, dt = 0.5 * wl["dt"], wl["dt"]
    for _ in range(3):  # warm-up of the plugin path
        force()
    # integrator.c:47-85 on the host (in place, on the host's cores), force on the device
    tv = [torch.from_numpy(getattr(s, f)) for f in ("vx", "vy", "vz")]
    tx = [torch.from_numpy(getattr(s, f)) for f in ("x", "y", "z")]
    ta = [torch.from_numpy(getattr(s, f)) for f in ("ax", "ay", "az")]
    t0 = time.perf_counter()
    for _ in range(steps):
        for v, a in zip(tv, ta):
            v.add_(a, alpha=h)
        for x, v in zip(tx, tv):
            x.add_(v, alpha=dt)
        force()
        for v, a in zip(tv, ta):
            v.add_(a, alpha=h)
    elapsed = time.perf_counter() - t0
    c2.close()
    return {"value": n * steps / elapsed, "unit": "particle-steps/s",
            "h2d_bytes_per_step": 4 * 8 * n, "d2h_bytes_per_step": 3 * 8 * n,
            "steps": steps, "path": "host leapfrog (in-place, host threads) + the plugin "
                                    "force function through its C ABI on pinned host arrays",
            "timer": "host wall clock"}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="bh_collision_1m", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-matched", action="store_true",
                    help="skip the matched-accuracy study of the Barnes-Hut workloads")
    ap.add_argument("--theta", type=float, default=None)
    ap.add_argument("--order", type=int, default=None, choices=[1, 2])
    ap.add_argument("--walk", default=None, choices=["lists", "stackless"])
    ap.add_argument("--leaf", type=int, default=None)
    args = ap.parse_args(argv)
    wl = dict(WORKLOADS[args.workload])
    for key in ("theta", "order", "walk", "leaf"):
        if getattr(args, key) is not None:
            wl[key] = getattr(args, key)
    if args.steps is None:
        args.steps = wl["steps"]
    args.warmup = max(args.warmup, 3)
    # the headline metric: the throughput of the workload's configuration, with the
    # chosen-vs-plain figures at rms <= 1e-3 (matched_accuracy) and the dominant
    # kernel's fraction of FP32 peak (roofline) on the same line
    metric = "particle-steps/s at 1e-3 rms force error, chosen vs plain on B200; % FP32 peak"
    unit = "particle-steps/s"
    config = {"workload": args.workload, "particles": wl["n"], "algorithm": wl["algorithm"],
              "theta": wl.get("theta"), "softening": wl["eps"], "timestep": wl["dt"],
              "integrator": "leapfrog_kdk", "multipole_order": wl.get("order"),
              "walk": wl.get("walk", "lists") if wl["algorithm"] == "barnes_hut" else None,
              "leaf_capacity": wl.get("leaf", 16) if wl["algorithm"] == "barnes_hut" else None,
              "initial_conditions": wl["ic"], "l2": "256 MiB write between timed steps",
              "parallelism": f"replicas x{args.gpus}"}

    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        threads = os.cpu_count() or 1
        pos, vel, mass = initial_conditions(wl["ic"], wl["n"], seed=42)
        steps = max(1, min(args.steps, 3))
        for _ in range(1):  # one untimed warm-up step
            reference_steps(wl, pos, vel, mass, 1, threads)
        sec = reference_steps(wl, pos, vel, mass, steps, threads)
        v = wl["n"] / sec
        line = {"impl": "reference", "metric": metric, "value": v, "unit": unit,
                "n_gpus": args.gpus, "steps": steps, "warmup": 1, "ms_per_step": sec * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": unit, "cores": threads, "kind": "reference",
                                 "sample": f"{steps} leapfrog steps of the full {wl['n']}-particle "
                                           f"system (reference engine, OMP_NUM_THREADS={threads}, "
                                           f"{cpu_model()})"},
                "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    world, rank, local = dist_setup(args.gpus)
    sharded = wl["algorithm"] == "all_pairs_sharded" or wl.get("sharded", False)
    if sharded:
        config["parallelism"] = f"sharded x{world}"
    if wl["algorithm"] == "ensemble":
        r = run_ensemble(args, wl, world, rank, local)
        config["particles"] = (sum(ensemble_sizes(wl)) if wl.get("sharded")
                               else r["stats"]["particles"])
    elif wl["algorithm"] == "all_pairs_sharded":
        r = run_sharded_allpairs(args, wl, world, rank, local)
    else:
        r = run_ours(args, wl, world, rank, local)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and wl["algorithm"] != "ensemble":
        try:
            pos, vel, mass = initial_conditions(wl["ic"], wl["n"], seed=42)
            threads = os.cpu_count() or 1
            sec = reference_steps(wl, pos, vel, mass, 1, threads)
            cpu = {"value": wl["n"] / sec, "unit": unit, "cores": threads, "kind": "reference",
                   "sample": f"1 leapfrog step of the full {wl['n']}-particle system, reference "
                             f"engine (oracle/_ref) with OMP_NUM_THREADS={threads} on {cpu_model()}"}
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": unit, "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {exc}"}
    if rank == 0:
        line = {"metric": metric, "value": r["value"], "unit": unit, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": r["total_ms"] / args.steps, "higher_is_better": True,
                "scaling": "strong" if sharded else "weak", "vs_baseline": None,
                "dtype": "f32-force/f64-state",
                "data": "synthetic", "config": config,
                "accuracy": {"rms_rel_force_err": r["rms"], "max_rel_force_err": r["max_rel"],
                             "energy_drift": r["drift"], "oracle": "FP64 device direct sum, "
                             "4096 seeded targets, final state"},
                "interactions_per_s": r["interactions_per_s"], "stats": r["stats"],
                "phase_ms": r["timings"], "roofline": r["roofline"], "cpu_baseline": cpu,
                "e2e": r["e2e"], "gpu_launches": r["launches"], "clocks": r["clocks"]}
        if r.get("matched") is not None:
            line["matched_accuracy"] = r["matched"]
            m = r["matched"]
            if m.get("plain") and m.get("chosen"):
                line["headline"] = {
                    "value_is": "the configuration's throughput (plain walk at its theta)",
                    "chosen_at_rms_1e-3": m["chosen"]["value"],
                    "chosen_method": {k: m["chosen"].get(k) for k in
                                      ("theta", "multipole_order", "opening", "relative_alpha",
                                       "leaf_capacity")},
                    "plain_at_rms_1e-3": m["plain"]["value"],
                    "chosen_over_plain": m.get("chosen_over_plain"),
                    "fp32_peak_frac": r["roofline"].get("frac")}
        if r.get("stages") is not None:
            line["stages_hbm"] = r["stages"]
        if r.get("interactions_split") is not None:
            line["interactions_split"] = r["interactions_split"]
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
