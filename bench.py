#!/usr/bin/env python
"""Benchmark of the B200 sweeping-preconditioned Helmholtz solve.

Metric: Helmholtz solve RHS/s to relative residual 1e-4 (GMRES(20)), mixed
precision (complex-single fronts and sweeps, FP64 GMRES) next to the plain
FP64 path; gradients/s beside it.

Workload (default ``large_220``): the 200 x 200 x 100 interior with 10 PML
points per face (220 x 220 x 120 points, 5.8M unknowns), a 12-layer velocity
of 1.5-6.0 with three dipping faults and one anticline, omega at 10 points
per wavelength of the slowest layer, 64 Gaussian sources; seeded synthetic
inputs built by psp_b200.workloads.

A step is one Solve of one GMRES block of right-hand sides against factors
from one Initialize: the 64 sources go through the solver in equal blocks
as wide as device memory allows next to the complex-single factors (the
width the library itself picks for a 64-source Solve; 32 on a B200), so a
64-source job is two steps.  ``value`` is solve-only RHS/s (right-hand
sides / device time of the Solve calls), the figure the reference's drivers
report when they time Solve apart from Initialize; Initialize is timed on
its own and setup+solve RHS/s is reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--config NAME]

Under torchrun every rank solves its own copy of the workload (weak scaling,
no collective on the data path); timing is the max over ranks of the device
time between CUDA events on the solver's stream.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Helmholtz solve RHS/s to rel. resid 1e-4: mixed vs FP64 on B200; gradients/s"
UNIT = "RHS/s"
REL_TOL = 1e-4
RESTART = 20

# GMRES(20) inner steps the FP64 path takes to 1e-4 on each workload; the
# CPU model multiplies its sampled per-step costs by this count (the FP64 GPU
# path runs the oracle's algorithm step for step, so its count is the
# oracle's).  Workloads not listed use the count of the run's own solve.
FP64_ITERATIONS = {"smooth_anomalies_116": 15, "plain_bump_50": 16, "large_220": 8}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="large_220")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison arm")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-grad", action="store_true", help="skip the gradients/s arm")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch-of-48-problems arm")
    ap.add_argument("--grad-config", default="layered_faults_96")
    ap.add_argument("--grid-probe", action="store_true",
                    help="time grid ingest: a ZYX-ordered velocity file loaded to the device and resampled 2x")
    ap.add_argument("--sweep-probe", action="store_true",
                    help="profiling driver: Initialize (mixed) + two sweeps on the device, then exit")
    ap.add_argument("--stencil-probe", action="store_true",
                    help="profiling driver: Initialize (mixed) + three global operator applications, then exit")
    return ap.parse_args()


def grid_probe(args):
    """Grid ingest on the device (SequentialLoad + InterpolateTo): the
    workload's velocity written as a ZYX-ordered binary file, loaded back
    in natural order, then resampled to twice the points per axis.  Times
    from CUDA events around the (synchronous) C-ABI calls; bytes are the
    file bytes (load: host read, copy and reorder) and the interpolation's
    output bytes plus one read of its input."""
    import torch
    import psp_b200 as P
    w = workload(args.config)
    nx, ny, nz = w.disc.nx, w.disc.ny, w.disc.nz
    path = os.path.join(tempfile.mkdtemp(), "velocity_zyx.bin")
    # ZYX order: z fastest, then y, then x
    np.ascontiguousarray(w.velocity.reshape(nz, ny, nx).transpose(2, 1, 0)).tofile(path)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for rep in range(3):  # the last repetition is reported
        e[0].record()
        vel = P.load_grid(path, nx, ny, nz, 1, P.ZYX)
        e[1].record()
        e[2].record()
        big = P.interpolate_grid(vel, (nx, ny, nz), (2 * nx, 2 * ny, 2 * nz))
        e[3].record()
        torch.cuda.synchronize()
    os.remove(path)
    n0, n1 = nx * ny * nz, 8 * nx * ny * nz
    t_load, t_int = e[0].elapsed_time(e[1]) * 1e-3, e[2].elapsed_time(e[3]) * 1e-3
    print(json.dumps({"probe": "grid_ingest", "grid": [nx, ny, nz], "load_s": t_load,
                      "load_gbs": 8 * n0 / t_load / 1e9, "interpolate_to": [2 * nx, 2 * ny, 2 * nz],
                      "interpolate_s": t_int, "interpolate_gbs": 8 * (n0 + n1) / t_int / 1e9,
                      "checksum": float(big.sum())}), flush=True)


def sweep_probe(args):
    import torch
    import psp_b200 as P
    w = workload(args.config)
    H = P.DistHelmholtz(w.disc)
    H.Initialize(torch.from_numpy(w.velocity.reshape(-1)).cuda(), precision=P.MIXED)
    B = torch.from_numpy(w.rhs.reshape(-1)).cuda()
    for _ in range(2):
        H.precondition_device(B)
    torch.cuda.synchronize()
    print("sweep probe done", args.config, flush=True)


def stencil_probe(args):
    import torch
    import psp_b200 as P
    w = workload(args.config)
    H = P.DistHelmholtz(w.disc)
    H.Initialize(torch.from_numpy(w.velocity.reshape(-1)).cuda(), precision=P.MIXED)
    B = w.rhs_torch("cuda")
    for _ in range(3):
        H.multiply_device(B)
    torch.cuda.synchronize()
    print("stencil probe done", args.config, flush=True)


def load_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return dict(hbm_gbs=p["hbm_gbs"], bf16_tflops=p["bf16_tflops"], source="measured")
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, source="fallback")


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = max(smax, float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    from psp_b200 import ranks
    ws, rank, local = ranks.from_env()
    if ws > 1:
        ranks.init("nccl", 300, local)
    return ws, rank, local


def max_over_ranks(x, ws):
    from psp_b200 import ranks
    return ranks.max_over_ranks(x, ws)


def barrier(ws):
    from psp_b200 import ranks
    ranks.barrier(ws)


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass


def workload(name):
    from psp_b200 import workloads as W
    return W.CONFIGS[name]()


def config_dict(name, w, kb):
    """The workload as both arms name it."""
    return {"workload": name, "grid": [w.disc.nx, w.disc.ny, w.disc.nz], "interior": list(w.interior),
            "pml": w.pml, "k": w.k, "rhs_per_step": kb, "gmres_restart": RESTART, "rel_tol": REL_TOL,
            "step": "Solve of one GMRES block of rhs_per_step right-hand sides (factors from one Initialize, "
                    "timed apart)",
            "l2": "inputs larger than L2 (factors > 10 GB)", "parallelism": "independent problem per GPU"}


# GMRES block width of each workload's mixed-precision solve on one B200
# (what the library picks for all k sources next to its complex-single
# factors); the reference arm, which runs without a GPU, names the same
# block.  Workloads not listed solve all k at once.
BLOCK_WIDTH = {"large_220": 32}


def ev():
    import torch
    return torch.cuda.Event(enable_timing=True)


def time_initialize(H, vel_d, precision, reps, stream):
    """Milliseconds of `reps` timed Initialize calls after one untimed one."""
    H.Initialize(vel_d, precision=precision)
    ms = []
    for _ in range(reps):
        e0, e1 = ev(), ev()
        e0.record(stream)
        H.Initialize(vel_d, precision=precision)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


def block_cols(w, kb, i):
    """Sources of block i (blocks of kb cycle over the k sources)."""
    nb = -(-w.k // kb)
    c0 = (i % nb) * kb
    return range(c0, min(w.k, c0 + kb))


def solve_steps(H, w, kb, steps, warmup, ws, stream, clocks=None):
    """Times `steps` block Solves (after `warmup` untimed ones) with CUDA
    events on the solver stream; each step's right-hand sides are written on
    the device before its events."""
    import torch
    N = w.disc.nx * w.disc.ny * w.disc.nz
    X = torch.empty(N * kb, dtype=torch.complex128, device="cuda")

    def step(i, rec):
        cols = block_cols(w, kb, i)
        Xv = X[:N * len(cols)]
        w.rhs_torch("cuda", Xv, cols)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        st = H.Solve(Xv, RESTART, REL_TOL)
        e1.record(stream)
        e1.synchronize()
        rec.append((e0.elapsed_time(e1), len(cols), st))

    junk = []
    for i in range(warmup):
        step(i, junk)
    barrier(ws)
    torch.cuda.synchronize()
    recs = []
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        for i in range(steps):
            step(warmup + i, recs)
        torch.cuda.synchronize()
    barrier(ws)
    total_ms = max_over_ranks(sum(r[0] for r in recs), ws)
    rhs = sum(r[1] for r in recs)
    return dict(total_ms=total_ms, rhs=rhs, stats=[r[2] for r in recs], X=X)


# timed gradients (and warm-up ones) at most, whatever the main arm's steps
GRAD_STEPS = 5


def gradient_arm(args, ws, local):
    """Gradients/s: each step is one full misfit gradient of a velocity model
    -- Initialize (mixed), forward solve of every source, adjoint solve with
    the same factors and the device gradient kernel -- through the torch
    autograd layer (psp_b200.autograd)."""
    import torch
    import psp_b200 as P
    from psp_b200.autograd import misfit_and_gradient
    w = workload(args.grad_config)
    N = w.disc.nx * w.disc.ny * w.disc.nz
    k = w.k
    H = P.DistHelmholtz(w.disc, device=local)
    vel = torch.from_numpy(w.velocity.reshape(-1)).cuda()
    f = torch.from_numpy(np.ascontiguousarray(w.rhs.reshape(N, k))).cuda()
    recv = torch.from_numpy(w.meta["receivers"]).cuda()
    H.Initialize(torch.from_numpy(w.meta["observed_model"].reshape(-1)).cuda(), precision=P.FP64)
    u_obs = f.clone()
    H.Solve(u_obs, RESTART, REL_TOL)
    data = u_obs[recv].clone()
    del u_obs
    steps, warmup = min(args.steps, GRAD_STEPS), min(args.warmup, GRAD_STEPS)
    for _ in range(max(1, warmup)):
        J, g = misfit_and_gradient(H, vel, f, recv, data, RESTART, REL_TOL, P.MIXED)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        J, g = misfit_and_gradient(H, vel, f, recv, data, RESTART, REL_TOL, P.MIXED)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), ws)
    out = {"value": ws * steps / (ms * 1e-3), "unit": "gradients/s", "ms_per_gradient": ms / steps,
           "steps": steps,
           "workload": args.grad_config, "grid": [w.disc.nx, w.disc.ny, w.disc.nz], "sources": k,
           "receivers": int(len(w.meta["receivers"])), "precision": "mixed",
           "step": "Initialize + forward solve + adjoint solve + gradient kernel",
           "misfit": float(J), "gradient_norm": float(torch.linalg.norm(g)),
           # the misfit relative to the data's own energy, 0.5 ||d||^2
           "relative_misfit": float(J) / (0.5 * float(torch.linalg.norm(data)) ** 2),
           "data_norm": float(torch.linalg.norm(data))}
    H.Finalize()
    return out


# problems in flight per rank in the batch arm (one handle and stream each)
BATCH_STREAMS = 4


def batch_arm(args, ws, rank, local):
    """Throughput over the batching workload: 48 independent problems (sides
    32-96, k = 1-8) split over the ranks by predicted cost (longest
    processing time first); every rank factors and solves its share
    (mixed precision) with no communication; RHS/s = all right-hand sides /
    the slowest rank's time.  Solutions stay on their rank (no gather)."""
    import torch
    import psp_b200 as P
    from psp_b200 import batch as B
    probs = W_batch()
    costs = [B.predicted_cost(p.disc, p.k) for p in probs]
    bins, loads = B.lpt_assign(costs, ws)
    warm = probs[min(range(len(probs)), key=lambda i: costs[i])]
    B.solve_batch([warm], precision=P.MIXED, device=local, costs=[1.0])
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, rep = B.solve_batch(probs, RESTART, REL_TOL, P.MIXED, rank, ws, local, gather=False, costs=costs,
                           streams=BATCH_STREAMS)
    torch.cuda.synchronize()
    sec = max_over_ranks(time.perf_counter() - t0, ws)
    total_k = sum(p.k for p in probs)
    return {"value": total_k / sec, "unit": "RHS/s", "seconds": sec, "problems": len(probs), "rhs": total_k,
            "workload": "batch_48", "precision": "mixed", "scaling": "strong (fixed batch over ranks)",
            "predicted_loads_s": [round(x, 4) for x in loads],
            "problems_per_rank": [len(b) for b in bins], "streams_per_rank": BATCH_STREAMS,
            "timing": "host wall clock around the rank's share, max over ranks (many short solves)"}


def W_batch():
    from psp_b200 import workloads as W
    return W.batch_problems()


def fp64_sample(H, w, vel_d, stream, mixed_block0):
    """The plain FP64 path on the same workload, measured once: one timed
    Initialize (after an untimed one; panels whose complex-double factors do
    not fit are recomputed during the sweeps), then one Solve of the first
    GMRES block the FP64 handle picks for the k sources."""
    import torch
    import psp_b200 as P
    setup = time_initialize(H, vel_d, P.FP64, 1, stream)
    mem = H.memory_info()
    kb = H.solve_block_width(w.k, RESTART)
    N = w.disc.nx * w.disc.ny * w.disc.nz
    cols = range(0, kb)
    X = w.rhs_torch("cuda", cols=cols)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record(stream)
    st = H.Solve(X, RESTART, REL_TOL)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    refactors = H.memory_info()["refactorizations"]
    out = {"value": kb / (ms * 1e-3), "unit": UNIT, "rhs": kb, "steps": 1,
           "solve_ms": ms, "setup_ms": setup[0], "iterations": st["iterations"],
           "final_rel_resid": st["final_max_rel_resid"], "converged": st["converged"],
           "resident_panels": mem["resident_panels"], "num_panels": mem["num_panels"],
           "refactorizations_in_solve": refactors,
           "setup_plus_solve_rhs_per_s": w.k / ((setup[0] + math.ceil(w.k / kb) * ms) * 1e-3),
           "note": ("one Solve of the first %d sources; setup+solve counts one Initialize and %d such blocks"
                    % (kb, math.ceil(w.k / kb)))}
    if mixed_block0 is not None:
        n = min(kb, mixed_block0.shape[-1])
        a = torch.from_numpy(mixed_block0[..., :n].reshape(-1)).cuda()
        b = X.view(N, kb)[:, :n].reshape(-1)
        out["mixed_rel_diff_vs_fp64"] = float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    del X
    return out


def e2e_arm(H, w, vel_h, kb, nsteps, ws, stream):
    """The same metric through the public API with host buffers: each step
    is one Solve of a block of kb host right-hand sides (numpy), so its
    host-to-device copy of the sources and device-to-host copy of the
    wavefields are inside the timed region; Initialize from the host
    velocity first (timed apart, as in the device-resident arm)."""
    import torch
    import psp_b200 as P
    H.Initialize(vel_h, precision=P.MIXED)
    blocks = [w.rhs_host(block_cols(w, kb, i)) for i in range(min(nsteps, -(-w.k // kb)))]
    B = blocks[0].copy()
    H.Solve(B, RESTART, REL_TOL)  # untimed: the handle's pinned staging and device scratch
    barrier(ws)
    torch.cuda.synchronize()
    ms = 0.0
    rhs = 0
    for i in range(nsteps):
        B = blocks[i % len(blocks)].copy()
        e0, e1 = ev(), ev()
        e0.record(stream)
        H.Solve(B, RESTART, REL_TOL)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        rhs += B.shape[-1]
    ms = max_over_ranks(ms, ws)
    N = w.disc.nx * w.disc.ny * w.disc.nz
    return {"value": ws * rhs / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(N * kb * 16),
            "d2h_bytes_per_step": int(N * kb * 16), "steps": nsteps,
            "path": "psp_cu_solve with host buffers (pinned staging ring, copies inside the timed region)"}


def profile_block(H, w, kb, stream):
    """One block Solve with per-kernel profiling (sweeps eager)."""
    import torch
    N = w.disc.nx * w.disc.ny * w.disc.nz
    X = w.rhs_torch("cuda", cols=block_cols(w, kb, 0))
    H.set_profiling(True)
    H.profile_reset()
    H.Solve(X, RESTART, REL_TOL)
    torch.cuda.synchronize()
    prof = H.profile()
    H.set_profiling(False)
    del X
    return prof


# DRAM bytes per algorithmic byte of a sweep launch, from one ncu capture
# of each 32-column tensor-core sweep kernel on the differentiation workload
# (forward depth 8 and backward depth 2: 96.7 + 29.0 MB of DRAM traffic for
# 73.4 + 30.5 MB of algorithmic bytes; profiles/)
SWEEP_TRAFFIC_RATIO = (96.7e6 + 29.0e6) / (73.4e6 + 30.5e6)


def roofline_entry(name, p, peaks):
    sec = p["ms"] * 1e-3
    ai = p["flops"] / max(p["bytes"], 1.0)
    ridge = peaks["bf16_tflops"] * 1e12 / (peaks["hbm_gbs"] * 1e9)
    if ai > ridge:
        out = {"bound": "tensor", "achieved": p["flops"] / sec / 1e12, "peak": peaks["bf16_tflops"],
               "unit": "TFLOP/s"}
    else:
        out = {"bound": "hbm", "achieved": p["bytes"] / sec / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s"}
    out["frac"] = out["achieved"] / out["peak"]
    out["kernel"] = name
    out["launches"] = p["launches"]
    out["avg_launch_us"] = p["ms"] * 1e3 / max(p["launches"], 1)
    out["algorithmic_flops_per_launch"] = p["flops"] / max(p["launches"], 1)
    out["algorithmic_bytes_per_launch"] = p["bytes"] / max(p["launches"], 1)
    out["peak_source"] = peaks["source"]
    return out


def roofline_from_profile(prof, peaks):
    kernels = {k: v for k, v in prof.items() if k != "sweep" and v["launches"] > 0}
    name = max(kernels, key=lambda k: kernels[k]["ms"])
    out = roofline_entry(name, kernels[name], peaks)
    if name == "solve_gemm":
        out["traffic"] = SWEEP_TRAFFIC_RATIO * kernels[name]["bytes"] / max(kernels[name]["launches"], 1)
        out["traffic_note"] = ("dram__bytes_read+write per launch, scaled from ncu captures of the 32-column "
                               "forward and backward sweep kernels (1.21x algorithmic)")
    else:
        out["traffic"] = None
    others = {n: roofline_entry(n, kernels[n], peaks) for n in ("stencil", "gmres_vector") if n in kernels}
    return out, others


def cpu_sample(w, its, kb, full_factor, steps, warmup):
    """Bounded CPU sample of the workload with the FP64 oracle restatement
    on every host thread: the global operator, one panel solve of the
    bottom panel class for as many right-hand sides as threads, one matvec
    of as many; the top panel's solve is scaled from it by its factor
    nonzeros (the panel solve streams the factors), right-hand sides
    linearly (they run one per thread).  With `full_factor` one bottom-class
    panel is also factored (timed) and the top panel's factorization scaled
    by its flops; otherwise the solves run on unit-diagonal fronts of the
    panel's structure (same bytes and operations as real factors).  Returns
    (modeled rates, per-step wall seconds, threads)."""
    import oracle
    import psp_b200 as P
    d = w.disc
    O = oracle.Oracle(oracle.make_disc(d.omega, d.nx, d.ny, d.nz, d.wx, d.wy, d.wz,
                                       pml=(d.bx, d.by, d.bz), sigma=d.sigmax))
    threads = oracle.num_threads()
    geo = O.geometry()
    np_ = geo.shape[0]
    t0 = time.time()
    O.form_operator(w.velocity)
    t_op = time.time() - t0
    # per-class factor nonzeros and flops (host analysis)
    nnz, flops = {}, {}
    for c in sorted(set(int(x) for x in geo[:, 3])):
        info, _ = P.analyze_class(w.disc, 4, 12, c)
        s, u = info[:, 1].astype(float), info[:, 2].astype(float)
        nnz[c] = float(((s + u) * s - s * (s - 1) / 2).sum())
        flops[c] = float((8 * (s ** 3 / 3 + s ** 2 * u) + 8 * s ** 3 / 6 + 8 * s ** 2 * u / 2 + 4 * s * u ** 2).sum())
    p0 = 0
    c0 = int(geo[p0, 3])
    t_factor = oracle.time_factor_panel(O, w.velocity, p0) if full_factor else None
    kS = max(1, min(threads, w.k))
    walls, ps, mv = [], [], []
    for i in range(warmup + steps):
        t = time.time()
        a = oracle.time_panel_solve(O, p0, kS)
        b = oracle.time_multiply(O, kS)
        if i >= warmup:
            walls.append(time.time() - t)
            ps.append(a)
            mv.append(b)
    oracle.release_panel(O, p0)
    ps0 = min(ps) * w.k / kS
    mvk = min(mv) * w.k / kS
    sweep = sum((1 if p == np_ - 1 else 2) * ps0 * nnz[int(geo[p, 3])] / nnz[c0] for p in range(np_))
    solve = (its + 1) * sweep + 2 * its * mvk
    out = {"solve_only_rhs_per_s": w.k / solve, "modeled_solve_s": solve, "sweep_s": sweep,
           "panel_solve_s": ps0, "matvec_s": mvk, "operator_s": t_op, "iterations": its}
    if t_factor is not None:
        setup = t_op + sum(t_factor * flops[int(geo[p, 3])] / flops[c0] for p in range(np_))
        out.update({"factor_panel_s": t_factor, "modeled_setup_s": setup,
                    "setup_plus_solve_rhs_per_s": w.k / (setup + solve)})
    return out, walls, threads


def workload_iterations(name, fallback):
    return FP64_ITERATIONS.get(name) or fallback


def model_check(name="plain_bump_50"):
    """The sampled model next to a whole oracle Initialize + Solve of the
    small FP64 reference case (seconds on the host cores)."""
    import oracle
    w = workload(name)
    d = w.disc
    m, _, _ = cpu_sample(w, workload_iterations(name, 20), w.k, True, 1, 0)
    O = oracle.Oracle(oracle.make_disc(d.omega, d.nx, d.ny, d.nz, d.wx, d.wy, d.wz,
                                       pml=(d.bx, d.by, d.bz), sigma=d.sigmax))
    t0 = time.time()
    O.initialize(w.velocity)
    t1 = time.time()
    _, st = O.solve(w.rhs, RESTART, REL_TOL)
    t2 = time.time()
    return {"workload": name, "iterations": st["iterations"],
            "modeled_solve_only_rhs_per_s": m["solve_only_rhs_per_s"], "measured_solve_only_rhs_per_s": w.k / (t2 - t1),
            "modeled_setup_plus_solve_rhs_per_s": m["setup_plus_solve_rhs_per_s"],
            "measured_setup_plus_solve_rhs_per_s": w.k / (t2 - t0)}


def main_reference(args):
    """CPU arm: the FP64 oracle restatement of the reference on the host
    cores, a bounded sample of the same workload per step (cpu_sample),
    reported in the same metric and config."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t_start = time.time()
    w = workload(args.config)
    kb = BLOCK_WIDTH.get(args.config, w.k)
    its = workload_iterations(args.config, 20)
    m, walls, threads = cpu_sample(w, its, kb, True, args.steps, args.warmup)
    value = m["solve_only_rhs_per_s"]
    sample = ("oracle FP64 restatement on %d host threads; once: global operator and one factorization of the "
              "bottom panel class (%.1f s, the top panel's scaled by its flops); per step: one solve of that "
              "panel and one matvec for %d right-hand sides (threads run one each), scaled linearly to the "
              "%d sources and, for the top panel, by its factor nonzeros; modeled Solve = (%d GMRES steps + 1) "
              "sweeps of 2P-1 panel solves + 2 matvecs per step" %
              (threads, m.get("factor_panel_s", 0.0), min(threads, w.k), w.k, its))
    check = model_check()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic", "config": config_dict(args.config, w, kb),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "model": m, "model_check": check, "wall_s": time.time() - t_start,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.grid_probe:
        return grid_probe(args)
    if args.sweep_probe:
        return sweep_probe(args)
    if args.stencil_probe:
        return stencil_probe(args)
    if args.impl == "reference":
        return main_reference(args)
    import torch
    import psp_b200 as P
    ws, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    w = workload(args.config)
    N = w.disc.nx * w.disc.ny * w.disc.nz
    vel_d = torch.from_numpy(w.velocity.reshape(-1)).to("cuda")
    H = P.DistHelmholtz(w.disc, device=local)
    stream = torch.cuda.ExternalStream(H.stream_ptr(), device=torch.device("cuda", local))
    peaks = load_peaks()

    # mixed precision: Initialize timed apart, then block Solve steps
    setup_ms = time_initialize(H, vel_d, P.MIXED, 2, stream)
    kb = H.solve_block_width(w.k, RESTART)
    clocks = ClockSampler(local)
    mixed = solve_steps(H, w, kb, args.steps, args.warmup, ws, stream, clocks)
    st_m = mixed["stats"][-1]
    value = ws * mixed["rhs"] / (mixed["total_ms"] * 1e-3)
    setup_s = max_over_ranks(statistics.mean(setup_ms), ws) * 1e-3
    block_s = mixed["total_ms"] * 1e-3 / args.steps
    nb = math.ceil(w.k / kb)
    setup_plus_solve = w.k / (setup_s + nb * block_s)
    # the first block's mixed wavefields, for the FP64 comparison
    X0 = w.rhs_torch("cuda", cols=block_cols(w, kb, 0))
    H.Solve(X0, RESTART, REL_TOL)
    mixed_block0 = X0.cpu().numpy().reshape(N, -1)
    del X0, mixed["X"]
    torch.cuda.empty_cache()
    prof = profile_block(H, w, kb, stream)
    roof, other_roofs = roofline_from_profile(prof, peaks)
    launches_per_step = sum(v["launches"] for n, v in prof.items() if n != "sweep")
    mem_mixed = H.memory_info()

    e2e = None
    if not args.no_e2e:
        vel_h = np.ascontiguousarray(w.velocity.reshape(-1))
        e2e = e2e_arm(H, w, vel_h, kb, max(1, min(args.steps, nb)), ws, stream)

    H.Finalize()
    torch.cuda.empty_cache()
    fp64 = None
    if not args.no_fp64:
        fp64 = fp64_sample(H, w, vel_d, stream, mixed_block0)
        H.Finalize()
        torch.cuda.empty_cache()

    batch = None
    if not args.no_batch:
        batch = batch_arm(args, ws, rank, local)

    grad = None
    if not args.no_grad:
        grad = gradient_arm(args, ws, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        its = workload_iterations(args.config, fp64["iterations"] if fp64 else st_m["iterations"])
        m, walls, threads = cpu_sample(w, its, kb, False, 2, 0)
        cpu = {"value": m["solve_only_rhs_per_s"], "unit": UNIT, "cores": threads, "kind": "port",
               "sample": ("oracle FP64 restatement on %d host threads: one bottom-class panel solve and one "
                          "matvec for %d right-hand sides on the full workload (%.1f s of CPU work), scaled to "
                          "the %d sources, every panel (top panel by its factor nonzeros) and %d GMRES steps"
                          % (threads, min(threads, w.k), sum(walls), w.k, its)),
               "model": m}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mixed["total_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 fronts/sweeps + c128 GMRES",
            "data": "synthetic", "config": config_dict(args.config, w, kb),
            "setup_ms": 1e3 * setup_s, "setup_plus_solve_rhs_per_s": setup_plus_solve,
            "iterations": st_m["iterations"], "final_rel_resid": st_m["final_max_rel_resid"],
            # device time of the last timed Solve by phase (events at GMRES's own sync points)
            "solve_phases_s": {"precondition": st_m["precondition_seconds"], "matvec": st_m["matvec_seconds"],
                               "arnoldi": st_m["arnoldi_seconds"], "preconditions": st_m["num_preconditions"],
                               "wall": st_m["solve_seconds"]},
            "converged": all(s["converged"] for s in mixed["stats"]),
            "memory": mem_mixed,
            "fp64": fp64,
            "mixed_over_fp64": (value / fp64["value"]) if fp64 else None,
            "mixed_over_fp64_setup_plus_solve": (setup_plus_solve / fp64["setup_plus_solve_rhs_per_s"])
            if fp64 else None,
            "e2e": e2e,
            "gradients_per_s": grad,
            "batch": batch,
            "roofline": roof,
            "rooflines_other": other_roofs,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "gpu_launches": int(launches_per_step * args.steps),
            "breakdown_ms": {n: round(v["ms"], 3) for n, v in prof.items() if v["launches"]},
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
