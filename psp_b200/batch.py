"""Batches of independent Helmholtz problems over GPUs and ranks.

The reference solves one problem per SPMD job.  Here many independent
problems (and independent right-hand-side blocks) are spread over devices:
each problem is factored and solved entirely on the GPU it lands on, so the
hot path has no collective; solutions are gathered once at the end.

Assignment is longest-processing-time-first bin packing of a predicted cost
(factor flops and factor bytes streamed by the sweeps, from the host symbolic
analysis of the panel class most panels share), which keeps the slowest
device within 4/3 of the optimum.

``solve_batch`` runs this rank's share.  With ``world > 1`` it is called by
every rank of an initialized ``torch.distributed`` process group (NCCL on
GPUs, gloo on CPU), and the solutions are exchanged with all_gather_object.
With ``streams > 1`` a rank keeps that many problems in flight at once, each
on its own handle and CUDA stream (host threads; the library's calls release
the interpreter lock), so the launches of small problems, which leave most
SMs idle, overlap on the GPU.
"""
import math
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import MIXED, DistHelmholtz, analyze_class

# Throughput assumptions of the cost model (B200, complex-single factors);
# only the ratios between problems matter for the assignment.
_FACTOR_FLOPS_PER_S = 20e12
_SWEEP_BYTES_PER_S = 1.2e12
_ITERATIONS = 15


@dataclass
class Problem:
    """One independent solve: a Discretization, its velocity (natural order,
    nx*ny*nz) and k right-hand sides (natural order, nx*ny*nz x k)."""
    disc: object
    velocity: np.ndarray
    rhs: np.ndarray
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def k(self):
        return self.rhs.size // (self.disc.nx * self.disc.ny * self.disc.nz)


def predicted_cost(disc, k, planes_per_panel=4, cutoff=12, iterations=_ITERATIONS, element_bytes=8):
    """Predicted seconds for Initialize + Solve of one problem."""
    info, _ = analyze_class(disc, planes_per_panel, cutoff, 0)
    s = info[:, 1].astype(np.float64)
    u = info[:, 2].astype(np.float64)
    factor_flops = float(np.sum(8 * (s ** 3 / 6 + s ** 2 * u / 2 + s * u * (u + 1) / 2)))
    factor_bytes = float(np.sum((s + u) * s)) * element_bytes
    panels = max(1, math.ceil(disc.nz / planes_per_panel))
    rhs_blocks = math.ceil(k / 64)
    sweeps = 2 * iterations + 2
    return panels * (factor_flops / _FACTOR_FLOPS_PER_S +
                     sweeps * 2 * rhs_blocks * factor_bytes / _SWEEP_BYTES_PER_S)


def lpt_assign(costs, bins):
    """Longest processing time first: problems in decreasing cost, each to the
    least-loaded bin (lowest index on ties).  Returns (bins, loads)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    out = [[] for _ in range(bins)]
    loads = [0.0] * bins
    for i in order:
        b = min(range(bins), key=lambda j: (loads[j], j))
        out[b].append(i)
        loads[b] += costs[i]
    return out, loads


def _gpu_solver(problem, device, precision):
    H = DistHelmholtz(problem.disc, device=device)
    H.Initialize(problem.velocity, precision=precision)
    return H


def solve_batch(problems, m=20, rel_tol=1e-4, precision=MIXED, rank=0, world=1, device=0, gather=True,
                costs=None, make_solver=None, streams=1):
    """Solves this rank's share of ``problems`` (LPT over ``world`` ranks).

    Returns (solutions, report): ``solutions`` maps problem index to
    (X, stats) for this rank's problems, or for every problem when
    ``gather`` and world > 1; ``report`` holds the assignment and predicted
    loads.  ``make_solver(problem, device, precision)`` returns an
    initialized object with ``Solve(X, m, rel_tol)`` and ``Finalize()``
    (default: a DistHelmholtz on ``device``).  ``streams``: problems in
    flight at once on this rank, taken in decreasing predicted cost; each
    result is the same as with one stream."""
    if costs is None:
        costs = [predicted_cost(p.disc, p.k) for p in problems]
    bins, loads = lpt_assign(costs, world)
    make_solver = make_solver or _gpu_solver

    def run(i):
        p = problems[i]
        H = make_solver(p, device, precision)
        X = np.ascontiguousarray(p.rhs, dtype=np.complex128).copy()
        st = H.Solve(X, m, rel_tol)
        H.Finalize()
        return i, (X, st)

    if streams > 1 and len(bins[rank]) > 1:
        with ThreadPoolExecutor(max_workers=streams) as ex:
            mine = dict(ex.map(run, bins[rank]))
    else:
        mine = dict(run(i) for i in bins[rank])
    report = {"bins": bins, "predicted_loads": loads, "rank": rank, "world": world, "streams": streams}
    if world > 1 and gather:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        merged = {}
        for part in parts:
            merged.update(part)
        return merged, report
    return mine, report
