"""Batches of independent problems: cost model and LPT assignment (CPU),
the multi-rank path with two gloo ranks on CPU (assignment, timing reduction
and the gather of solutions, with a sparse direct solver standing in for the
GPU), and GPU batches against one-by-one solves."""
import itertools
import os
import socket

import numpy as np
import pytest

import helmholtz_np as hn
from psp_b200 import batch as B
from psp_b200 import workloads as W


def test_lpt_assignment_is_complete_and_balanced():
    rng = np.random.Generator(np.random.PCG64(3))
    for n, bins in ((7, 2), (9, 3), (12, 4)):
        costs = list(rng.uniform(1, 10, size=n))
        out, loads = B.lpt_assign(costs, bins)
        assert sorted(itertools.chain(*out)) == list(range(n))
        assert np.allclose(loads, [sum(costs[i] for i in b) for b in out])
        best = min(max(sum(costs[i] for i in range(n) if a[i] == b) for b in range(bins))
                   for a in itertools.product(range(bins), repeat=n)) if n <= 9 else sum(costs) / bins
        assert max(loads) <= 4.0 / 3.0 * best + 1e-9


def test_predicted_cost_grows_with_size():
    small = W.make_disc((20, 20, 20), 5, 20.0)
    large = W.make_disc((40, 40, 40), 5, 20.0)
    assert B.predicted_cost(large, 4) > 4 * B.predicted_cost(small, 4)
    assert B.predicted_cost(small, 128) > B.predicted_cost(small, 4)


def test_batch_workload_shapes():
    probs = W.batch_problems(count=6)
    for p in probs:
        n = p.disc.nx * p.disc.ny * p.disc.nz
        assert p.velocity.shape == (n,) and p.rhs.shape[0] == n and 1 <= p.k <= 8
        assert 0.6 <= p.velocity.min() and p.velocity.max() <= 1.8
        assert all(32 <= m <= 96 for m in p.meta["sides"])


class _DirectSolver:
    """Sparse direct solve of the global operator (CPU stand-in for a GPU)."""

    def __init__(self, p):
        import scipy.sparse.linalg as spla
        d = p.disc
        self.lu = spla.splu(hn.global_matrix(d, p.velocity.reshape(d.nz, d.ny, d.nx)).tocsc())

    def Solve(self, X, m, rel_tol):
        X[...] = self.lu.solve(np.ascontiguousarray(X))
        return {"iterations": 0}

    def Finalize(self):
        pass


def _tiny_problems():
    return W.batch_problems(count=5, seed=77, sides=(20, 22, 24), pml=4, n_anom=1)


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from psp_b200 import ranks
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    ranks.init("gloo", timeout_s=60)
    try:
        assert ranks.max_over_ranks(float(rank) + 0.5, world) == world - 0.5
        ranks.barrier(world)
        probs = _tiny_problems()
        sols, rep = B.solve_batch(probs, rank=rank, world=world, make_solver=lambda p, dev, prec: _DirectSolver(p))
        assert sorted(sols) == list(range(len(probs)))
        assert set(rep["bins"][rank]) <= set(sols)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), *[sols[i][0] for i in range(len(probs))])
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_share_and_gather_a_batch(tmp_path, monkeypatch):
    import torch.multiprocessing as mp
    # one BLAS thread per rank: two ranks' thread pools on the same cores
    # stall the sparse factorizations
    for v in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
        monkeypatch.setenv(v, "1")
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    probs = _tiny_problems()
    ref, _ = B.solve_batch(probs, make_solver=lambda p, dev, prec: _DirectSolver(p))
    for r in range(2):
        got = np.load(tmp_path / ("rank%d.npz" % r))
        for i in range(len(probs)):
            # same solves; BLAS threading may differ between the ranks and this process
            assert np.linalg.norm(got["arr_%d" % i] - ref[i][0]) <= 1e-12 * np.linalg.norm(ref[i][0])


def test_concurrent_streams_give_the_same_solutions():
    probs = _tiny_problems()
    make = lambda p, dev, prec: _DirectSolver(p)
    ref, _ = B.solve_batch(probs, make_solver=make)
    got, rep = B.solve_batch(probs, make_solver=make, streams=3)
    assert sorted(got) == sorted(ref) and rep["streams"] == 3
    for i in ref:
        assert np.array_equal(got[i][0], ref[i][0])


@pytest.mark.gpu
@pytest.mark.parametrize("precision,streams", [("fp64", 1), ("fp64", 3), ("mixed", 3)])
def test_gpu_batch_matches_individual_solves(product_lib, precision, streams):
    import psp_b200 as P
    prec = P.FP64 if precision == "fp64" else P.MIXED
    probs = W.batch_problems(count=4, seed=5, sides=(32, 36, 40))
    sols, rep = B.solve_batch(probs, rel_tol=1e-8, precision=prec, streams=streams)
    for i, p in enumerate(probs):
        H = P.DistHelmholtz(p.disc)
        H.Initialize(p.velocity, precision=prec)
        X = p.rhs.copy()
        H.Solve(X, 20, 1e-8)
        # the same kernels on the same inputs: problems in flight together
        # on other streams change nothing
        assert np.linalg.norm(sols[i][0] - X) <= 1e-12 * np.linalg.norm(X)
        assert sols[i][1]["converged"]


@pytest.mark.gpu
def test_c_abi_batch_calls_match_individual_calls(product_lib):
    import psp_b200 as P
    probs = W.batch_problems(count=3, seed=9, sides=(32, 36))
    solvers = [P.DistHelmholtz(p.disc) for p in probs]
    P.initialize_batch(solvers, [p.velocity for p in probs], precision=P.FP64)
    grids = [np.ascontiguousarray(p.rhs).copy() for p in probs]
    stats = P.solve_batch(solvers, grids, 20, 1e-8)
    assert all(s["converged"] for s in stats)
    for p, g in zip(probs, grids):
        H = P.DistHelmholtz(p.disc)
        H.Initialize(p.velocity, precision=P.FP64)
        X = np.ascontiguousarray(p.rhs).copy()
        H.Solve(X, 20, 1e-8)
        assert np.linalg.norm(g - X) <= 1e-12 * np.linalg.norm(X)
    with pytest.raises(P.LogicError):
        P.solve_batch(solvers[:1], [np.zeros(7, dtype=np.complex128)])
