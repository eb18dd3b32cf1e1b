"""The z-panel pipeline (psp_b200.zpanel): panels split over ranks, boundary
planes passed forward and backward through the sweep, halo planes through
the matvec, GMRES inner products summed over ranks.

CPU: two gloo ranks (processes) and three thread ranks, with the FP64
oracle's panel solves and global operator standing in for the GPU, against
the one-process oracle sweep and GMRES solve.  GPU: two ranks as threads of
one process (they only wait for each other on the host), each with a handle
that factors its own panels, against one handle that factors them all.
"""
import os
import socket
import threading

import numpy as np
import pytest

from conftest import oracle_for, rel
from psp_b200 import panel_geometry, workloads as W
from psp_b200 import zpanel as Z

CASE = dict(interior=(12, 13, 22), pml=5, freq=2.0, k=3, seed=17, top_pml=True)


def _case():
    return W.small_case(**CASE)


class OracleSlabBackend:
    """CPU stand-in for the device backend: the oracle's panel solve T_p and
    its global operator, on slabs (the coupling terms of in_mode 1 and 2
    are the operator's entries between the panel and the plane next to it,
    as in the reference's SubdiagonalUpdate / MultiplySuperdiagonal)."""

    def __init__(self, w, layout, O=None):
        self.w, self.L = w, layout
        self.O = O or oracle_for(w.disc)
        if O is None:
            self.O.initialize(w.velocity)
        self.A = self.O.global_operator_natural()
        d = w.disc
        self.shape = (d.nz, d.ny, d.nx)

    def _full(self, W, k):
        L = self.L
        full = np.zeros((L.nz, L.nxy, k), dtype=np.complex128)
        full[L.zs:L.ze] = W.numpy()
        return full

    def _apply(self, full, k):
        return (self.A @ full.reshape(-1, k)).reshape(full.shape)

    def solve_panel(self, W, k, p, in_mode, out_acc, zs):
        import torch
        L = self.L
        lowv, depth = int(L.geometry[p, 0]), int(L.geometry[p, 1])
        z0, z1 = L.nz - lowv - depth, L.nz - lowv  # panel planes [z0, z1)
        full = self._full(W, k)
        rhs = np.zeros_like(full)
        if in_mode in (0, 1):
            rhs[z0:z1] = full[z0:z1]
        if in_mode == 1:  # the plane below the panel in v (above it in z)
            nb = np.zeros_like(full)
            nb[z1] = full[z1]
            rhs[z0:z1] -= self._apply(nb, k)[z0:z1]
        if in_mode == 2:  # the plane above the panel in v
            nb = np.zeros_like(full)
            nb[z0 - 1] = full[z0 - 1]
            rhs[z0:z1] = -self._apply(nb, k)[z0:z1]
        out = self.O.solve_panel(rhs.reshape(*self.shape, k), p).reshape(full.shape)
        res = torch.from_numpy(np.ascontiguousarray(out[z0:z1]))
        if out_acc:
            W[z0 - zs:z1 - zs] += res
        else:
            W[z0 - zs:z1 - zs] = res

    def multiply(self, X, Y, k, z_first, z_count, zs, Bv=None):
        import torch
        full = self._full(X, k)
        ax = self._apply(full, k)[z_first:z_first + z_count]
        sl = slice(z_first - zs, z_first + z_count - zs)
        out = torch.from_numpy(np.ascontiguousarray(ax))
        Y[sl] = (Bv[sl] - out) if Bv is not None else out


def _layouts(w, world):
    geo, costs = Z.panel_costs(w.disc)
    ranges = Z.partition(costs, world)
    return [Z.Layout(geo, w.disc.nz, w.disc.nx * w.disc.ny, r, ranges) for r in range(world)]


def _gather(layouts, parts, shape):
    full = np.zeros(shape, dtype=np.complex128)
    for L, own in zip(layouts, parts):
        full[L.zlo:L.zhi + 1] = own
    return full


def test_partition_is_contiguous_and_balanced():
    costs = [1, 1, 1, 1, 5, 1, 1, 1]
    for world in (1, 2, 3, 4, 8):
        parts = Z.partition(costs, world)
        assert parts[0][0] == 0 and parts[-1][1] == len(costs)
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        assert all(p1 > p0 for p0, p1 in parts)
    assert Z.partition(costs, 2) == [(0, 4), (4, 8)]
    with pytest.raises(ValueError):
        Z.partition(costs, 9)


def test_layout_planes_cover_the_grid_once():
    w = _case()
    geo = panel_geometry(w.disc)
    assert geo.shape[0] >= 4
    for world in (1, 2, 3):
        Ls = _layouts(w, world)
        owned = sorted(z for L in Ls for z in range(L.zlo, L.zhi + 1))
        assert owned == list(range(w.disc.nz))
        for a, b in zip(Ls, Ls[1:]):   # rank r+1 holds the higher panels: lower z
            assert b.zhi + 1 == a.zlo


def _thread_ranks(world, fn):
    comms = Z.ThreadComm.group(world)
    out, errs = [None] * world, []

    def run(r):
        try:
            out[r] = fn(r, comms[r])
        except BaseException as e:  # surface every rank's failure
            errs.append(e)

    th = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    return out


@pytest.mark.parametrize("blocks", [1, 2, 3])
def test_three_thread_ranks_sweep_and_solve_match_one_process(blocks):
    """blocks > 1: the sweep pipelined over blocks of right-hand-side
    columns (a rank passes a block's boundary plane on and starts the next
    block), which must not change any column's result."""
    import torch
    torch.set_num_threads(1)
    w = _case()
    d = w.disc
    O = oracle_for(d)
    O.initialize(w.velocity)
    k, nxy = w.k, d.nx * d.ny
    grid = w.rhs.reshape(d.nz, nxy, k)
    Ls = _layouts(w, 3)

    def rank(r, comm):
        L = Ls[r]
        be = OracleSlabBackend(w, L, O)
        S = Z.ZPanelSolver(L, be, comm, k, blocks=blocks)
        M = Z.scatter_slab(L, grid, k)
        S.precondition(M)
        X = Z.scatter_slab(L, grid, k)
        st = S.solve(X, 20, 1e-8)
        return M[L.own].numpy(), X[L.own].numpy(), st

    res = _thread_ranks(3, rank)
    ref = O.precondition(w.rhs).reshape(d.nz, nxy, k)
    assert rel(_gather(Ls, [r[0] for r in res], ref.shape), ref) < 1e-12
    Xo, sto = O.solve(w.rhs, 20, 1e-8)
    X = _gather(Ls, [r[1] for r in res], ref.shape)
    assert all(r[2]["converged"] and r[2]["iterations"] == sto["iterations"] for r in res)
    assert rel(X, Xo.reshape(ref.shape)) < 1e-9


def _gloo_rank(rank, world, port, out_dir, blocks=1):
    import torch
    import torch.distributed as dist
    from psp_b200 import ranks
    torch.set_num_threads(1)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    ranks.init("gloo", timeout_s=120)
    try:
        w = _case()
        d = w.disc
        k, nxy = w.k, d.nx * d.ny
        grid = w.rhs.reshape(d.nz, nxy, k)
        L = _layouts(w, world)[rank]
        S = Z.ZPanelSolver(L, OracleSlabBackend(w, L), Z.TorchComm(), k, blocks=blocks)
        M = Z.scatter_slab(L, grid, k)
        S.precondition(M)
        X = Z.scatter_slab(L, grid, k)
        st = S.solve(X, 20, 1e-8)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), M=M[L.own].numpy(), X=X[L.own].numpy(),
                 its=st["iterations"], conv=st["converged"])
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("blocks", [1, 2])
def test_two_gloo_ranks_sweep_and_solve_match_one_process(tmp_path, monkeypatch, blocks):
    import torch.multiprocessing as mp
    for v in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
        monkeypatch.setenv(v, "1")
    mp.spawn(_gloo_rank, args=(2, _free_port(), str(tmp_path), blocks), nprocs=2, join=True)
    w = _case()
    d = w.disc
    O = oracle_for(d)
    O.initialize(w.velocity)
    shape = (d.nz, d.nx * d.ny, w.k)
    Ls = _layouts(w, 2)
    got = [np.load(tmp_path / ("rank%d.npz" % r)) for r in range(2)]
    ref = O.precondition(w.rhs).reshape(shape)
    assert rel(_gather(Ls, [g["M"] for g in got], shape), ref) < 1e-12
    Xo, sto = O.solve(w.rhs, 20, 1e-8)
    assert all(bool(g["conv"]) and int(g["its"]) == sto["iterations"] for g in got)
    assert rel(_gather(Ls, [g["X"] for g in got], shape), Xo.reshape(shape)) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_gpu_thread_ranks_match_one_handle(product_lib, world):
    """Ranks as threads of one process on one GPU, each with a handle that
    factors only its panels (FP64): the pipeline's sweep and solve equal one
    handle's over all panels."""
    import torch
    import psp_b200 as P
    w = _case()
    d = w.disc
    k, nxy = w.k, d.nx * d.ny
    grid = w.rhs.reshape(d.nz, nxy, k)
    H = P.DistHelmholtz(d)
    H.Initialize(w.velocity, precision=P.FP64)
    Mref = H.precondition(w.rhs).reshape(d.nz, nxy, k)
    Xref = w.rhs.copy()
    st_ref = H.Solve(Xref, 20, 1e-8)
    Ls = _layouts(w, world)
    vel = torch.from_numpy(np.ascontiguousarray(w.velocity.reshape(-1))).cuda()

    def rank(r, comm):
        L = Ls[r]
        be = Z.DeviceBackend(d, L, vel, P.FP64)
        S = Z.ZPanelSolver(L, be, comm, k)
        M = Z.scatter_slab(L, grid, k).cuda()
        S.precondition(M)
        X = Z.scatter_slab(L, grid, k).cuda()
        st = S.solve(X, 20, 1e-8)
        info = be.h.memory_info()
        return M[L.own].cpu().numpy(), X[L.own].cpu().numpy(), st, info

    res = _thread_ranks(world, rank)
    shape = Mref.shape
    assert rel(_gather(Ls, [r[0] for r in res], shape), Mref) < 1e-12
    assert all(r[2]["converged"] and r[2]["iterations"] == st_ref["iterations"] for r in res)
    assert rel(_gather(Ls, [r[1] for r in res], shape), Xref.reshape(shape)) < 1e-9
    # each rank holds only its own panels' factors
    assert [r[3]["resident_panels"] for r in res] == [L.p1 - L.p0 for L in Ls]
