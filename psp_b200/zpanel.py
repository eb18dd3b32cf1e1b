"""The z-panel pipeline: one sweeping-preconditioned solve spread over ranks.

The reference distributes every panel over all MPI ranks; on GPUs the panels
themselves are split instead.  Rank r owns a contiguous range of panels
(their factors live only on its GPU: the handle factors panels [p0, p1),
``psp_cu_set_panel_range``) and the grid planes of those panels; its vectors
are slabs of the grid holding those planes plus one halo plane on each side.

* The sweep (Precondition, solve.hpp:681-734) is the reference's block LDL^T
  sweep with its two coupling steps across rank boundaries: the forward
  sweep passes the boundary plane of a rank's last panel to the next rank
  (SubdiagonalUpdate, solve.hpp:884-948: B_{i+1} -= A_{i+1,i} B_i reads that
  plane), the backward sweep passes the boundary plane of a rank's first
  panel back (MultiplySuperdiagonal, solve.hpp:969-1047).  One nx*ny*k plane
  crosses each boundary in each direction per sweep.
* The matvec (Multiply, solve.hpp:613-679) exchanges one halo plane with
  each neighbour and applies the operator to the rank's own planes.
* GMRES (InternalSolveWithGMRES, solve.hpp:241-611) runs on every rank over
  its own planes; norms and inner products are sums over ranks
  (environment.hpp:177-257: the reference's AllReduce of local dots), and
  the small Hessenberg/Givens work is repeated identically on every rank.

Ranks talk through a communicator object (``TorchComm`` over
torch.distributed: NCCL between GPUs, gloo on CPU; ``ThreadComm`` for ranks
that are threads of one process).  The panel solves and matvecs go through a
backend: ``DeviceBackend`` drives the CUDA library through the C ABI; the
tests substitute a CPU stand-in with the same four methods.
"""
import math
import queue
import threading

import numpy as np

# ---------------------------------------------------------------- layout


def partition(costs, world):
    """Contiguous split of the panels (per-panel costs) over `world` ranks
    minimizing the largest load: list of (p0, p1), one per rank."""
    n = len(costs)
    if world < 1 or world > n:
        raise ValueError("need between 1 and %d ranks for %d panels" % (n, n))
    pre = np.concatenate([[0.0], np.cumsum(costs)])
    lo, hi = max(costs), pre[-1]
    # the smallest feasible cap, by bisection on the greedy split
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        parts, start, ok = [], 0, True
        for r in range(world):
            end = start
            while end < n and pre[end + 1] - pre[start] <= mid and n - (end + 1) >= world - r - 1:
                end += 1
            if end == start:
                ok = False
                break
            parts.append((start, end))
            start = end
        ok = ok and start == n
        if ok:
            hi = mid
        else:
            lo = mid
    parts, start = [], 0
    for r in range(world):
        end = start
        while end < n and pre[end + 1] - pre[start] <= hi * (1 + 1e-12) and n - (end + 1) >= world - r - 1:
            end += 1
        parts.append((start, max(end, start + 1)))
        start = parts[-1][1]
    parts[-1] = (parts[-1][0], n)
    return parts


class Layout:
    """Panels, planes and slabs of one rank.  ``geometry`` rows are (lowest
    v, depth, padding, class) per panel with v = nz - 1 - z
    (psp_b200.panel_geometry)."""

    def __init__(self, geometry, nz, nxy, rank, ranges):
        self.geometry = np.asarray(geometry)
        self.nz, self.nxy = nz, nxy
        self.rank, self.world = rank, len(ranges)
        self.ranges = ranges
        self.num_panels = self.geometry.shape[0]
        self.p0, self.p1 = ranges[rank]
        vlo = int(self.geometry[self.p0, 0])
        vhi = int(self.geometry[self.p1 - 1, 0] + self.geometry[self.p1 - 1, 1] - 1)
        # own planes z in [zlo, zhi]; the first panels (low v) sit at high z
        self.zlo, self.zhi = nz - 1 - vhi, nz - 1 - vlo
        self.zs = max(0, self.zlo - 1)             # slab: own planes and one halo plane each side
        self.ze = min(nz, self.zhi + 2)
        self.nplanes = self.ze - self.zs
        self.own = slice(self.zlo - self.zs, self.zhi + 1 - self.zs)  # own planes within the slab
        self.up = self.rank - 1    # neighbour holding the planes above zhi (lower panels)
        self.down = self.rank + 1  # neighbour holding the planes below zlo (higher panels)

    def has_up(self):
        return self.rank > 0

    def has_down(self):
        return self.rank < self.world - 1


def panel_costs(disc, planes_per_panel=4, cutoff=12):
    """Predicted factorization cost of every panel (flops of its class)."""
    from . import analyze_class, panel_geometry
    geo = panel_geometry(disc, planes_per_panel)
    cls_cost = {}
    for c in sorted(set(int(x) for x in geo[:, 3])):
        info, _ = analyze_class(disc, planes_per_panel, cutoff, c)
        s, u = info[:, 1].astype(float), info[:, 2].astype(float)
        cls_cost[c] = float((s ** 3 / 3 + s ** 2 * u + s ** 3 / 6 + s ** 2 * u / 2 + s * u ** 2 / 2).sum())
    return geo, [cls_cost[int(c)] for c in geo[:, 3]]


# ---------------------------------------------------------------- communicators


class TorchComm:
    """torch.distributed point-to-point and all-reduce (NCCL or gloo)."""

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        self.cpu = dist.get_backend() != "nccl"

    def _t(self, x):
        return x.cpu() if self.cpu and x.is_cuda else x

    def send(self, x, dst):
        self.dist.send(self._t(x.contiguous()), dst)

    def recv(self, x, src):
        buf = self._t(x) if self.cpu else x
        if not buf.is_contiguous():
            buf = buf.contiguous()
        self.dist.recv(buf, src)
        if buf is not x:
            x.copy_(buf)

    def allreduce_sum(self, x):
        buf = self._t(x).contiguous()
        self.dist.all_reduce(buf)
        if buf is not x:
            x.copy_(buf)
        return x


class ThreadComm:
    """Ranks that are threads of one process (tests; a GPU may host several
    such ranks because they only wait for each other on the host)."""

    class _Shared:
        def __init__(self, size):
            self.size = size
            self.boxes = {(a, b): queue.Queue() for a in range(size) for b in range(size)}
            self.barrier = threading.Barrier(size)
            self.lock = threading.Lock()
            self.acc = None

    @classmethod
    def group(cls, size):
        sh = cls._Shared(size)
        return [cls(sh, r) for r in range(size)]

    def __init__(self, shared, rank):
        self.sh, self.rank, self.size = shared, rank, shared.size

    def send(self, x, dst):
        self.sh.boxes[(self.rank, dst)].put(x.clone())

    def recv(self, x, src):
        x.copy_(self.sh.boxes[(src, self.rank)].get(timeout=120))

    def allreduce_sum(self, x):
        # every rank adds its part in rank order (a deterministic sum)
        parts = self._gather(x.clone())
        total = parts[0].clone()
        for p in parts[1:]:
            total += p.to(total.device)
        x.copy_(total)
        return x

    def _gather(self, x):
        sh = self.sh
        with sh.lock:
            if sh.acc is None:
                sh.acc = [None] * sh.size
            sh.acc[self.rank] = x
        sh.barrier.wait(timeout=120)
        parts = list(sh.acc)
        sh.barrier.wait(timeout=120)
        with sh.lock:
            sh.acc = None
        sh.barrier.wait(timeout=120)
        return parts


# ---------------------------------------------------------------- backend


class DeviceBackend:
    """The CUDA library through the C ABI: a handle that factors only the
    rank's panels."""

    def __init__(self, disc, layout, velocity, precision, device=0, damping=7.0, planes_per_panel=4, cutoff=12):
        from . import DistHelmholtz
        self.h = DistHelmholtz(disc, damping, planes_per_panel, cutoff, device)
        self.h.set_panel_range(layout.p0, layout.p1)
        self.h.Initialize(velocity, precision=precision)

    def solve_panel(self, W, k, p, in_mode, out_acc, zs):
        self.h.solve_panel_slab(W, k, p, in_mode, out_acc, zs)

    def multiply(self, X, Y, k, z_first, z_count, zs, Bv=None):
        self.h.multiply_slab(X, Y, k, z_first, z_count, zs, Bv)


# ---------------------------------------------------------------- solver


class ZPanelSolver:
    """One rank of the pipeline.  Vectors are tensors of shape
    (layout.nplanes, nxy, k) complex128 (slab with halos).

    ``blocks`` > 1 pipelines the sweep over that many blocks of
    right-hand-side columns: a rank hands a block's boundary plane on and
    starts the next block while the neighbouring rank works on the one it
    received, so with R ranks a sweep takes about R + blocks - 1 block
    steps instead of R full ones.  Every column's arithmetic is unchanged
    (the sweep treats columns independently); each block is solved on its
    own contiguous copy of the slab."""

    def __init__(self, layout, backend, comm, k, blocks=1):
        self.L, self.be, self.comm, self.k = layout, backend, comm, k
        self.blocks = max(1, min(int(blocks), k))

    def new(self, like):
        import torch
        return torch.zeros((self.L.nplanes, self.L.nxy, self.k), dtype=torch.complex128, device=like.device)

    def _plane(self, z):
        return z - self.L.zs

    # -- sweep
    def _forward(self, W, k):
        L = self.L
        if L.has_up():  # plane below the first panel in v: the previous rank's last panel
            self.comm.recv(W[self._plane(L.zhi + 1)], L.up)
        for p in range(L.p0, L.p1):
            self.be.solve_panel(W, k, p, 0 if p == 0 else 1, 0, L.zs)
        if L.has_down():
            self.comm.send(W[self._plane(L.zlo)], L.down)

    def _backward(self, W, k):
        # every panel but the top one, from the top down
        L = self.L
        if L.has_down():
            self.comm.recv(W[self._plane(L.zlo - 1)], L.down)
        for p in range(min(L.p1, L.num_panels - 1) - 1, L.p0 - 1, -1):
            self.be.solve_panel(W, k, p, 2, 1, L.zs)
        if L.has_up():
            self.comm.send(W[self._plane(L.zhi)], L.up)

    def column_blocks(self):
        """(first, end) column ranges of the sweep's blocks."""
        nb, k = self.blocks, self.k
        edges = [k * i // nb for i in range(nb + 1)]
        return [(edges[i], edges[i + 1]) for i in range(nb)]

    def precondition(self, W):
        """W := M^{-1} W on the own planes (halo planes are overwritten)."""
        if self.blocks == 1:
            self._forward(W, self.k)
            self._backward(W, self.k)
            return W
        parts = [(c0, c1, W[..., c0:c1].contiguous()) for c0, c1 in self.column_blocks()]
        # every rank takes the blocks in the same order in each direction,
        # so each message meets the receive posted for it
        for c0, c1, Wb in parts:
            self._forward(Wb, c1 - c0)
        for c0, c1, Wb in parts:
            self._backward(Wb, c1 - c0)
        for c0, c1, Wb in parts:
            W[..., c0:c1] = Wb
        return W

    # -- matvec
    def exchange_halo(self, X):
        L = self.L
        # send up first, then down; receive in the matching order (no cycle)
        if L.has_up():
            self.comm.send(X[self._plane(L.zhi)], L.up)
        if L.has_down():
            self.comm.recv(X[self._plane(L.zlo - 1)], L.down)
        if L.has_down():
            self.comm.send(X[self._plane(L.zlo)], L.down)
        if L.has_up():
            self.comm.recv(X[self._plane(L.zhi + 1)], L.up)

    def multiply(self, X, Y, Bv=None):
        """Y := A X (or Bv - A X) on the own planes."""
        self.exchange_halo(X)
        L = self.L
        self.be.multiply(X, Y, self.k, L.zlo, L.zhi + 1 - L.zlo, L.zs, Bv)

    # -- reductions over the own planes of every rank
    def norms(self, X):
        import torch
        v = X[self.L.own]
        out = (v.real.square() + v.imag.square()).sum(dim=(0, 1))
        return torch.sqrt(self.comm.allreduce_sum(out))

    def dots(self, V, W):
        """conj(V) . W per right-hand side, summed over ranks."""
        out = (V[self.L.own].conj() * W[self.L.own]).sum(dim=(0, 1))
        return self.comm.allreduce_sum(out)

    # -- GMRES
    def solve(self, B, m=20, rel_tol=1e-4, max_iterations=0):
        """Left-preconditioned GMRES(m) on the own planes of slab B (in
        place): the reference's InternalSolveWithGMRES (solve.hpp:241-611)
        with x and the true residual recomputed every inner step and all
        right-hand sides iterating until the slowest converges.  Returns
        a stats dict."""
        import torch
        k, own = self.k, self.L.own
        b = B.clone()
        x = torch.zeros_like(B)
        w = b.clone()
        orig = self.norms(w).cpu().numpy()
        if np.isnan(orig).any():
            raise RuntimeError("Original residual norms had a NaN")
        it, converged, max_rel = 0, False, 0.0
        V = [None] * m
        while not converged:
            x0 = x.clone()
            self.precondition(w)
            beta = self.norms(w)
            V[0] = w / beta
            z = np.zeros((k, m + 1), dtype=np.complex128)
            z[:, 0] = beta.cpu().numpy()
            H = np.zeros((k, m, m), dtype=np.complex128)  # H[r][row][col]
            cs = np.zeros((k, m))
            sn = np.zeros((k, m), dtype=np.complex128)
            y = np.zeros((k, m), dtype=np.complex128)
            for j in range(m):
                w = self.new(B)
                self.multiply(V[j], w)
                self.precondition(w)
                for i in range(j + 1):
                    h = self.dots(V[i], w)
                    w -= h * V[i]
                    H[:, i, j] = h.cpu().numpy()
                delta = self.norms(w)
                dn = delta.cpu().numpy()
                if np.isnan(dn).any():
                    raise RuntimeError("delta list had a NaN")
                if (dn == 0).any():  # lucky breakdown: B keeps the right-hand sides (solve.hpp:405-414)
                    return dict(iterations=it, converged=False, lucky_breakdown=True, final_max_rel_resid=max_rel)
                if j + 1 < m:
                    V[j + 1] = w / delta
                for r in range(k):
                    for i in range(j):
                        a, bb = H[r, i, j], H[r, i + 1, j]
                        H[r, i, j] = cs[r, i] * a + sn[r, i] * bb
                        H[r, i + 1, j] = -np.conj(sn[r, i]) * a + cs[r, i] * bb
                    c, s, rho = _givens(H[r, j, j], dn[r])
                    H[r, j, j], cs[r, j], sn[r, j] = rho, c, s
                    zj, zj1 = z[r, j], z[r, j + 1]
                    z[r, j], z[r, j + 1] = c * zj + s * zj1, -np.conj(s) * zj + c * zj1
                    for i in range(j, -1, -1):
                        acc = z[r, i] - sum(H[r, i, q] * y[r, q] for q in range(i + 1, j + 1))
                        y[r, i] = acc / H[r, i, i]
                yt = torch.from_numpy(y[:, :j + 1].T.copy()).to(B.device)  # (j+1, k)
                x = x0.clone()
                for i in range(j + 1):
                    x += yt[i] * V[i]
                w = self.new(B)
                self.multiply(x, w, b)
                resid = self.norms(w).cpu().numpy()
                max_rel = float(np.max(resid / orig))
                if max_rel < rel_tol:
                    converged = True
                    it += 1
                    break
                it += 1
                if max_iterations and it >= max_iterations:
                    break
            if max_iterations and it >= max_iterations:
                break
        B[own] = x[own]
        return dict(iterations=it, converged=converged, lucky_breakdown=False, final_max_rel_resid=max_rel)


def _givens(f, g):
    """lapack::ComputeGivens (solve.hpp:486-487): [c s; -conj(s) c][f; g] =
    [rho; 0] with c real."""
    af, ag = abs(f), abs(g)
    if ag == 0:
        return 1.0, 0j, f
    if af == 0:
        return 0.0, np.conj(g) / ag, ag + 0j
    nrm = math.hypot(af, ag)
    return af / nrm, (f / af) * np.conj(g) / nrm, (f / af) * nrm


def scatter_slab(layout, grid, k, like=None):
    """A copy of the rank's slab (with halos) of a natural-order (nz, nxy, k)
    grid, as a CPU tensor or on the device of `like`."""
    import torch
    t = torch.from_numpy(np.array(grid.reshape(layout.nz, layout.nxy, k)[layout.zs:layout.ze], copy=True))
    return t.to(like.device) if like is not None else t


def own_planes(layout, slab):
    """(z range, own planes of the slab)."""
    return (layout.zlo, layout.zhi + 1), slab[layout.own]
