"""ORACLE — test infrastructure only (the checker, never the product).

ctypes front-end for ``liboracle.so``, the FP64 CPU restatement of PSP's
sweeping-preconditioned Helmholtz solve built from ``psp_oracle.cpp``.
Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module.

Grids are numpy arrays in natural order (x fastest, then y, then z), complex
grids carry the ``k`` right-hand sides interleaved per point, i.e. shape
``(nz, ny, nx, k)`` -- the layout of a one-process ``DistUniformGrid`` with
``numScalars = k`` (dist_uniform_grid.hpp:292-342).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

PML, DIRICHLET = 0, 1


class _Disc(ctypes.Structure):
    _fields_ = [
        ("omega", ctypes.c_double),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("wx", ctypes.c_double), ("wy", ctypes.c_double), ("wz", ctypes.c_double),
        ("frontBC", ctypes.c_int), ("rightBC", ctypes.c_int), ("backBC", ctypes.c_int),
        ("leftBC", ctypes.c_int), ("topBC", ctypes.c_int),
        ("bx", ctypes.c_int), ("by", ctypes.c_int), ("bz", ctypes.c_int),
        ("sigmax", ctypes.c_double), ("sigmay", ctypes.c_double), ("sigmaz", ctypes.c_double),
    ]


class _Stats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int), ("converged", ctypes.c_int),
        ("lucky_breakdown", ctypes.c_int), ("final_max_rel_resid", ctypes.c_double),
        ("setup_seconds", ctypes.c_double), ("solve_seconds", ctypes.c_double),
    ]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.oracle_create.argtypes = [ctypes.POINTER(_Disc), ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_void_p)]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_geometry.argtypes = [vp, ip, ip]
        L.oracle_nd_to_natural.argtypes = [vp, ip]
        L.oracle_tree.argtypes = [vp, ctypes.c_int, ip, ip]
        L.oracle_initialize.argtypes = [vp, dp]
        L.oracle_global_operator.argtypes = [vp, ip, ip, ip, dp]
        L.oracle_multiply.argtypes = [vp, dp, ctypes.c_int]
        L.oracle_precondition.argtypes = [vp, dp, ctypes.c_int]
        L.oracle_solve_panel.argtypes = [vp, dp, ctypes.c_int, ctypes.c_int]
        L.oracle_solve.argtypes = [vp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.POINTER(_Stats), dp, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a, ctype=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def make_disc(omega, nx, ny, nz, wx, wy, wz, bcs=(PML,) * 5, pml=(5, 5, 5), sigma=None):
    """Discretization<R> (discretization.hpp:36-110). ``sigma=None`` uses
    the reference default 1.2*max width (discretization.hpp:59-62)."""
    d = _Disc()
    d.omega = omega
    d.nx, d.ny, d.nz = nx, ny, nz
    d.wx, d.wy, d.wz = wx, wy, wz
    d.frontBC, d.rightBC, d.backBC, d.leftBC, d.topBC = bcs
    d.bx, d.by, d.bz = pml
    s = 1.2 * max(wx, wy, wz) if sigma is None else sigma
    d.sigmax = d.sigmay = d.sigmaz = s
    return d


class Oracle:
    """FP64 CPU DistHelmholtz restatement (one process)."""

    def __init__(self, disc, damping=7.0, planes_per_panel=4, cutoff=12):
        self.disc = disc
        h = ctypes.c_void_p()
        if lib().oracle_create(ctypes.byref(disc), damping, planes_per_panel, cutoff, ctypes.byref(h)):
            raise ValueError(lib().oracle_last_error().decode())
        self._h = h
        self.shape = (disc.nz, disc.ny, disc.nx)
        self.N = disc.nx * disc.ny * disc.nz

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def geometry(self):
        n = ctypes.c_int()
        lib().oracle_geometry(self._h, ctypes.byref(n), None)
        info = np.zeros(4 * n.value, dtype=np.int32)
        lib().oracle_geometry(self._h, ctypes.byref(n), _ptr(info, ctypes.c_int))
        return info.reshape(n.value, 4)  # (vLow, depth, padding, class)

    def stretch(self, which, idx, v_offset=0):
        """PML stretch `which` (1 s1Inv, 2 s2Inv, 3 s3Inv, 4 s3InvArtificial
        with v_offset) at the indices idx, complex128."""
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        out = np.zeros(idx.size, dtype=np.complex128)
        lib().oracle_stretch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                         ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        lib().oracle_stretch(self._h, which, idx.size, _ptr(idx, ctypes.c_int), v_offset, _ptr(out.view(np.float64)))
        return out

    def panel_front(self, velocity, p, t):
        """Node t of panel p: the first s columns of its front, (s+u) x s
        complex128, as assembled from the velocity before any update."""
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(-1)
        L = lib()
        L.oracle_panel_front.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_double)]
        s, u = ctypes.c_int(), ctypes.c_int()
        if L.oracle_panel_front(self._h, _ptr(v), p, t, ctypes.byref(s), ctypes.byref(u), None):
            raise ValueError("no such panel or node")
        out = np.zeros(((s.value + u.value) * s.value), dtype=np.complex128)
        L.oracle_panel_front(self._h, _ptr(v), p, t, ctypes.byref(s), ctypes.byref(u), _ptr(out.view(np.float64)))
        return out.reshape(s.value, s.value + u.value).T

    def nd_to_natural(self):
        out = np.zeros(self.N, dtype=np.int32)
        lib().oracle_nd_to_natural(self._h, _ptr(out, ctypes.c_int))
        return out

    def tree(self, cls):
        n = ctypes.c_int()
        lib().oracle_tree(self._h, cls, ctypes.byref(n), None)
        info = np.zeros(4 * n.value, dtype=np.int32)
        lib().oracle_tree(self._h, cls, ctypes.byref(n), _ptr(info, ctypes.c_int))
        return info.reshape(n.value, 4)  # (off, size, lowerSize, parent)

    def initialize(self, velocity):
        v = np.ascontiguousarray(velocity, dtype=np.float64)
        assert v.size == self.N
        if lib().oracle_initialize(self._h, _ptr(v)):
            raise RuntimeError(lib().oracle_last_error().decode())

    def form_operator(self, velocity):
        """Forms the global operator only (no panel factorization)."""
        v = np.ascontiguousarray(velocity, dtype=np.float64)
        lib().oracle_form_operator.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        lib().oracle_form_operator(self._h, _ptr(v))

    def global_operator_natural(self):
        """The global operator as a scipy CSR matrix in natural ordering."""
        import scipy.sparse as sp
        nnz = ctypes.c_int()
        lib().oracle_global_operator(self._h, ctypes.byref(nnz), None, None, None)
        rp = np.zeros(self.N + 1, dtype=np.int32)
        cols = np.zeros(nnz.value, dtype=np.int32)
        vals = np.zeros(2 * nnz.value, dtype=np.float64)
        lib().oracle_global_operator(self._h, ctypes.byref(nnz), _ptr(rp, ctypes.c_int),
                                     _ptr(cols, ctypes.c_int), _ptr(vals))
        A_nd = sp.csr_matrix((vals.view(np.complex128), cols, rp), shape=(self.N, self.N))
        perm = self.nd_to_natural()
        P = sp.csr_matrix((np.ones(self.N), (perm, np.arange(self.N))), shape=(self.N, self.N))
        return (P @ A_nd @ P.T).tocsr()

    def _grid_call(self, fn, B, *extra):
        X = np.ascontiguousarray(B, dtype=np.complex128).copy()
        k = X.size // self.N
        if fn(self._h, _ptr(X.view(np.float64)), k, *extra):
            raise RuntimeError(lib().oracle_last_error().decode())
        return X

    def multiply(self, B):
        return self._grid_call(lib().oracle_multiply, B)

    def precondition(self, B):
        return self._grid_call(lib().oracle_precondition, B)

    def solve_panel(self, B, p):
        return self._grid_call(lib().oracle_solve_panel, B, p)

    def solve(self, B, m=20, rel_tol=1e-4, max_its=0, history=64):
        """Returns (X, stats dict)."""
        X = np.ascontiguousarray(B, dtype=np.complex128).copy()
        k = X.size // self.N
        st = _Stats()
        hist = np.zeros(max(history, 1), dtype=np.float64)
        if lib().oracle_solve(self._h, _ptr(X.view(np.float64)), k, m, rel_tol, max_its,
                              ctypes.byref(st), _ptr(hist), history):
            raise RuntimeError(lib().oracle_last_error().decode())
        stats = dict(iterations=st.iterations, converged=bool(st.converged),
                     lucky_breakdown=bool(st.lucky_breakdown),
                     final_max_rel_resid=st.final_max_rel_resid,
                     history=hist[:min(st.iterations, history)].copy())
        return X, stats


def first_cycle_hessenberg(orc):
    """The unrotated Hessenberg matrices of the first GMRES restart cycle of
    the last ``orc.solve`` (the reference's HListCopy, solve.hpp:257-261,
    391-395, 422-426): complex array (k, count, count), whose eigenvalues
    are the Ritz values solve.hpp:589-608 prints."""
    L = lib()
    ip = ctypes.POINTER(ctypes.c_int)
    L.oracle_first_cycle_hessenberg.argtypes = [ctypes.c_void_p, ip, ip, ip, ctypes.POINTER(ctypes.c_double)]
    count, m, k = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.oracle_first_cycle_hessenberg(orc._h, ctypes.byref(count), ctypes.byref(m), ctypes.byref(k), None)
    H = np.zeros((k.value, m.value, m.value), dtype=np.complex128)  # [r][col][row]
    L.oracle_first_cycle_hessenberg(orc._h, ctypes.byref(count), ctypes.byref(m), ctypes.byref(k),
                                    _ptr(H.view(np.float64)))
    c = count.value
    return np.ascontiguousarray(H.transpose(0, 2, 1)[:, :c, :c])


def sample_costs(orc, velocity, k, reps=2):
    """Bounded timing sample of one workload (see oracle_sample in
    psp_oracle.cpp): dict of seconds per unit of work."""
    L = lib()
    L.oracle_sample.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_double)]
    v = np.ascontiguousarray(velocity, dtype=np.float64)
    out = np.zeros(8)
    if L.oracle_sample(orc._h, _ptr(v), k, reps, _ptr(out)):
        raise RuntimeError(L.oracle_last_error().decode())
    return dict(operator=out[0], factor=[out[1], out[2], out[3]], panel_solve=[out[4], out[5], out[6]],
                matvec=out[7])


def modeled_rhs_per_s(orc, costs, k, iterations, restarts=1):
    """Setup+solve and solve-only RHS/s of the oracle extrapolated from a
    bounded sample: panels are factored one after another (threads inside
    the fronts), each GMRES inner step costs one sweep (2P-1 panel solves)
    and two matvecs, every restart one extra sweep."""
    geo = orc.geometry()
    P = geo.shape[0]
    setup = costs["operator"] + sum(costs["factor"][c] for c in geo[:, 3])
    sweep = sum((1 if p == P - 1 else 2) * costs["panel_solve"][geo[p, 3]] for p in range(P))
    solve = (iterations + restarts) * sweep + 2 * iterations * costs["matvec"]
    return dict(setup_seconds=setup, solve_seconds=solve, sweep_seconds=sweep,
                rhs_per_s=k / (setup + solve), solve_only_rhs_per_s=k / solve)


def time_factor_panel(orc, velocity, p):
    """Seconds of one panel factorization (panel p's fronts are kept)."""
    L = lib()
    L.oracle_time_factor_panel.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double)]
    v = np.ascontiguousarray(velocity, dtype=np.float64)
    t = ctypes.c_double()
    if L.oracle_time_factor_panel(orc._h, _ptr(v), p, ctypes.byref(t)):
        raise RuntimeError(L.oracle_last_error().decode())
    return t.value


def time_panel_solve(orc, p, k):
    """Seconds of one panel solve of k right-hand sides (unit-diagonal zero
    fronts of the panel's structure stand in when it holds no factors)."""
    L = lib()
    L.oracle_time_panel_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    t = ctypes.c_double()
    if L.oracle_time_panel_solve(orc._h, p, k, ctypes.byref(t)):
        raise RuntimeError(L.oracle_last_error().decode())
    return t.value


def release_panel(orc, p):
    lib().oracle_release_panel.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib().oracle_release_panel(orc._h, p)


def time_multiply(orc, k):
    """Seconds of one global matvec of k right-hand sides."""
    L = lib()
    L.oracle_time_multiply.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    t = ctypes.c_double()
    if L.oracle_time_multiply(orc._h, k, ctypes.byref(t)):
        raise RuntimeError(L.oracle_last_error().decode())
    return t.value


def num_threads():
    lib().oracle_num_threads.restype = ctypes.c_int
    return lib().oracle_num_threads()
