"""ORACLE — test infrastructure only (the checker, never the product).

ctypes front-end for ``_ref/libpspref.so``: the reference's own
psp::DistUniformGrid (include/psp/dist_uniform_grid.hpp of the reference,
compiled unchanged against the one-process Elemental/MPI stand-in in
refshim/ by ``make ref``).  Tests use it to check oracle/grid_io.py and the
product's grid kernels against the reference code itself.  ``available()``
is False where the library was not built (the reference tree is only
present where the repository is developed).

Grids are numpy arrays of shape (nz, ny, nx, numScalars) in natural order,
float64 or complex128.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libpspref.so")
REF_TREE = os.environ.get("PSP_REFERENCE_TREE", "/root/reference")
_lib = None


def build():
    """Build _ref/libpspref.so from the reference tree, if it is present."""
    if os.path.exists(os.path.join(REF_TREE, "include", "psp", "dist_uniform_grid.hpp")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", "REF=" + REF_TREE], check=True)


def available():
    return os.path.exists(_LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp, cp, i = ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_int
        L.ref_grid_error.restype = cp
        L.ref_grid_load.argtypes = [cp, i, i, i, i, i, i, dp]
        L.ref_grid_interpolate.argtypes = [dp, i, i, i, i, i, i, i, i, dp]
        L.ref_grid_write_plane.argtypes = [dp, i, i, i, i, i, i, i, cp]
        L.ref_grid_write_volume.argtypes = [dp, i, i, i, i, i, cp]
        _lib = L
    return _lib


def _check(code):
    if code:
        raise RuntimeError(lib().ref_grid_error().decode())


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _in(grid):
    g = np.ascontiguousarray(grid)
    return g, int(np.iscomplexobj(g))


def sequential_load(path, nx, ny, nz, numScalars, order, is_complex=False):
    """DistUniformGrid(nx, ny, nz, comm, numScalars, order).SequentialLoad(path)."""
    out = np.empty((nz, ny, nx, numScalars), dtype=np.complex128 if is_complex else np.float64)
    _check(lib().ref_grid_load(os.fsencode(path), nx, ny, nz, numScalars, order, int(is_complex), _dp(out)))
    return out


def interpolate_to(grid, nx, ny, nz):
    g, c = _in(grid)
    nzO, nyO, nxO, ns = g.shape
    out = np.empty((nz, ny, nx, ns), dtype=g.dtype)
    _check(lib().ref_grid_interpolate(_dp(g), nxO, nyO, nzO, ns, c, nx, ny, nz, _dp(out)))
    return out


def write_plane(grid, plane, which, basename):
    g, c = _in(grid)
    nz, ny, nx, ns = g.shape
    _check(lib().ref_grid_write_plane(_dp(g), nx, ny, nz, ns, c, plane, which, os.fsencode(basename)))


def write_volume(grid, basename):
    g, c = _in(grid)
    nz, ny, nx, ns = g.shape
    _check(lib().ref_grid_write_volume(_dp(g), nx, ny, nz, ns, c, os.fsencode(basename)))


class RefHelmholtz:
    """The reference's own psp::DistHelmholtz<double> on one process, built
    by its constructor (geometry, nested-dissection ordering and elimination
    trees; Clique's symbolic analysis is not reproduced), for the members
    that need no frontal structure: PanelV / PanelDepth / PanelPadding, the
    global row order, the PML stretches and the global rows Initialize
    forms.  ``disc`` is a psp_b200 Discretization."""

    def __init__(self, disc, damping=7.0, planes_per_panel=4, cutoff=12):
        L = lib()
        L.ref_dh_error.restype = ctypes.c_char_p
        self.disc = disc
        bcs = (ctypes.c_int * 5)(disc.frontBC, disc.rightBC, disc.backBC, disc.leftBC, disc.topBC)
        h = ctypes.c_void_p()
        d = ctypes.c_double
        code = L.ref_dh_create(d(disc.omega), disc.nx, disc.ny, disc.nz, d(disc.wx), d(disc.wy), d(disc.wz), bcs,
                               disc.bx, disc.by, disc.bz, d(disc.sigmax), d(disc.sigmay), d(disc.sigmaz), d(damping),
                               planes_per_panel, cutoff, ctypes.byref(h))
        if code:
            raise RuntimeError(L.ref_dh_error().decode())
        self._h = h
        self.N = disc.nx * disc.ny * disc.nz
        self.trees = self._recorded_trees()

    def _recorded_trees(self):
        """The elimination trees the constructor built for Clique's symbolic
        analysis (bottom, leftover inner if any, top): per tree (info, lower)
        with info rows (offset, size, parent, original lower-structure size)
        and lower the list of each node's original lower structure."""
        L = lib()
        out = []
        for t in range(3):
            n, nl = ctypes.c_int(), ctypes.c_int()
            if L.ref_dh_tree(t, ctypes.byref(n), ctypes.byref(nl), None, None):
                break
            info = np.zeros(4 * n.value, dtype=np.int32)
            low = np.zeros(max(nl.value, 1), dtype=np.int32)
            L.ref_dh_tree(t, ctypes.byref(n), ctypes.byref(nl), info.ctypes.data_as(ctypes.c_void_p),
                          low.ctypes.data_as(ctypes.c_void_p))
            info = info.reshape(n.value, 4)
            ends = np.cumsum(info[:, 3])
            out.append((info, [low[e - c:e] for e, c in zip(ends, info[:, 3])]))
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ref_dh_destroy(self._h)
            self._h = None

    def _call(self, fn, *args):
        if fn(self._h, *args):
            raise RuntimeError(lib().ref_dh_error().decode())

    def geometry(self):
        """(num_panels, 3) int array: lowest v, depth, padding per panel."""
        n = ctypes.c_int()
        self._call(lib().ref_dh_geometry, ctypes.byref(n), None)
        out = np.zeros(3 * n.value, dtype=np.int32)
        self._call(lib().ref_dh_geometry, ctypes.byref(n), out.ctypes.data_as(ctypes.c_void_p))
        return out.reshape(n.value, 3)

    def local_to_natural(self):
        out = np.zeros(self.N, dtype=np.int32)
        self._call(lib().ref_dh_local_to_natural, out.ctypes.data_as(ctypes.c_void_p))
        return out

    def rows(self, velocity):
        """(row offsets, complex entries) of the global rows in the
        reference's order for a natural-order velocity."""
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(-1)
        nnz = ctypes.c_int()
        self._call(lib().ref_dh_rows, v.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nnz), None, None)
        ro = np.zeros(self.N + 1, dtype=np.int32)
        ent = np.zeros(nnz.value, dtype=np.complex128)
        self._call(lib().ref_dh_rows, v.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nnz),
                   ro.ctypes.data_as(ctypes.c_void_p), ent.ctypes.data_as(ctypes.c_void_p))
        return ro, ent

    def global_operator_natural(self, velocity):
        """The global operator as a scipy CSR matrix in natural order: row
        entries in FormGlobalRow's order (centre, then the -x, +x, -y, +y,
        -v, +v neighbours that exist; v = nz - 1 - z)."""
        import scipy.sparse as sp
        ro, ent = self.rows(velocity)
        nat = self.local_to_natural()
        nx, ny, nz = self.disc.nx, self.disc.ny, self.disc.nz
        x, y, z = nat % nx, (nat // nx) % ny, nat // (nx * ny)
        v = nz - 1 - z
        steps = [(x > 0, -1), (x + 1 < nx, 1), (y > 0, -nx), (y + 1 < ny, nx), (v > 0, nx * ny),
                 (v + 1 < nz, -nx * ny)]
        cols = np.zeros(ent.size, dtype=np.int64)
        pos = ro[:-1].astype(np.int64).copy()
        cols[pos] = nat
        pos += 1
        for have, step in steps:
            cols[pos[have]] = nat[have] + step
            pos[have] += 1
        if not np.array_equal(pos, ro[1:]):
            raise RuntimeError("row lengths do not match the stencil")
        rows = np.repeat(nat, np.diff(ro))
        return sp.csr_matrix((ent, (rows, cols)), shape=(self.N, self.N))

    def stretch(self, which, idx, v_offset=0):
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        out = np.zeros(idx.size, dtype=np.complex128)
        self._call(lib().ref_dh_stretch, which, idx.size, idx.ctypes.data_as(ctypes.c_void_p), v_offset,
                   out.ctypes.data_as(ctypes.c_void_p))
        return out

    def solve(self, velocity, orc, B, m=20, rel_tol=1e-4):
        """The reference's own Solve (solve.hpp:12-611) of the right-hand
        sides B (natural order, (nz, ny, nx, k) complex128) on a copy, with
        the global rows formed from `velocity` and the panel solves of the
        initialized oracle `orc` in place of Clique's.  Returns (X, log,
        iterations): what the reference printed, and its GMRES step count
        (its "finished iteration" lines plus the converged one)."""
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(-1)
        X = np.ascontiguousarray(B, dtype=np.complex128).copy()
        k = X.size // self.N
        L = lib()
        L.ref_dh_log.restype = ctypes.c_char_p
        code = L.ref_dh_solve(self._h, orc._h, v.ctypes.data_as(ctypes.c_void_p), X.ctypes.data_as(ctypes.c_void_p),
                              k, m, ctypes.c_double(rel_tol))
        log = L.ref_dh_log().decode()
        if code:
            raise RuntimeError(L.ref_dh_error().decode())
        its = log.count("finished iteration") + log.count("converged with relative tolerance")
        return X, log, its

    def panel_front(self, velocity, p, t):
        """Node t of panel p's front as the reference's Initialize fills it
        (GetPanelVelocity, FillPanelFronts): the first s columns, (s+u) x s
        complex128, before any update is added."""
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(-1)
        s, u = ctypes.c_int(), ctypes.c_int()
        self._call(lib().ref_dh_panel_front, v.ctypes.data_as(ctypes.c_void_p), p, t, ctypes.byref(s),
                   ctypes.byref(u), None)
        out = np.zeros((s.value + u.value) * s.value, dtype=np.complex128)
        self._call(lib().ref_dh_panel_front, v.ctypes.data_as(ctypes.c_void_p), p, t, ctypes.byref(s),
                   ctypes.byref(u), out.ctypes.data_as(ctypes.c_void_p))
        return out.reshape(s.value, s.value + u.value).T

    def apply(self, velocity, orc, B, op, panel=0):
        """One of the reference's operators on a copy of B (natural order):
        "multiply" (B := A B), "precondition" (the sweep around the
        oracle's panel solves) or "panel" (SolvePanel of `panel`), each
        between the reference's own pull and push of the right-hand
        sides."""
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(-1)
        X = np.ascontiguousarray(B, dtype=np.complex128).copy()
        k = X.size // self.N
        code = {"multiply": 0, "precondition": 1, "panel": 2}[op]
        self._call(lib().ref_dh_apply, orc._h, v.ctypes.data_as(ctypes.c_void_p),
                   X.ctypes.data_as(ctypes.c_void_p), k, code, panel)
        return X
