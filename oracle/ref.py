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
