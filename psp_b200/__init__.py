"""psp_b200 — B200-native drop-in for PSP's sweeping-preconditioned Helmholtz solve.

Python mirror of the reference's C++ surface over the C ABI of
``libpsp_b200.so`` (include/psp_b200.h):

* :class:`Discretization` — ``psp::Discretization<R>`` (discretization.hpp:36-110)
* :class:`DistUniformGrid` — ``psp::DistUniformGrid<F>`` for one process
  (dist_uniform_grid.hpp:48-145), natural order with ``numScalars`` entries
  interleaved per point
* :class:`DistHelmholtz` — ``psp::DistHelmholtz<R>`` (dist_helmholtz.hpp:21-287):
  ``Initialize(velocity, panelScheme)``, ``Solve(B, m, relTol)`` (alias
  ``SolveWithGMRES``) and ``Finalize()``

The compute path is the CUDA library; there is no CPU fallback: importing
works without a GPU, but every compute call fails loudly when the library or
the device is missing.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpsp_b200.so")

PML, DIRICHLET = 0, 1
CLIQUE_LDL_1D, CLIQUE_LDL_SELINV_1D = 0, 1
FP64, MIXED = 0, 1
XYZ, XZY, YXZ, YZX, ZXY, ZYX = range(6)
XY, XZ, YZ = range(3)  # PlaneType (dist_uniform_grid.hpp:24-28)

_STATUS = {0: "ok", 1: "logic error", 2: "runtime error", 3: "CUDA error", 4: "out of memory",
           5: "not initialized", 6: "no CUDA device"}


class LogicError(ValueError):
    """``std::logic_error`` of the reference (bad arguments, shallow domain, ...)."""


class PspRuntimeError(RuntimeError):
    """``std::runtime_error`` of the reference (NaN in GMRES, zero pivot, ...)."""


class CudaError(RuntimeError):
    """A CUDA failure (including out-of-memory and no device)."""


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
        ("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("lucky_breakdown", ctypes.c_int),
        ("final_max_rel_resid", ctypes.c_double), ("solve_seconds", ctypes.c_double),
        ("precondition_seconds", ctypes.c_double), ("matvec_seconds", ctypes.c_double),
        ("arnoldi_seconds", ctypes.c_double), ("num_preconditions", ctypes.c_int),
    ]


C_ABI_SYMBOLS = [
    "psp_cu_last_error", "psp_cu_create", "psp_cu_destroy", "psp_cu_initialize", "psp_cu_initialize_device",
    "psp_cu_solve", "psp_cu_solve_device", "psp_cu_finalize", "psp_cu_multiply", "psp_cu_precondition",
    "psp_cu_multiply_device", "psp_cu_precondition_device", "psp_cu_solve_panel", "psp_cu_set_max_iterations",
    "psp_cu_geometry", "psp_cu_setup_info", "psp_cu_analyze_class", "psp_cu_get_stream",
    "psp_cu_set_profiling", "psp_cu_profile_reset", "psp_cu_profile_get", "psp_cu_sweep_cost",
    "psp_cu_multiply_device_noalloc", "psp_cu_gradient_device", "psp_cu_initialize_batch", "psp_cu_solve_batch",
    "psp_cu_grid_load", "psp_cu_grid_interpolate", "psp_cu_grid_write_plane", "psp_cu_grid_write_volume",
    "psp_cu_set_view_iterates", "psp_cu_set_ritz_values", "psp_cu_get_ritz_values", "psp_cu_hessenberg_eigenvalues",
    "psp_cu_memory_info", "psp_cu_solve_block_width", "psp_cu_plan_block_width",
    "psp_cu_set_panel_range", "psp_cu_solve_panel_slab", "psp_cu_multiply_slab", "psp_cu_panel_geometry",
]

PROFILE_CATEGORIES = ["factor_gemm", "solve_gemm", "ldl_diag", "ldl_trsm", "assemble", "extend_add",
                      "gather_scatter", "stencil", "gmres_vector", "sweep"]

_lib = None


def lib():
    """The loaded C ABI library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libpsp_b200.so is missing: run `python -m psp_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.psp_cu_last_error.restype = ctypes.c_char_p
        L.psp_cu_create.argtypes = [ctypes.POINTER(_Disc), ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.POINTER(vp)]
        L.psp_cu_destroy.argtypes = [vp]
        L.psp_cu_destroy.restype = None
        L.psp_cu_initialize.argtypes = [vp, dp, ctypes.c_int, ctypes.c_int]
        L.psp_cu_initialize_device.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int]
        L.psp_cu_solve.argtypes = [vp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(_Stats)]
        L.psp_cu_solve_device.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.POINTER(_Stats)]
        L.psp_cu_finalize.argtypes = [vp]
        L.psp_cu_multiply.argtypes = [vp, dp, ctypes.c_int]
        L.psp_cu_precondition.argtypes = [vp, dp, ctypes.c_int]
        L.psp_cu_multiply_device.argtypes = [vp, vp, ctypes.c_int]
        L.psp_cu_precondition_device.argtypes = [vp, vp, ctypes.c_int]
        L.psp_cu_solve_panel.argtypes = [vp, dp, ctypes.c_int, ctypes.c_int]
        L.psp_cu_set_max_iterations.argtypes = [vp, ctypes.c_int]
        L.psp_cu_geometry.argtypes = [vp, ip, ip]
        L.psp_cu_setup_info.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_longlong)]
        L.psp_cu_analyze_class.argtypes = [ctypes.POINTER(_Disc), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ip, ip, ip, ip]
        L.psp_cu_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.psp_cu_set_profiling.argtypes = [vp, ctypes.c_int]
        L.psp_cu_profile_reset.argtypes = [vp]
        L.psp_cu_profile_get.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), dp, dp, dp]
        L.psp_cu_sweep_cost.argtypes = [vp, ctypes.c_int, dp, dp]
        L.psp_cu_multiply_device_noalloc.argtypes = [vp, vp, ctypes.c_int]
        L.psp_cu_gradient_device.argtypes = [vp, vp, vp, ctypes.c_int, vp, ctypes.c_int]
        L.psp_cu_initialize_batch.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(dp), ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ip]
        L.psp_cu_solve_batch.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(dp), ip, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.POINTER(_Stats), ip]
        ci = ctypes.c_int
        L.psp_cu_grid_load.argtypes = [ctypes.c_char_p, ci, ci, ci, ci, ci, ci, vp]
        L.psp_cu_grid_interpolate.argtypes = [vp, ci, ci, ci, ci, ci, vp, ci, ci, ci]
        L.psp_cu_grid_write_plane.argtypes = [dp, ci, ci, ci, ci, ci, ci, ci, ctypes.c_char_p]
        L.psp_cu_grid_write_volume.argtypes = [dp, ci, ci, ci, ci, ci, ctypes.c_char_p]
        L.psp_cu_set_view_iterates.argtypes = [vp, ctypes.c_char_p]
        L.psp_cu_set_ritz_values.argtypes = [vp, ci]
        L.psp_cu_get_ritz_values.argtypes = [vp, ip, ip, dp]
        L.psp_cu_hessenberg_eigenvalues.argtypes = [ci, dp, ci, dp]
        L.psp_cu_solve_block_width.argtypes = [vp, ci, ci, ip]
        L.psp_cu_plan_block_width.argtypes = [ci, ctypes.c_double, ctypes.c_double, ci, ip]
        L.psp_cu_set_panel_range.argtypes = [vp, ci, ci]
        L.psp_cu_panel_geometry.argtypes = [ctypes.POINTER(_Disc), ci, ip, ip]
        L.psp_cu_solve_panel_slab.argtypes = [vp, vp, ci, ci, ci, ci, ci]
        L.psp_cu_multiply_slab.argtypes = [vp, vp, vp, vp, ci, ci, ci, ci]
        L.psp_cu_memory_info.argtypes = [vp, ip, ip, ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong)]
        _lib = L
    return _lib


def _check(code):
    if code == 0:
        return
    msg = lib().psp_cu_last_error().decode()
    if code == 1:
        raise LogicError(msg)
    if code in (2, 5):
        raise PspRuntimeError(msg)
    raise CudaError("%s: %s" % (_STATUS.get(code, code), msg))


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Discretization:
    """``psp::Discretization<R>`` (discretization.hpp:36-110).

    Mirrors the four constructors: ``Discretization(omega, nx, ny, nz, wx, wy, wz)``
    plus optional boundary conditions ``bcs=(front, right, back, left, top)``
    and either ``pml=(bx, by, bz)`` (sigma = 1.2*max width) or
    ``pml=size, sigma=value``.  Widths are those of the PML-padded box.
    """

    def __init__(self, omega, nx, ny, nz, wx, wy, wz, bcs=(PML,) * 5, pml=(5, 5, 5), sigma=None):
        self.omega = float(omega)
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.wx, self.wy, self.wz = float(wx), float(wy), float(wz)
        self.frontBC, self.rightBC, self.backBC, self.leftBC, self.topBC = bcs
        if np.isscalar(pml):
            pml = (pml, pml, pml)
        self.bx, self.by, self.bz = (int(v) for v in pml)
        s = 1.2 * max(self.wx, self.wy, self.wz) if sigma is None else float(sigma)
        self.sigmax = self.sigmay = self.sigmaz = s

    def _c(self):
        d = _Disc()
        for name, _ in _Disc._fields_:
            setattr(d, name, getattr(self, name))
        return d


class DistUniformGrid:
    """``psp::DistUniformGrid<F>`` on one process (dist_uniform_grid.hpp:48-145).

    ``data`` has shape (nz, ny, nx, numScalars) in XYZ order -- exactly the
    reference's local buffer with px = py = pz = 1.  Other storage orders are
    accepted by :meth:`from_order` and converted to XYZ.
    """

    def __init__(self, nx, ny, nz, numScalars=1, dtype=np.complex128, data=None):
        self.nx, self.ny, self.nz, self.numScalars = nx, ny, nz, numScalars
        if data is None:
            data = np.zeros((nz, ny, nx, numScalars), dtype=dtype)
        self.data = np.ascontiguousarray(np.asarray(data, dtype=dtype).reshape(nz, ny, nx, numScalars))

    def XSize(self): return self.nx
    def YSize(self): return self.ny
    def ZSize(self): return self.nz
    def NumScalars(self): return self.numScalars
    def XShift(self): return 0
    def YShift(self): return 0
    def ZShift(self): return 0
    def XStride(self): return 1
    def YStride(self): return 1
    def ZStride(self): return 1
    def XLocalSize(self): return self.nx
    def YLocalSize(self): return self.ny
    def ZLocalSize(self): return self.nz
    def OwningProcess(self, *args): return 0

    def NaturalIndex(self, x, y, z):
        return x + y * self.nx + z * self.nx * self.ny

    def LocalIndex(self, x, y, z):
        """Offset of point (x, y, z) in the flat buffer (dist_uniform_grid.hpp:316-342)."""
        return self.NaturalIndex(x, y, z) * self.numScalars

    def Buffer(self):
        return self.data.reshape(-1)

    @classmethod
    def from_order(cls, buf, nx, ny, nz, numScalars, order, dtype=np.complex128):
        """Build an XYZ grid from a flat buffer stored in one of the six
        GridDataOrder layouts (dist_uniform_grid.hpp:316-339)."""
        a = np.asarray(buf, dtype=dtype).reshape(-1, numScalars)
        dims = {XYZ: (nz, ny, nx), XZY: (ny, nz, nx), YXZ: (nz, nx, ny), YZX: (nx, nz, ny),
                ZXY: (ny, nx, nz), ZYX: (nx, ny, nz)}[order]
        # transpose taking the stored (slowest..fastest) axes to (z, y, x)
        perm = {XYZ: (0, 1, 2), XZY: (1, 0, 2), YXZ: (0, 2, 1), YZX: (1, 2, 0),
                ZXY: (2, 0, 1), ZYX: (2, 1, 0)}[order]
        v = np.transpose(a.reshape(*dims, numScalars), perm + (3,))
        return cls(nx, ny, nz, numScalars, dtype, v)

    def _is_complex(self):
        return np.iscomplexobj(self.data)

    def SequentialLoad(self, filename, order=XYZ):
        """Fill the grid from a binary file stored in GridDataOrder ``order``
        (SequentialLoad, dist_uniform_grid.hpp:349-482); the file is
        reordered on the GPU (device 0 unless torch's current device)."""
        t = load_grid(filename, self.nx, self.ny, self.nz, self.numScalars, order, self._is_complex())
        self.data = np.ascontiguousarray(t.cpu().numpy()).reshape(self.nz, self.ny, self.nx, self.numScalars)

    def InterpolateTo(self, nx, ny, nz):
        """Trilinear resampling to nx x ny x nz (InterpolateTo,
        dist_uniform_grid.hpp:484-714), computed on the GPU."""
        import torch
        src = torch.from_numpy(self.data.reshape(-1)).cuda()
        out = interpolate_grid(src, (self.nx, self.ny, self.nz), (nx, ny, nz), self.numScalars)
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.data = np.ascontiguousarray(out.cpu().numpy()).reshape(self.nz, self.ny, self.nx, self.numScalars)

    def WritePlane(self, planeType, whichPlane, basename):
        """ASCII VTK files of one plane, one per scalar (WritePlane,
        dist_uniform_grid.hpp:716-1631)."""
        a = np.ascontiguousarray(self.data)
        _check(lib().psp_cu_grid_write_plane(_dptr(a.view(np.float64)), self.nx, self.ny, self.nz, self.numScalars,
                                             int(self._is_complex()), int(planeType), int(whichPlane),
                                             str(basename).encode()))

    def WriteVolume(self, basename):
        """ASCII VTK volume files, one .pvti + piece per scalar (WriteVolume,
        dist_uniform_grid.hpp:1788-2200, one process)."""
        a = np.ascontiguousarray(self.data)
        _check(lib().psp_cu_grid_write_volume(_dptr(a.view(np.float64)), self.nx, self.ny, self.nz, self.numScalars,
                                              int(self._is_complex()), str(basename).encode()))


def hessenberg_eigenvalues(H):
    """Eigenvalues of a complex upper Hessenberg matrix (entries below the
    first subdiagonal ignored), as Elemental's lapack::HessenbergEig returns
    them for the Ritz values of solve.hpp:597-598.  Host only."""
    A = np.asfortranarray(np.asarray(H, dtype=np.complex128))
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise LogicError("Hessenberg matrix must be square")
    n = A.shape[0]
    w = np.zeros(n, dtype=np.complex128)
    _check(lib().psp_cu_hessenberg_eigenvalues(n, _dptr(A.reshape(-1, order="F").view(np.float64)), max(n, 1),
                                               _dptr(w.view(np.float64))))
    return w


def panel_geometry(disc, planes_per_panel=4):
    """Panel split of ``disc`` (host only): int array (num_panels, 4) of
    (lowest v, depth, padding, class) per panel, v = nz - 1 - z."""
    d = disc._c()
    n = ctypes.c_int()
    _check(lib().psp_cu_panel_geometry(ctypes.byref(d), int(planes_per_panel), ctypes.byref(n), None))
    info = np.zeros(4 * n.value, dtype=np.int32)
    _check(lib().psp_cu_panel_geometry(ctypes.byref(d), int(planes_per_panel), ctypes.byref(n), _iptr(info)))
    return info.reshape(n.value, 4)


def plan_block_width(k, avail_bytes, per_rhs_bytes, cap=0):
    """GMRES block width for k right-hand sides given the device bytes left
    and one right-hand side's workspace (psp_cu_plan_block_width; host only)."""
    wd = ctypes.c_int()
    _check(lib().psp_cu_plan_block_width(int(k), float(avail_bytes), float(per_rhs_bytes), int(cap),
                                         ctypes.byref(wd)))
    return wd.value


def analyze_class(disc, planes_per_panel=4, cutoff=12, cls=0):
    """Host-only symbolic analysis of one panel class: returns (info, ndToNat)
    with info rows (ND offset, pivot count, update count, parent)."""
    d = disc._c()
    n = ctypes.c_int()
    vs = ctypes.c_int()
    _check(lib().psp_cu_analyze_class(ctypes.byref(d), planes_per_panel, cutoff, cls, ctypes.byref(n),
                                      ctypes.byref(vs), None, None))
    info = np.zeros(4 * n.value, dtype=np.int32)
    nd = np.zeros(disc.nx * disc.ny * vs.value, dtype=np.int32)
    _check(lib().psp_cu_analyze_class(ctypes.byref(d), planes_per_panel, cutoff, cls, ctypes.byref(n),
                                      ctypes.byref(vs), _iptr(info), _iptr(nd)))
    return info.reshape(n.value, 4), nd


def load_grid(filename, nx, ny, nz, numScalars=1, order=XYZ, is_complex=False, device=None):
    """A binary grid file stored in GridDataOrder ``order`` as a CUDA tensor
    in natural order, shape (nz, ny, nx, numScalars), float64 or complex128
    (SequentialLoad, dist_uniform_grid.hpp:349-482; the reorder runs on the
    GPU)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    dtype = torch.complex128 if is_complex else torch.float64
    out = torch.empty((nz, ny, nx, numScalars), dtype=dtype, device=dev)
    with torch.cuda.device(dev):
        torch.cuda.synchronize()
        _check(lib().psp_cu_grid_load(str(filename).encode(), nx, ny, nz, numScalars, int(is_complex), int(order),
                                      ctypes.c_void_p(out.data_ptr())))
    return out


def interpolate_grid(grid, old_sizes, new_sizes, numScalars=1):
    """Trilinear resampling of a natural-order CUDA grid (float64 or
    complex128, nx*ny*nz*numScalars values) from old_sizes = (nx, ny, nz) to
    new_sizes (InterpolateTo, dist_uniform_grid.hpp:484-714); returns a new
    tensor of shape (nz, ny, nx, numScalars)."""
    import torch
    src = grid.contiguous()
    nx0, ny0, nz0 = (int(v) for v in old_sizes)
    nx, ny, nz = (int(v) for v in new_sizes)
    if src.numel() != nx0 * ny0 * nz0 * numScalars:
        raise LogicError("grid size does not match its dimensions")
    is_complex = src.is_complex()
    _device_tensor(src, "grid", "complex128" if is_complex else "float64", src.device.index)
    out = torch.empty((nz, ny, nx, numScalars), dtype=src.dtype, device=src.device)
    with torch.cuda.device(src.device):
        torch.cuda.synchronize()
        _check(lib().psp_cu_grid_interpolate(ctypes.c_void_p(src.data_ptr()), nx0, ny0, nz0, numScalars,
                                             int(is_complex), ctypes.c_void_p(out.data_ptr()), nx, ny, nz))
    return out


class DistHelmholtz:
    """``psp::DistHelmholtz<double>`` on one B200 (dist_helmholtz.hpp:21-287).

    ``DistHelmholtz(disc, damping=7.0, numPlanesPerPanel=4, cutoff=12)``;
    the MPI communicator of the reference is replaced by a CUDA device index.
    """

    def __init__(self, disc, damping=7.0, numPlanesPerPanel=4, cutoff=12, device=0):
        self.disc = disc
        self._h = None
        h = ctypes.c_void_p()
        self._d = disc._c()
        _check(lib().psp_cu_create(ctypes.byref(self._d), float(damping), int(numPlanesPerPanel), int(cutoff),
                                   int(device), ctypes.byref(h)))
        self._h = h
        self.device = int(device)
        self.N = disc.nx * disc.ny * disc.nz
        self.last_stats = None
        self._geometry = None

    def __del__(self):
        if getattr(self, "_h", None):
            lib().psp_cu_destroy(self._h)
            self._h = None

    def geometry(self):
        n = ctypes.c_int()
        _check(lib().psp_cu_geometry(self._h, ctypes.byref(n), None))
        info = np.zeros(4 * n.value, dtype=np.int32)
        _check(lib().psp_cu_geometry(self._h, ctypes.byref(n), _iptr(info)))
        return info.reshape(n.value, 4)

    def Initialize(self, velocity, panelScheme=CLIQUE_LDL_SELINV_1D, precision=FP64):
        """Assemble and factor every panel (initialize_finalize.hpp:12-377).
        ``velocity`` is a DistUniformGrid, a numpy array (natural order) or a
        CUDA torch tensor of float64."""
        if isinstance(velocity, DistUniformGrid):
            if (velocity.nx, velocity.ny, velocity.nz) != (self.disc.nx, self.disc.ny, self.disc.nz):
                raise LogicError("Velocity grid is incorrect")
            if velocity.numScalars != 1:
                raise LogicError("Velocity grid should have one entry per point")
            velocity = velocity.data
        if _is_cuda_tensor(velocity):
            if velocity.numel() != self.N:
                raise LogicError("Velocity grid is incorrect")
            v = velocity.contiguous()
            _device_tensor(v, "velocity", "float64", self.device, numel=self.N)
            _check(lib().psp_cu_initialize_device(self._h, ctypes.c_void_p(v.data_ptr()), panelScheme, precision))
            self.factor_version = getattr(self, "factor_version", 0) + 1
            return
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(-1)
        if v.size != self.N:
            raise LogicError("Velocity grid is incorrect")
        _check(lib().psp_cu_initialize(self._h, _dptr(v), panelScheme, precision))
        self.factor_version = getattr(self, "factor_version", 0) + 1

    def Solve(self, B, m=20, relTol=1e-4, viewIterates=False):
        """Solve in place (solve.hpp:12-56).  ``B`` is a complex DistUniformGrid
        whose numScalars right-hand sides are replaced by the solutions, or a
        CUDA complex128 torch tensor of nx*ny*nz*k entries.  ``viewIterates``
        (True, or a basename in place of the reference's "iterates") writes
        the iterate of every inner step that does not converge with
        WriteVolume as <basename>-<it> (solve.hpp:579-585)."""
        if not viewIterates:
            return self._solve(B, m, relTol)
        base = "iterates" if viewIterates is True else os.fspath(viewIterates)
        _check(lib().psp_cu_set_view_iterates(self._h, base.encode()))
        try:
            return self._solve(B, m, relTol)
        finally:
            lib().psp_cu_set_view_iterates(self._h, None)

    def _solve(self, B, m, relTol):
        if _is_cuda_tensor(B):
            k = _device_tensor(B, "B", "complex128", self.device, per=self.N)
            st = _Stats()
            _check(lib().psp_cu_solve_device(self._h, ctypes.c_void_p(B.data_ptr()), k, m, relTol,
                                             ctypes.byref(st)))
            self.last_stats = _stats_dict(st)
            return self.last_stats
        grid = B if isinstance(B, DistUniformGrid) else None
        arr = grid.data if grid is not None else B
        if arr.dtype != np.complex128 or not arr.flags["C_CONTIGUOUS"]:
            raise LogicError("B must be a C-contiguous complex128 grid")
        k = arr.size // self.N
        if k * self.N != arr.size:
            raise LogicError("B does not match the grid")
        st = _Stats()
        _check(lib().psp_cu_solve(self._h, _dptr(arr.view(np.float64)), k, m, relTol, ctypes.byref(st)))
        self.last_stats = _stats_dict(st)
        return self.last_stats

    SolveWithGMRES = Solve

    def Finalize(self):
        _check(lib().psp_cu_finalize(self._h))

    def set_max_iterations(self, n):
        _check(lib().psp_cu_set_max_iterations(self._h, int(n)))

    def SetRitzValues(self, mode):
        """PRINT_RITZ_VALUES (solve.hpp:589-608) at run time: 0 off, 1 record
        the Ritz values of the first GMRES restart cycle of every Solve, 2
        record and print them as the reference does."""
        _check(lib().psp_cu_set_ritz_values(self._h, int(mode)))

    def RitzValues(self):
        """Ritz values of the last Solve that recorded them: complex array
        (numRhs, steps of the first restart cycle)."""
        count, k = ctypes.c_int(), ctypes.c_int()
        _check(lib().psp_cu_get_ritz_values(self._h, ctypes.byref(count), ctypes.byref(k), None))
        out = np.zeros(count.value * k.value, dtype=np.complex128)
        if out.size:
            _check(lib().psp_cu_get_ritz_values(self._h, ctypes.byref(count), ctypes.byref(k),
                                                _dptr(out.view(np.float64))))
        return out.reshape(k.value, count.value)

    def setup_info(self):
        s = ctypes.c_double()
        b = ctypes.c_longlong()
        _check(lib().psp_cu_setup_info(self._h, ctypes.byref(s), ctypes.byref(b)))
        return s.value, b.value

    def memory_info(self):
        """Factor storage: dict(resident_panels, num_panels,
        refactorizations, scratch_bytes) (psp_cu_memory_info)."""
        r, n = ctypes.c_int(), ctypes.c_int()
        f, b = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().psp_cu_memory_info(self._h, ctypes.byref(r), ctypes.byref(n), ctypes.byref(f), ctypes.byref(b)))
        return dict(resident_panels=r.value, num_panels=n.value, refactorizations=f.value, scratch_bytes=b.value)

    def solve_block_width(self, k, m=20):
        """Right-hand sides per GMRES block that Solve of k right-hand sides
        would use now (psp_cu_solve_block_width)."""
        wd = ctypes.c_int()
        _check(lib().psp_cu_solve_block_width(self._h, int(k), int(m), ctypes.byref(wd)))
        return wd.value

    def _grid_op(self, fn, B, *extra):
        X = np.ascontiguousarray(B, dtype=np.complex128).copy()
        k = X.size // self.N
        if k == 0 or k * self.N != X.size:
            raise LogicError("B does not match the grid")
        _check(fn(self._h, _dptr(X.view(np.float64)), k, *extra))
        return X

    def multiply(self, B):
        """B := A B (Multiply, solve.hpp:613-679) on a copy."""
        return self._grid_op(lib().psp_cu_multiply, B)

    def precondition(self, B):
        """B := M^{-1} B (Precondition, solve.hpp:681-734) on a copy."""
        return self._grid_op(lib().psp_cu_precondition, B)

    def solve_panel(self, B, p):
        """B := T_p B on panel p only (SolvePanel, solve.hpp:736-882) on a copy."""
        return self._grid_op(lib().psp_cu_solve_panel, B, int(p))

    def stream_ptr(self):
        """The cudaStream_t the handle issues all work on (as an int)."""
        s = ctypes.c_void_p()
        _check(lib().psp_cu_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def set_profiling(self, on):
        _check(lib().psp_cu_set_profiling(self._h, 1 if on else 0))

    def profile_reset(self):
        _check(lib().psp_cu_profile_reset(self._h))

    def profile(self):
        """Per-category {launches, ms, flops, bytes} of profiled launches."""
        out = {}
        for i, name in enumerate(PROFILE_CATEGORIES):
            n = ctypes.c_longlong()
            ms, fl, by = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
            _check(lib().psp_cu_profile_get(self._h, i, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(fl),
                                            ctypes.byref(by)))
            out[name] = dict(launches=n.value, ms=ms.value, flops=fl.value, bytes=by.value)
        return out

    def sweep_cost(self, k):
        f, b = ctypes.c_double(), ctypes.c_double()
        _check(lib().psp_cu_sweep_cost(self._h, int(k), ctypes.byref(f), ctypes.byref(b)))
        return f.value, b.value

    def set_panel_range(self, p0, p1):
        """Factor only panels [p0, p1) (a z-panel pipeline rank); before the
        first Initialize."""
        _check(lib().psp_cu_set_panel_range(self._h, int(p0), int(p1)))

    def _panel_planes(self, panel, in_mode):
        """(lowest, highest) grid plane z that SolvePanel of `panel` reads or
        writes: its own planes, and the plane below (in_mode 1) or above
        (in_mode 2) it."""
        if self._geometry is None:
            self._geometry = self.geometry()
        if not 0 <= panel < self._geometry.shape[0]:
            raise LogicError("panel index out of range")
        low_v, depth = int(self._geometry[panel, 0]), int(self._geometry[panel, 1])
        nz = self.disc.nz
        z_lo, z_hi = nz - 1 - (low_v + depth - 1), nz - 1 - low_v
        if in_mode == 2:
            z_lo -= 1
        elif in_mode == 1:
            z_hi += 1
        if z_lo < 0 or z_hi > nz - 1:
            raise LogicError("panel %d has no neighbouring panel for in_mode %d" % (panel, in_mode))
        return z_lo, z_hi

    def solve_panel_slab(self, B, k, panel, in_mode, out_accumulate, z_base):
        """SolvePanel on a CUDA complex128 slab of planes z_base.. (in place)."""
        nxy = self.disc.nx * self.disc.ny
        planes = _device_tensor(B, "B", "complex128", self.device, per=nxy * int(k))
        z_lo, z_hi = self._panel_planes(int(panel), int(in_mode))
        if z_base > z_lo or z_base + planes - 1 < z_hi:
            raise LogicError("the slab (planes %d..%d) must hold planes %d..%d of panel %d"
                             % (z_base, z_base + planes - 1, z_lo, z_hi, panel))
        _check(lib().psp_cu_solve_panel_slab(self._h, ctypes.c_void_p(B.data_ptr()), int(k), int(panel),
                                             int(in_mode), int(out_accumulate), int(z_base)))

    def multiply_slab(self, X, Y, k, z_first, z_count, z_slab, Bv=None):
        """Y := A X (or Bv - A X) on planes [z_first, z_first + z_count) of
        CUDA complex128 slabs whose first stored plane is z_slab."""
        nxy, nz = self.disc.nx * self.disc.ny, self.disc.nz
        planes = _device_tensor(X, "X", "complex128", self.device, per=nxy * int(k))
        for t, name in ((Y, "Y"), (Bv, "Bv")):
            if t is not None and _device_tensor(t, name, "complex128", self.device, per=nxy * int(k)) != planes:
                raise LogicError("%s must be a slab of the same planes as X" % name)
        z_lo, z_hi = max(0, z_first - 1), min(nz - 1, z_first + z_count)  # with the halo planes
        if z_count < 1 or z_slab > z_lo or z_slab + planes - 1 < z_hi:
            raise LogicError("the slabs (planes %d..%d) must hold planes %d..%d"
                             % (z_slab, z_slab + planes - 1, z_lo, z_hi))
        _check(lib().psp_cu_multiply_slab(self._h, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(Y.data_ptr()),
                                          ctypes.c_void_p(Bv.data_ptr()) if Bv is not None else None, int(k),
                                          int(z_first), int(z_count), int(z_slab)))

    def multiply_device(self, B):
        k = _device_tensor(B, "B", "complex128", self.device, per=self.N)
        _check(lib().psp_cu_multiply_device(self._h, ctypes.c_void_p(B.data_ptr()), k))

    def multiply_device_noalloc(self, B):
        """B := A B in place on a CUDA tensor without any device allocation
        (for callers inside their own stream capture, or with a fixed memory
        reservation); nx*ny*nz*k must not exceed 1048576, and calls that
        overlap on the GPU race on the shared scratch array."""
        k = _device_tensor(B, "B", "complex128", self.device, per=self.N)
        _check(lib().psp_cu_multiply_device_noalloc(self._h, ctypes.c_void_p(B.data_ptr()), k))

    def precondition_device(self, B):
        k = _device_tensor(B, "B", "complex128", self.device, per=self.N)
        _check(lib().psp_cu_precondition_device(self._h, ctypes.c_void_p(B.data_ptr()), k))

    def gradient_device(self, U, Z, grad=None, accumulate=False):
        """Velocity gradient -Re(dA_ii/dvel_i * sum_r Z[i,r] U[i,r]) of a real
        misfit from forward fields U and adjoint fields Z (CUDA complex128
        tensors of nx*ny*nz*k entries, natural order); returns (or adds to)
        a CUDA float64 tensor of nx*ny*nz entries."""
        import torch
        U, Z = U.contiguous(), Z.contiguous()
        k = _device_tensor(U, "U", "complex128", self.device, per=self.N)
        if _device_tensor(Z, "Z", "complex128", self.device, per=self.N) != k:
            raise LogicError("U and Z must be grids of the same k right-hand sides")
        if grad is None:
            grad = torch.zeros(self.N, dtype=torch.float64, device=U.device)
            accumulate = False
        _device_tensor(grad, "grad", "float64", self.device, numel=self.N)
        _check(lib().psp_cu_gradient_device(self._h, ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(Z.data_ptr()), k,
                                            ctypes.c_void_p(grad.data_ptr()), 1 if accumulate else 0))
        return grad


def initialize_batch(solvers, velocities, panelScheme=CLIQUE_LDL_SELINV_1D, precision=FP64):
    """psp_cu_initialize_batch: factor independent problems (one DistHelmholtz
    each, host velocities in natural order) in one call."""
    n = len(solvers)
    vs = [np.ascontiguousarray(v, dtype=np.float64).reshape(-1) for v in velocities]
    for s, v in zip(solvers, vs):
        if v.size != s.N:
            raise LogicError("Velocity grid is incorrect")
    hs = (ctypes.c_void_p * n)(*[s._h.value for s in solvers])
    ps = (ctypes.POINTER(ctypes.c_double) * n)(*[_dptr(v) for v in vs])
    failed = ctypes.c_int()
    _check(lib().psp_cu_initialize_batch(hs, ps, n, panelScheme, precision, ctypes.byref(failed)))
    for s in solvers:
        s.factor_version = getattr(s, "factor_version", 0) + 1


def solve_batch(solvers, grids, m=20, relTol=1e-4):
    """psp_cu_solve_batch: solve in place host grids (C-contiguous complex128,
    nx*ny*nz*k each) of independent problems; returns their stats."""
    n = len(solvers)
    ks = []
    for s, g in zip(solvers, grids):
        if g.dtype != np.complex128 or not g.flags["C_CONTIGUOUS"] or g.size % s.N:
            raise LogicError("B must be a C-contiguous complex128 grid")
        ks.append(g.size // s.N)
    hs = (ctypes.c_void_p * n)(*[s._h.value for s in solvers])
    ps = (ctypes.POINTER(ctypes.c_double) * n)(*[_dptr(g.view(np.float64)) for g in grids])
    karr = (ctypes.c_int * n)(*ks)
    st = (_Stats * n)()
    failed = ctypes.c_int()
    _check(lib().psp_cu_solve_batch(hs, ps, karr, n, m, relTol, st, ctypes.byref(failed)))
    return [_stats_dict(st[i]) for i in range(n)]


def _stats_dict(st):
    return dict(iterations=st.iterations, converged=bool(st.converged), lucky_breakdown=bool(st.lucky_breakdown),
                final_max_rel_resid=st.final_max_rel_resid, solve_seconds=st.solve_seconds,
                precondition_seconds=st.precondition_seconds, matvec_seconds=st.matvec_seconds,
                arnoldi_seconds=st.arnoldi_seconds, num_preconditions=st.num_preconditions)


def _is_cuda_tensor(x):
    return getattr(x, "is_cuda", False) and hasattr(x, "data_ptr")


def _device_tensor(t, what, dtype, device, per=None, numel=None):
    """Checks a CUDA tensor before its pointer crosses the C ABI, which sees
    only an address and a count: another dtype, a strided view, a size that
    is not a whole number of grids or a tensor on another GPU would make the
    kernels read or write outside it.  Returns numel // per (or numel)."""
    import torch
    want = getattr(torch, dtype)
    if t.dtype != want:
        raise LogicError("%s must be a %s tensor, not %s" % (what, dtype, str(t.dtype).replace("torch.", "")))
    if not t.is_contiguous():
        raise LogicError("%s must be contiguous" % what)
    if t.is_conj() or t.is_neg():
        raise LogicError("%s is a lazily conjugated or negated view: resolve it first" % what)
    if t.device.index != device:
        raise LogicError("%s is on cuda:%s but the handle runs on cuda:%d" % (what, t.device.index, device))
    n = t.numel()
    if numel is not None and n != numel:
        raise LogicError("%s must hold %d entries, not %d" % (what, numel, n))
    if per is not None:
        if n == 0 or n % per:
            raise LogicError("%s must hold a positive multiple of %d entries, not %d" % (what, per, n))
        return n // per
    return n
