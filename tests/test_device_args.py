"""Checks of device-tensor arguments in the Python binding (CPU).

The C ABI receives only an address and a count, so a tensor of the wrong
dtype, a strided or lazily conjugated view, a size that is not a whole
number of grids, a tensor on another GPU or a slab that does not hold the
planes a call touches would make the kernels read or write outside it.  The
binding refuses those before any pointer crosses; these tests drive it with
stand-in tensors whose pointer must never be taken, and check that the
calls the z-panel pipeline makes pass every check.
"""
import pytest
import torch

import psp_b200 as P
from psp_b200 import workloads as W
from psp_b200 import zpanel as Z

CASE = dict(interior=(10, 9, 14), pml=4, freq=1.5, k=3, seed=3, top_pml=True)


class PointerTaken(Exception):
    pass


class FakeCuda:
    """A CUDA tensor as far as the binding's checks can see."""
    is_cuda = True

    def __init__(self, n, dtype=torch.complex128, index=0, contiguous=True, conj=False):
        self.dtype, self._n, self.device = dtype, int(n), torch.device("cuda", index)
        self._contig, self._conj = contiguous, conj

    def numel(self):
        return self._n

    def is_contiguous(self):
        return self._contig

    def is_conj(self):
        return self._conj

    def is_neg(self):
        return False

    def is_complex(self):
        return self.dtype.is_complex

    def contiguous(self):
        return self

    def data_ptr(self):
        raise PointerTaken()


def _unbound(case):
    """A DistHelmholtz whose checks run without a GPU (no C ABI handle)."""
    w = W.small_case(**case)
    H = object.__new__(P.DistHelmholtz)
    H._h, H.device, H.disc, H.last_stats = None, 0, w.disc, None
    H.N = w.disc.nx * w.disc.ny * w.disc.nz
    H._geometry = P.panel_geometry(w.disc, 4)
    return w, H


@pytest.fixture(scope="module")
def handle():
    return _unbound(CASE)


@pytest.mark.parametrize("call", ["multiply_device", "multiply_device_noalloc", "precondition_device", "Solve"])
def test_grid_tensors_are_checked(handle, call):
    w, H = handle
    f = getattr(H, call)
    with pytest.raises(P.LogicError, match="complex128"):
        f(FakeCuda(H.N * 2, torch.complex64))
    with pytest.raises(P.LogicError, match="contiguous"):
        f(FakeCuda(H.N * 2, contiguous=False))
    with pytest.raises(P.LogicError, match="conjugated"):
        f(FakeCuda(H.N * 2, conj=True))
    with pytest.raises(P.LogicError, match="cuda:1"):
        f(FakeCuda(H.N * 2, index=1))
    with pytest.raises(P.LogicError, match="multiple"):
        f(FakeCuda(H.N * 2 + 1))
    with pytest.raises(P.LogicError, match="multiple"):
        f(FakeCuda(0))
    with pytest.raises(PointerTaken):
        f(FakeCuda(H.N * 2))


def test_velocity_and_gradient_tensors_are_checked(handle):
    w, H = handle
    with pytest.raises(P.LogicError, match="float64"):
        H.Initialize(FakeCuda(H.N, torch.float32))
    with pytest.raises(P.LogicError, match="incorrect"):
        H.Initialize(FakeCuda(H.N + 1, torch.float64))
    with pytest.raises(PointerTaken):
        H.Initialize(FakeCuda(H.N, torch.float64))
    U = FakeCuda(H.N * 2)
    with pytest.raises(P.LogicError, match="same k"):
        H.gradient_device(U, FakeCuda(H.N * 3))
    with pytest.raises(P.LogicError, match="complex128"):
        H.gradient_device(U, FakeCuda(H.N * 2, torch.complex64))
    with pytest.raises(P.LogicError, match="float64"):
        H.gradient_device(U, FakeCuda(H.N * 2), grad=FakeCuda(H.N, torch.float32))
    with pytest.raises(P.LogicError, match="entries"):
        H.gradient_device(U, FakeCuda(H.N * 2), grad=FakeCuda(H.N + 1, torch.float64))
    with pytest.raises(PointerTaken):
        H.gradient_device(U, FakeCuda(H.N * 2), grad=FakeCuda(H.N, torch.float64))


def test_interpolation_source_is_checked():
    with pytest.raises(P.LogicError, match="float64"):
        P.interpolate_grid(FakeCuda(4 * 4 * 4, torch.float32), (4, 4, 4), (8, 8, 8))
    with pytest.raises(P.LogicError, match="match"):
        P.interpolate_grid(FakeCuda(4 * 4 * 5, torch.float64), (4, 4, 4), (8, 8, 8))


def test_slabs_must_hold_the_planes_a_call_touches(handle):
    w, H = handle
    d = w.disc
    nxy, nz, k = d.nx * d.ny, d.nz, 2
    geo = H._geometry
    np_ = geo.shape[0]
    # panel 1's own planes and the plane below it (in_mode 1)
    low_v, depth = int(geo[1, 0]), int(geo[1, 1])
    z_lo, z_hi = nz - 1 - (low_v + depth - 1), nz - low_v
    slab = FakeCuda((z_hi - z_lo + 1) * nxy * k)
    with pytest.raises(PointerTaken):
        H.solve_panel_slab(slab, k, 1, 1, 0, z_lo)
    with pytest.raises(P.LogicError, match="must hold"):
        H.solve_panel_slab(slab, k, 1, 1, 0, z_lo + 1)       # starts above the panel's top plane
    with pytest.raises(P.LogicError, match="must hold"):
        H.solve_panel_slab(FakeCuda((z_hi - z_lo) * nxy * k), k, 1, 1, 0, z_lo)  # misses the plane below
    with pytest.raises(P.LogicError, match="must hold"):
        H.solve_panel_slab(slab, k, 1, 2, 0, z_lo)           # in_mode 2 reads the plane above
    with pytest.raises(P.LogicError, match="multiple"):
        H.solve_panel_slab(FakeCuda(slab.numel() + nxy), k, 1, 1, 0, z_lo)
    with pytest.raises(P.LogicError, match="no neighbouring panel"):
        H.solve_panel_slab(FakeCuda(nz * nxy * k), k, 0, 1, 0, 0)        # nothing below the bottom panel
    with pytest.raises(P.LogicError, match="no neighbouring panel"):
        H.solve_panel_slab(FakeCuda(nz * nxy * k), k, np_ - 1, 2, 0, 0)  # nothing above the top panel
    with pytest.raises(P.LogicError, match="out of range"):
        H.solve_panel_slab(FakeCuda(nz * nxy * k), k, np_, 0, 0, 0)
    # the matvec needs one halo plane on each side that exists
    X = FakeCuda(6 * nxy * k)
    with pytest.raises(PointerTaken):
        H.multiply_slab(X, FakeCuda(6 * nxy * k), k, 4, 4, 3)
    with pytest.raises(P.LogicError, match="must hold"):
        H.multiply_slab(X, FakeCuda(6 * nxy * k), k, 4, 4, 4)   # no halo plane below plane 4
    with pytest.raises(P.LogicError, match="must hold"):
        H.multiply_slab(X, FakeCuda(6 * nxy * k), k, 4, 5, 3)   # no halo plane above plane 8
    with pytest.raises(P.LogicError, match="same planes"):
        H.multiply_slab(X, FakeCuda(5 * nxy * k), k, 4, 4, 3)
    with pytest.raises(PointerTaken):
        H.multiply_slab(FakeCuda(nz * nxy * k), FakeCuda(nz * nxy * k), k, 0, nz, 0)


# the pipeline tests' workload (tests/test_zpanel.py) beside this file's
PIPELINE_CASES = [CASE, dict(interior=(12, 13, 22), pml=5, freq=2.0, k=3, seed=17, top_pml=True)]


@pytest.mark.parametrize("case", range(len(PIPELINE_CASES)))
@pytest.mark.parametrize("world", [1, 2, 3])
def test_pipeline_calls_pass_the_checks(world, case):
    """Every panel solve and matvec a z-panel rank issues (forward, backward,
    halo matvec; whole and column-blocked slabs) passes the checks."""
    w, H = _unbound(PIPELINE_CASES[case])
    d = w.disc
    nxy = d.nx * d.ny
    geo, costs = Z.panel_costs(d)
    ranges = Z.partition(costs, world)
    for r in range(world):
        L = Z.Layout(geo, d.nz, nxy, r, ranges)
        for k in (w.k, 1):
            W_ = FakeCuda(L.nplanes * nxy * k)
            for p in range(L.p0, L.p1):
                with pytest.raises(PointerTaken):
                    H.solve_panel_slab(W_, k, p, 0 if p == 0 else 1, 0, L.zs)
            for p in range(min(L.p1, L.num_panels - 1) - 1, L.p0 - 1, -1):
                with pytest.raises(PointerTaken):
                    H.solve_panel_slab(W_, k, p, 2, 1, L.zs)
            with pytest.raises(PointerTaken):
                H.multiply_slab(W_, FakeCuda(W_.numel()), k, L.zlo, L.zhi + 1 - L.zlo, L.zs, FakeCuda(W_.numel()))
