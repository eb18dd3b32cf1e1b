"""C ABI surface checks that need no GPU: the library loads, exports every
entry point declared in include/psp_b200.h, converts errors into status
codes, and the Python mirror of the reference types behaves like the
reference's value types."""
import ctypes
import os
import re

import numpy as np
import pytest

import psp_b200 as P

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "psp_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(psp_cu_\w+)\s*\(", text)))


def test_header_declares_the_binding_list():
    assert declared_symbols() == sorted(P.C_ABI_SYMBOLS)


def test_library_exports_every_declared_symbol(product_lib):
    for name in declared_symbols():
        assert hasattr(product_lib, name), name
        assert isinstance(getattr(product_lib, name), ctypes._CFuncPtr)


def test_null_arguments_are_logic_errors(product_lib):
    h = ctypes.c_void_p()
    assert product_lib.psp_cu_create(None, 7.0, 4, 12, 0, ctypes.byref(h)) == 1
    assert b"null" in product_lib.psp_cu_last_error()
    assert product_lib.psp_cu_finalize(None) == 1
    # the diagnostics switches and their read-out check the handle too
    assert product_lib.psp_cu_set_view_iterates(None, b"iterates") == 1
    assert product_lib.psp_cu_set_ritz_values(None, 1) == 1
    count, k = ctypes.c_int(-1), ctypes.c_int(-1)
    assert product_lib.psp_cu_get_ritz_values(None, ctypes.byref(count), ctypes.byref(k), None) == 1
    assert count.value == -1 and k.value == -1


def test_compute_without_device_fails_loudly(product_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    d = P.Discretization(10.0, 20, 20, 25, 1.0, 1.0, 1.0, pml=(5, 5, 5))
    with pytest.raises(P.CudaError, match="no CUDA device"):
        P.DistHelmholtz(d)


def test_discretization_defaults_follow_reference():
    d = P.Discretization(30.0, 40, 40, 40, 1.0, 2.0, 1.5)
    assert (d.bx, d.by, d.bz) == (5, 5, 5)
    assert d.sigmax == d.sigmay == d.sigmaz == pytest.approx(1.2 * 2.0)
    assert (d.frontBC, d.rightBC, d.backBC, d.leftBC, d.topBC) == (P.PML,) * 5
    d2 = P.Discretization(30.0, 40, 40, 40, 1.0, 1.0, 1.0, bcs=(P.PML,) * 4 + (P.DIRICHLET,), pml=8, sigma=1.5)
    assert (d2.bx, d2.by, d2.bz, d2.sigmax, d2.topBC) == (8, 8, 8, 1.5, P.DIRICHLET)


def test_grid_local_index_and_orders():
    g = P.DistUniformGrid(4, 3, 2, numScalars=3)
    assert g.LocalIndex(1, 2, 1) == (1 + 2 * 4 + 1 * 12) * 3
    rng = np.random.default_rng(0)
    ref = rng.standard_normal((2, 3, 4, 3)) + 0j   # (z, y, x, k)
    layouts = {
        P.XYZ: ref,
        P.XZY: ref.transpose(1, 0, 2, 3),
        P.YXZ: ref.transpose(0, 2, 1, 3),
        P.YZX: ref.transpose(2, 0, 1, 3),
        P.ZXY: ref.transpose(1, 2, 0, 3),
        P.ZYX: ref.transpose(2, 1, 0, 3),
    }
    for order, stored in layouts.items():
        h = P.DistUniformGrid.from_order(stored.ravel(), 4, 3, 2, 3, order)
        assert np.array_equal(h.data, ref), order


def test_gmres_block_width_choice():
    """The GMRES block width for the memory left (host-only form of the
    choice Solve makes): all right-hand sides when they fit; otherwise equal
    blocks as wide as fit, rounded up to whole 16-column sweep tiles when
    that still fits; the environment-style cap; out-of-memory, with the
    sizes, when not even one right-hand side fits."""
    GB = 1e9
    per = 2.6 * GB
    assert P.plan_block_width(16, 100 * GB, per) == 16
    assert P.plan_block_width(64, 96 * GB, per) == 32          # fit 35: two blocks of 32
    assert P.plan_block_width(64, 80 * GB, per) == 22          # fit 29: three blocks of 22 (32 does not fit)
    assert P.plan_block_width(64, 60 * GB, per) == 16          # fit 21: four blocks of 16
    assert P.plan_block_width(3, 100 * GB, per, cap=2) == 2    # blocks of 2 (the last padded)
    assert P.plan_block_width(5, 3 * GB, per) == 1
    with pytest.raises(P.CudaError, match="does not fit"):
        P.plan_block_width(4, 2 * GB, per)
    with pytest.raises(P.LogicError):
        P.plan_block_width(0, 100 * GB, per)
