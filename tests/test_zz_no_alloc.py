"""The allocation-free multiply (psp_cu_multiply_device_noalloc).

Some callers cannot allocate device memory at call time: code running inside
its own CUDA stream capture, and services that reserve all device memory when
they start.  For them the C ABI offers an in-place B := A B whose temporary
lives in a fixed 16 MiB device array instead of a per-call allocation.  This
file checks it through the C ABI against psp_cu_multiply_device on the same
inputs, twice in a row (the shared array keeps the previous call's contents),
and checks the size limit.  It is collected last on purpose.
"""
import numpy as np
import pytest

import psp_b200 as P
from conftest import rel
from psp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_noalloc_multiply_matches_allocating_multiply(product_lib):
    import torch
    w = W.small_case(interior=(12, 13, 14), pml=5, freq=2.0, k=3, seed=21)
    H = P.DistHelmholtz(w.disc)
    H.Initialize(w.velocity, precision=P.FP64)
    rng = np.random.default_rng(5)
    for call in range(2):
        X = w.rhs + call * (rng.standard_normal(w.rhs.shape) + 1j * rng.standard_normal(w.rhs.shape))
        ref = torch.from_numpy(X.reshape(-1).copy()).cuda()
        got = torch.from_numpy(X.reshape(-1).copy()).cuda()
        H.multiply_device(ref)
        H.multiply_device_noalloc(got)
        torch.cuda.synchronize()
        assert rel(got.cpu().numpy(), ref.cpu().numpy()) < 1e-13, call


def test_noalloc_multiply_leaves_device_memory_untouched(product_lib):
    """After the first call on a device (which only resolves the array's
    address), repeated calls change neither the device's free memory nor
    the caller's current device."""
    import torch
    w = W.small_case(interior=(12, 13, 14), pml=5, freq=2.0, k=2, seed=21)
    H = P.DistHelmholtz(w.disc)
    H.Initialize(w.velocity, precision=P.FP64)
    B = torch.from_numpy(w.rhs.reshape(-1).copy()).cuda()
    H.multiply_device_noalloc(B)
    torch.cuda.synchronize()
    dev = torch.cuda.current_device()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        H.multiply_device_noalloc(B)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.current_device() == dev


def test_noalloc_multiply_rejects_grids_beyond_its_scratch(product_lib):
    import torch
    w = W.small_case(interior=(12, 13, 14), pml=5, freq=2.0, k=1, seed=21)
    H = P.DistHelmholtz(w.disc)
    H.Initialize(w.velocity, precision=P.FP64)
    k = (1 << 20) // H.N + 1           # nx*ny*nz*k just above 1048576
    B = torch.zeros(H.N * k, dtype=torch.complex128, device="cuda")
    with pytest.raises(P.LogicError, match="exceeds"):
        H.multiply_device_noalloc(B)
