"""Host-buffer entry points over the pinned staging ring.

Grids larger than one 64 MB staging chunk cross several chunks and reuse the
ring's slots within one call and across calls; the results must equal the
device-buffer entry points bit for bit.
"""
import numpy as np
import pytest
import torch

import psp_b200 as P
from psp_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle(product_lib):
    w = W.small_case(interior=(40, 36, 12), pml=5, freq=2.5, k=1, seed=5, top_pml=True)
    H = P.DistHelmholtz(w.disc)
    H.Initialize(w.velocity, precision=P.MIXED)
    return w, H


def _rhs(H, k, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((H.N, k)) + 1j * rng.standard_normal((H.N, k))


def test_multichunk_multiply_matches_device_path(handle):
    w, H = handle
    k = 240  # 50 * 46 * 22 points x 240 RHS x 16 B = 194 MB: four chunks, ring reused
    B = _rhs(H, k, 1)
    host = H.multiply(B)
    dev = torch.from_numpy(B.reshape(-1)).cuda()
    H.multiply_device(dev)
    assert np.array_equal(host.reshape(-1), dev.cpu().numpy())
    # a second, smaller call through the same (already larger) ring
    B2 = _rhs(H, 3, 2)
    dev2 = torch.from_numpy(B2.reshape(-1)).cuda()
    H.multiply_device(dev2)
    assert np.array_equal(H.multiply(B2).reshape(-1), dev2.cpu().numpy())


def test_host_initialize_matches_device_initialize(handle):
    w, H = handle
    B = _rhs(H, 2, 3)
    H.Initialize(w.velocity, precision=P.MIXED)
    x_host = H.precondition(B)
    H.Initialize(torch.from_numpy(w.velocity.reshape(-1)).cuda(), precision=P.MIXED)
    x_dev = H.precondition(B)
    assert np.array_equal(x_host, x_dev)
