"""The tensor-core factorization GEMM (complex single, split TF32) against
the CUDA-core GEMM and the FP64 factorization.

Every batched-GEMM form of the frontal factorization goes through the
tensor-core tiles here (blocked LDL^T updates: transposed B, diagonal
scaling, lower-only output; the recursive-doubling inverse: triangular A
and B; G21 and the Schur complement), on fronts large enough for several
128 x 64 tiles with ragged edges.  The panel solves apply exactly those
factors, so a wrong tile shows up as an O(1) difference, while the two
complex-single factorizations agree to single-precision rounding.
"""
import os

import numpy as np
import pytest

import psp_b200 as P
from conftest import rel
from psp_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASE = dict(interior=(40, 36, 12), pml=5, freq=2.5, k=2, seed=21, top_pml=True)


def _mixed(w, cuda_cores):
    old = os.environ.get("PSP_B200_FACTOR_CUDA_CORES")
    os.environ["PSP_B200_FACTOR_CUDA_CORES"] = "1" if cuda_cores else "0"
    try:
        H = P.DistHelmholtz(w.disc)
        H.Initialize(w.velocity, precision=P.MIXED)
    finally:
        if old is None:
            del os.environ["PSP_B200_FACTOR_CUDA_CORES"]
        else:
            os.environ["PSP_B200_FACTOR_CUDA_CORES"] = old
    return H


@pytest.fixture(scope="module")
def handles(product_lib):
    w = W.small_case(**CASE)
    H64 = P.DistHelmholtz(w.disc)
    H64.Initialize(w.velocity, precision=P.FP64)
    return w, H64, _mixed(w, False), _mixed(w, True)


def test_panel_solves_match_cuda_core_factors(handles):
    w, H64, Htc, Hcc = handles
    worst_cc = worst_64 = 0.0
    for p in range(H64.geometry().shape[0]):
        x64 = H64.solve_panel(w.rhs, p)
        xtc = Htc.solve_panel(w.rhs, p)
        xcc = Hcc.solve_panel(w.rhs, p)
        worst_cc = max(worst_cc, rel(xtc, xcc))
        worst_64 = max(worst_64, rel(xtc, x64))
        # the tensor-core factors are as close to FP64 as the CUDA-core ones
        assert rel(xtc, x64) < 3 * rel(xcc, x64) + 1e-6, p
    assert worst_cc < 1e-4 and worst_64 < 1e-4, (worst_cc, worst_64)


def test_mixed_solve_with_tensor_core_factors(handles):
    w, H64, Htc, _ = handles
    X = w.rhs.copy()
    st = Htc.SolveWithGMRES(X, 20, 1e-7)
    assert st["converged"] and st["final_max_rel_resid"] < 1e-7
    X64 = w.rhs.copy()
    H64.SolveWithGMRES(X64, 20, 1e-7)
    assert rel(X, X64) < 1e-5
