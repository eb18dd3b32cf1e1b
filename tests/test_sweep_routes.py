"""Per-depth choice between the tensor-core and the CUDA-core sweep kernels
(complex single).

The sweep plan times every candidate (kernel and K-chunk) of every tree
depth of one panel solve per panel class and keeps the fastest for each
depth and direction.  Both
kernels read and write the same front work vectors, so any mix must give
the same preconditioner up to single-precision rounding: a fixed
alternating mix, tensor cores everywhere, CUDA cores everywhere and the
timed choice are compared with each other and with the FP64 oracle.
"""
import os

import numpy as np
import pytest

import psp_b200 as P
from conftest import oracle_for, rel
from psp_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASE = dict(interior=(40, 36, 12), pml=5, freq=2.5, k=3, seed=21, top_pml=True)


def _with_env(env, fn):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: v for k, v in env.items() if v is not None})
    for k, v in env.items():
        if v is None:
            os.environ.pop(k, None)
    try:
        return fn()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _mixed_handle(w, env):
    # both variables are read when the handle's factor store and its sweep
    # plan are built: at Initialize and at the first panel solve
    def make():
        H = P.DistHelmholtz(w.disc)
        H.Initialize(w.velocity, precision=P.MIXED)
        H.precondition(w.rhs)
        return H
    return _with_env(env, make)


@pytest.fixture(scope="module")
def setup(product_lib):
    w = W.small_case(**CASE)
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    routes = {
        "auto": {"PSP_B200_SWEEP_AUTOTUNE": "1", "PSP_B200_SWEEP_CUDA_CORES": None},
        "tensor": {"PSP_B200_SWEEP_AUTOTUNE": "0", "PSP_B200_SWEEP_CUDA_CORES": None},
        "alternate": {"PSP_B200_SWEEP_AUTOTUNE": "alternate", "PSP_B200_SWEEP_CUDA_CORES": None},
        "cuda_cores": {"PSP_B200_SWEEP_AUTOTUNE": None, "PSP_B200_SWEEP_CUDA_CORES": "1"},
    }
    return w, O, {name: _mixed_handle(w, env) for name, env in routes.items()}


def test_every_route_gives_the_same_preconditioner(setup):
    w, O, H = setup
    ref = O.precondition(w.rhs)
    out = {name: h.precondition(w.rhs) for name, h in H.items()}
    for name, x in out.items():
        assert rel(x, ref) < 1e-4, name
        assert rel(x, out["cuda_cores"]) < 2e-5, name
        assert rel(x, out["tensor"]) < 2e-5, name


def test_every_route_gives_the_same_panel_solves(setup):
    w, O, H = setup
    for p in range(O.geometry().shape[0]):
        ref = O.solve_panel(w.rhs, p)
        for name, h in H.items():
            assert rel(h.solve_panel(w.rhs, p), ref) < 1e-4, (name, p)


def test_mixed_route_solve_converges(setup):
    w, O, H = setup
    X, sto = O.solve(w.rhs, 20, 1e-6)
    for name in ("alternate", "auto"):
        Xm = w.rhs.copy()
        st = H[name].SolveWithGMRES(Xm, 20, 1e-6)
        assert st["converged"] and st["final_max_rel_resid"] < 1e-6, name
        assert abs(st["iterations"] - sto["iterations"]) <= 2, name
        assert rel(Xm, X) < 1e-4, name


@pytest.mark.parametrize("k", [16, 32, 40])
def test_wide_tensor_core_tiles_match(product_lib, k):
    """Tile widths of the tensor-core kernels: more than 16 right-hand sides
    take 32-wide tiles (each G stage split once for all of them; k = 40
    leaves a partly filled last tile), 16 take 16-wide ones; the small
    fronts' short K-chunks exercise the split-K reduction per 16-column
    sub-tile.  The preconditioner and every panel solve agree with the
    CUDA-core kernels and the oracle, and a mixed solve converges like the
    oracle's."""
    w = W.small_case(**dict(CASE, k=k))
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    wide = _mixed_handle(w, {"PSP_B200_SWEEP_AUTOTUNE": "0", "PSP_B200_SWEEP_CUDA_CORES": None})
    cc = _mixed_handle(w, {"PSP_B200_SWEEP_AUTOTUNE": None, "PSP_B200_SWEEP_CUDA_CORES": "1"})
    ref = O.precondition(w.rhs)
    x = wide.precondition(w.rhs)
    assert rel(x, ref) < 1e-4
    assert rel(x, cc.precondition(w.rhs)) < 2e-5
    for p in range(O.geometry().shape[0]):
        assert rel(wide.solve_panel(w.rhs, p), O.solve_panel(w.rhs, p)) < 1e-4, p
    X, sto = O.solve(w.rhs, 20, 1e-6)
    Xm = w.rhs.copy()
    st = wide.Solve(Xm, 20, 1e-6)
    assert st["converged"] and abs(st["iterations"] - sto["iterations"]) <= 2
    assert rel(Xm, X) < 1e-4


def test_long_chunks_sum_their_chains_in_fp32(product_lib):
    """The tensor core adds each MMA's products into its FP32 accumulator
    with truncation, so a tile keeps at most four 16-column stages (64
    complex K) in one TMEM accumulator and the epilogue sums these chains in
    FP32.  A tiling of 512-column K-chunks (chains summed inside the tile)
    and one of 64-column chunks (one chain per tile, the chunks summed by the
    split-K reduction) run the same MMAs per chain and must agree to FP32
    rounding (a lost or repeated chain would be off by O(1)); both agree with
    the CUDA-core kernels and the oracle.  The root fronts here have K ranges
    of several hundred columns, so the long tiles hold up to eight chains."""
    w = W.small_case(**dict(CASE, k=32))
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    env = {"PSP_B200_SWEEP_AUTOTUNE": "0", "PSP_B200_SWEEP_CUDA_CORES": None}
    long_ = _mixed_handle(w, dict(env, PSP_B200_SWEEP_TC_CHUNK="512"))
    short = _mixed_handle(w, dict(env, PSP_B200_SWEEP_TC_CHUNK="64"))
    cc = _mixed_handle(w, {"PSP_B200_SWEEP_AUTOTUNE": None, "PSP_B200_SWEEP_CUDA_CORES": "1"})
    x_long, x_short = long_.precondition(w.rhs), short.precondition(w.rhs)
    assert rel(x_long, x_short) < 1e-6
    assert rel(x_long, cc.precondition(w.rhs)) < 2e-5
    assert rel(x_long, O.precondition(w.rhs)) < 1e-4
    for p in range(O.geometry().shape[0]):
        assert rel(long_.solve_panel(w.rhs, p), short.solve_panel(w.rhs, p)) < 1e-6, p
