"""Grid ingest and output (psp::DistUniformGrid::SequentialLoad,
InterpolateTo, WritePlane, WriteVolume) against the numpy restatement in
oracle/grid_io.py.

CPU: the oracle's storage orders agree with the grid class's own reorder;
the C-ABI VTK writers produce the oracle's text byte for byte; argument
errors follow the reference.  GPU: files in all six storage orders load
bit-exactly; trilinear resampling (real and complex, several scalars, up
and down) equals the oracle bit for bit; a velocity model loaded from a
file and resampled on the device feeds Initialize exactly as the oracle's
resampled model does.
"""
import os

import numpy as np
import pytest

import psp_b200 as P
from oracle import grid_io as O


def _grid(nx, ny, nz, ns, complex_, seed):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((nz, ny, nx, ns))
    if complex_:
        g = g + 1j * rng.standard_normal((nz, ny, nx, ns))
    # a few entries the writers print specially
    g.reshape(-1)[0] = 1e-310
    g.reshape(-1)[1] = -0.0
    g.reshape(-1)[2] = 123456789.0
    return g


@pytest.mark.parametrize("order", range(6))
def test_oracle_orders_match_grid_reorder(order):
    g = _grid(5, 4, 3, 2, True, order)
    flat = O.to_file_order(g, order)
    assert np.array_equal(O.sequential_load(flat, 5, 4, 3, 2, order), g)
    h = P.DistUniformGrid.from_order(flat, 5, 4, 3, 2, order)
    assert np.array_equal(h.data, g)


@pytest.mark.parametrize("complex_", [False, True])
@pytest.mark.parametrize("plane,which", [(O.XY, 0), (O.XY, 2), (O.XZ, 3), (O.YZ, 4)])
def test_write_plane_matches_oracle(tmp_path, complex_, plane, which):
    g = _grid(6, 5, 4, 2, complex_, 11)
    grid = P.DistUniformGrid(6, 5, 4, 2, dtype=g.dtype, data=g)
    base = str(tmp_path / "plane")
    grid.WritePlane(plane, which, base)
    want = O.plane_text(g, plane, which)
    for suffix, text in want.items():
        with open(base + suffix + ".vti") as f:
            assert f.read() == text, suffix
    assert len(os.listdir(tmp_path)) == len(want)


@pytest.mark.parametrize("complex_", [False, True])
def test_write_volume_matches_oracle(tmp_path, complex_):
    g = _grid(4, 3, 5, 2, complex_, 12)
    grid = P.DistUniformGrid(4, 3, 5, 2, dtype=g.dtype, data=g)
    base = str(tmp_path / "vol")
    grid.WriteVolume(base)
    for name, text in O.volume_texts(g, base).items():
        with open(name) as f:
            assert f.read() == text, name


def test_writer_errors_follow_the_reference(tmp_path):
    grid = P.DistUniformGrid(4, 3, 2, 1, dtype=np.float64)
    with pytest.raises(P.LogicError, match="Invalid plane"):
        grid.WritePlane(P.XY, 2, str(tmp_path / "p"))
    with pytest.raises(P.LogicError, match="Invalid plane"):
        grid.WritePlane(P.YZ, -1, str(tmp_path / "p"))
    with pytest.raises(P.LogicError, match="Could not open"):
        grid.WritePlane(P.XZ, 0, str(tmp_path / "missing_dir" / "p"))


def test_oracle_interpolation_reproduces_linear_fields():
    nz, ny, nx = 4, 5, 6
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    g = (0.5 + 2.0 * x + 3.0 * y - 1.5 * z)[..., None].astype(np.float64)
    out = O.interpolate_to(g, 11, 7, 9)
    zz, yy, xx = np.meshgrid(np.arange(9) * 3 / 8, np.arange(7) * 4 / 6, np.arange(11) * 5 / 10, indexing="ij")
    assert np.allclose(out[..., 0], 0.5 + 2.0 * xx + 3.0 * yy - 1.5 * zz, rtol=0, atol=1e-12)


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("order", range(6))
@pytest.mark.parametrize("complex_", [False, True])
def test_load_every_order_bit_exact(product_lib, tmp_path, order, complex_):
    g = _grid(7, 5, 6, 3, complex_, 20 + order)
    path = tmp_path / "grid.bin"
    O.to_file_order(g, order).tofile(path)
    t = P.load_grid(path, 7, 5, 6, 3, order, complex_)
    assert np.array_equal(t.cpu().numpy(), g)
    grid = P.DistUniformGrid(7, 5, 6, 3, dtype=g.dtype)
    grid.SequentialLoad(path, order)
    assert np.array_equal(grid.data, g)


@pytest.mark.gpu
def test_load_errors(product_lib, tmp_path):
    with pytest.raises(P.LogicError, match="Could not open"):
        P.load_grid(tmp_path / "absent.bin", 4, 4, 4)
    path = tmp_path / "short.bin"
    np.zeros(10).tofile(path)
    with pytest.raises(P.LogicError, match="fewer values"):
        P.load_grid(path, 4, 4, 4)


@pytest.mark.gpu
@pytest.mark.parametrize("complex_", [False, True])
@pytest.mark.parametrize("old,new", [((9, 7, 5), (17, 12, 9)), ((20, 16, 12), (7, 9, 5)), ((6, 6, 6), (6, 11, 6))])
def test_interpolation_bit_exact(product_lib, complex_, old, new):
    import torch
    g = _grid(*old, 2, complex_, 31)
    src = torch.from_numpy(g.reshape(-1)).cuda()
    out = P.interpolate_grid(src, old, new, 2).cpu().numpy()
    want = O.interpolate_to(g, *new)
    assert out.shape == want.shape
    assert np.array_equal(out, want)


@pytest.mark.gpu
def test_loaded_model_feeds_the_solver(product_lib, tmp_path):
    import torch
    from psp_b200 import workloads as W
    w = W.small_case(interior=(12, 13, 14), pml=5, freq=2.0, k=2, seed=7, top_pml=True)
    nx, ny, nz = w.disc.nx, w.disc.ny, w.disc.nz
    # a coarse model stored in ZYX order, resampled onto the discretization
    rng = np.random.default_rng(8)
    coarse = 1.0 + 0.2 * rng.random((9, 10, 11, 1))
    path = tmp_path / "model.bin"
    O.to_file_order(coarse, O.ZYX).tofile(path)
    t = P.load_grid(path, 11, 10, 9, 1, O.ZYX)
    vel = P.interpolate_grid(t, (11, 10, 9), (nx, ny, nz))
    want = O.interpolate_to(coarse, nx, ny, nz)
    assert np.array_equal(vel.cpu().numpy(), want)
    H = P.DistHelmholtz(w.disc)
    H.Initialize(vel.reshape(-1), precision=P.FP64)
    X1 = w.rhs.copy()
    s1 = H.SolveWithGMRES(X1, 20, 1e-6)
    H.Initialize(want.reshape(-1), precision=P.FP64)
    X2 = w.rhs.copy()
    s2 = H.SolveWithGMRES(X2, 20, 1e-6)
    assert s1["converged"] and s1["iterations"] == s2["iterations"]
    assert np.array_equal(X1, X2)
