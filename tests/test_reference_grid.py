"""The reference's own grid code against the oracle restatement and the
product (CPU).

oracle/_ref/libpspref.so is include/psp/dist_uniform_grid.hpp of the
reference compiled unchanged against a one-process stand-in for the
Elemental / MPI names it uses (oracle/refshim, ``make -C oracle ref``).  Its
SequentialLoad, InterpolateTo, WritePlane and WriteVolume must agree with
oracle/grid_io.py bit for bit and byte for byte, which pins the oracle that
the device kernels are tested against (tests/test_grid_io.py) to the
reference code itself; the product's host writers are compared with the
reference directly.  Skipped where the reference tree was not available to
build the library.
"""
import os

import numpy as np
import pytest

import psp_b200 as P
from oracle import grid_io as O
from oracle import ref

pytestmark = pytest.mark.skipif(
    not (ref.available() or os.path.isdir(os.path.join(ref.REF_TREE, "include", "psp"))),
    reason="the reference's grid code is not built here")


def _grid(nx, ny, nz, ns, complex_, seed):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((nz, ny, nx, ns))
    if complex_:
        g = g + 1j * rng.standard_normal((nz, ny, nx, ns))
    # entries the writers print specially
    g.reshape(-1)[0] = 1e-310
    g.reshape(-1)[1] = -0.0
    g.reshape(-1)[2] = 123456789.0
    return g


@pytest.mark.parametrize("complex_", [False, True])
@pytest.mark.parametrize("order", range(6))
def test_sequential_load_matches_reference(tmp_path, order, complex_):
    # The reference's ZXY layout multiplies by zLocalSize * yLocalSize where
    # zLocalSize * xLocalSize is meant (dist_uniform_grid.hpp:334); it is a
    # permutation only when nx == ny, so that order is checked on a grid
    # with nx == ny.
    nx = 4 if order == O.ZXY else 6
    g = _grid(nx, 4, 5, 2, complex_, 10 + order)
    path = str(tmp_path / "grid.bin")
    flat = O.to_file_order(g, order)
    flat.tofile(path)
    got = ref.sequential_load(path, nx, 4, 5, 2, order, complex_)
    assert np.array_equal(got, g)
    assert np.array_equal(O.sequential_load(flat, nx, 4, 5, 2, order), got)


@pytest.mark.parametrize("complex_", [False, True])
@pytest.mark.parametrize("shape", [(11, 7, 9), (3, 3, 2), (6, 4, 5), (12, 8, 10)])
def test_interpolate_to_matches_reference(complex_, shape):
    g = _grid(6, 4, 5, 3, complex_, 21)
    got = ref.interpolate_to(g, *shape)
    want = O.interpolate_to(g, *shape)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


@pytest.mark.parametrize("complex_", [False, True])
@pytest.mark.parametrize("plane,which", [(O.XY, 0), (O.XY, 2), (O.XZ, 3), (O.YZ, 4)])
def test_write_plane_matches_reference(tmp_path, complex_, plane, which):
    g = _grid(6, 5, 4, 2, complex_, 31)
    (tmp_path / "ref").mkdir()
    (tmp_path / "ours").mkdir()
    ref.write_plane(g, plane, which, str(tmp_path / "ref" / "plane"))
    P.DistUniformGrid(6, 5, 4, 2, dtype=g.dtype, data=g).WritePlane(plane, which, str(tmp_path / "ours" / "plane"))
    want = O.plane_text(g, plane, which)
    assert sorted(os.listdir(tmp_path / "ref")) == sorted("plane%s.vti" % s for s in want)
    for suffix, text in want.items():
        name = "plane%s.vti" % suffix
        with open(tmp_path / "ref" / name) as f:
            got = f.read()
        assert got == text, suffix
        with open(tmp_path / "ours" / name) as f:
            assert f.read() == got, suffix


@pytest.mark.parametrize("complex_", [False, True])
def test_write_volume_matches_reference(tmp_path, monkeypatch, complex_):
    g = _grid(6, 5, 4, 2, complex_, 41)
    for d in ("ref", "ours"):
        (tmp_path / d).mkdir()
    monkeypatch.chdir(tmp_path / "ref")
    ref.write_volume(g, "vol")
    monkeypatch.chdir(tmp_path / "ours")
    P.DistUniformGrid(6, 5, 4, 2, dtype=g.dtype, data=g).WriteVolume("vol")
    want = O.volume_texts(g, "vol")
    for name, text in want.items():
        with open(tmp_path / "ref" / name) as f:
            got = f.read()
        assert got == text, name
        with open(tmp_path / "ours" / name) as f:
            assert f.read() == got, name
