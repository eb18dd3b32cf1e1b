"""The reference-style C++ surface (include/psp/psp.hpp) compiles against the
C ABI, rejects a shallow domain with std::logic_error on the host, and (on a
GPU) drives a full Initialize/Solve like the reference's UnitCube driver."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "drivers", "unit_cube.cpp")


@pytest.fixture(scope="module")
def driver(product_lib, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("drv") / "unit_cube")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    libdir = os.path.join(ROOT, "psp_b200")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), SRC, "-o", out,
                    "-L", libdir, "-lpsp_b200", "-Wl,-rpath," + libdir], check=True)
    return out


def test_driver_compiles_and_reports_shallow_domain(driver):
    # n = 18 with PML 5 and 4 planes per panel is too shallow to sweep
    r = subprocess.run([driver, "18"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "shallow" in r.stderr


@pytest.mark.gpu
def test_driver_solves_on_gpu(driver):
    for prec in ("0", "1"):
        r = subprocess.run([driver, "30", "15", prec], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "converged 1" in r.stdout


GRID_SRC = os.path.join(ROOT, "tests", "drivers", "grid_io.cpp")


@pytest.fixture(scope="module")
def grid_driver(product_lib, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("grid") / "grid_io")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    libdir = os.path.join(ROOT, "psp_b200")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), GRID_SRC, "-o", out,
                    "-L", libdir, "-lpsp_b200", "-Wl,-rpath," + libdir], check=True)
    return out


def _driver_grid():
    import numpy as np
    z, y, x = np.meshgrid(np.arange(4), np.arange(5), np.arange(6), indexing="ij")
    return (1.0 + 0.25 * x - 0.5 * y + 0.125 * x * z + 0.01 * y * y)[..., None]


def test_grid_writers_from_cpp(grid_driver, tmp_path):
    from oracle import grid_io as O
    r = subprocess.run([grid_driver, "write", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    g = _driver_grid()
    for suffix, text in O.plane_text(g, O.XY, 1).items():
        assert open(str(tmp_path / "plane") + suffix + ".vti").read() == text
    for name, text in O.volume_texts(g, str(tmp_path / "volume")).items():
        assert open(name).read() == text


@pytest.mark.gpu
def test_grid_load_and_resample_from_cpp(grid_driver, tmp_path):
    import numpy as np
    from oracle import grid_io as O
    r = subprocess.run([grid_driver, "load", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(str(tmp_path / "resampled.bin"), dtype=np.float64).reshape(7, 9, 11, 1)
    assert np.array_equal(got, O.interpolate_to(_driver_grid(), 11, 9, 7))


@pytest.mark.gpu
def test_driver_diagnostics(driver, tmp_path):
    # viewIterates and the Ritz-value printout through psp.hpp
    r = subprocess.run([driver, "30", "15", "0", "20", "1e-5", "3"], capture_output=True, text=True,
                       cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    its = int(r.stdout.split("iterations ")[1].split()[0])
    for it in range(its - 1):
        for rhs in range(2):
            for part in ("real", "imag"):
                stem = tmp_path / ("iterates-%d_%d_%s" % (it, rhs, part))
                assert (tmp_path / (stem.name + ".pvti")).exists() and (stem / "0.vti").exists()
    assert not (tmp_path / ("iterates-%d_0_real.pvti" % (its - 1))).exists()
    lines = r.stdout.splitlines()
    for rhs in range(2):
        i = lines.index("Ritz values for %d'th right-hand side before first restart:" % rhs)
        assert len(lines[i + 1].split()) == min(its, 20)
