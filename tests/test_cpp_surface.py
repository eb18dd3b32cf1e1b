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
