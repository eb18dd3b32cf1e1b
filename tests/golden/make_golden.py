"""Regenerates the golden fixtures of tests/golden from the FP64 oracle.

    python tests/golden/make_golden.py

small_fp64.npz: a seeded small workload (psp_b200.workloads.small_case with
the cfg_* parameters stored in the file), one application of the sweeping
preconditioner and the GMRES(20) solution at relative tolerance 1e-8, with
its inner-step count.  The oracle itself is pinned against sparse direct
solves in tests/test_oracle.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from psp_b200 import workloads as W  # noqa: E402

CFG = dict(interior=(8, 9, 10), pml=4, freq=1.5, k=2, seed=5, top_pml=True)
REL_TOL = 1e-8


def main():
    w = W.small_case(**CFG)
    d = w.disc
    od = oracle.make_disc(d.omega, d.nx, d.ny, d.nz, d.wx, d.wy, d.wz,
                          bcs=(d.frontBC, d.rightBC, d.backBC, d.leftBC, d.topBC),
                          pml=(d.bx, d.by, d.bz), sigma=d.sigmax)
    O = oracle.Oracle(od)
    O.initialize(w.velocity)
    pre = O.precondition(w.rhs)
    X, st = O.solve(w.rhs, 20, REL_TOL)
    assert st["converged"]
    out = {"cfg_" + k: np.asarray(v) for k, v in CFG.items()}
    out.update(velocity=w.velocity, rhs=w.rhs, precondition=pre, solution=X,
               iterations=np.asarray(st["iterations"]), rel_tol=np.asarray(REL_TOL))
    np.savez_compressed(os.path.join(HERE, "small_fp64.npz"), **out)
    print("wrote small_fp64.npz, iterations", st["iterations"])


if __name__ == "__main__":
    main()
