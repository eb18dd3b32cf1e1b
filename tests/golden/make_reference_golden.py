"""Regenerates tests/golden/reference_dirichlet_top.npz from the reference's
own code.

    make -C oracle ref            # oracle/_ref/libpspref.so from the reference tree
    python tests/golden/make_reference_golden.py

The library is the reference's psp::DistHelmholtz (include/psp/
dist_helmholtz.hpp and dist_helmholtz/*.hpp) compiled unchanged on one
process against the Clique/Elemental stand-in of oracle/refshim.  On a
seeded small workload with a Dirichlet top face (psp_b200.workloads.small_case
with the cfg_* parameters stored in the file) the fixture holds what the
reference computes:

* multiply: its Multiply (solve.hpp:613-679) over its own FormGlobalRow rows
  (initialize_finalize.hpp:527-587), between its PullRightHandSides and
  PushRightHandSides (solve.hpp:58-239);
* precondition: its Precondition (solve.hpp:681-734), the sweep with its
  sub- and superdiagonal couplings (solve.hpp:884-1061);
* solution / iterations / log: its Solve (solve.hpp:12-611), GMRES(20) at
  relative tolerance 1e-8, its step count and what it printed.

Clique is not part of the reference tree, so the panel factorizations and
panel solves inside the sweep are the oracle's (equal to sparse LU solves of
the padded panel matrices, tests/test_oracle.py); every other step is the
reference's.  The fixture travels with the tests, so the oracle and the CUDA
path are checked against the reference's outputs where the reference tree is
absent.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import ref  # noqa: E402
from psp_b200 import workloads as W  # noqa: E402

CFG = dict(interior=(11, 9, 12), pml=4, freq=1.5, k=2, seed=11, top_pml=False)
REL_TOL = 1e-8
NAME = "reference_dirichlet_top.npz"


def main():
    w = W.small_case(**CFG)
    d = w.disc
    od = oracle.make_disc(d.omega, d.nx, d.ny, d.nz, d.wx, d.wy, d.wz,
                          bcs=(d.frontBC, d.rightBC, d.backBC, d.leftBC, d.topBC),
                          pml=(d.bx, d.by, d.bz), sigma=d.sigmax)
    O = oracle.Oracle(od)
    O.initialize(w.velocity)
    R = ref.RefHelmholtz(d)
    mult = R.apply(w.velocity, O, w.rhs, "multiply")
    pre = R.apply(w.velocity, O, w.rhs, "precondition")
    X, log, its = R.solve(w.velocity, O, w.rhs, 20, REL_TOL)
    if "converged with relative tolerance" not in log:
        raise RuntimeError("the reference's Solve did not converge:\n" + log)
    out = {"cfg_" + k: np.asarray(v) for k, v in CFG.items()}
    out.update(velocity=w.velocity, rhs=w.rhs, multiply=mult, precondition=pre, solution=X,
               iterations=np.asarray(its), rel_tol=np.asarray(REL_TOL), log=np.asarray(log))
    np.savez_compressed(os.path.join(HERE, NAME), **out)
    print("wrote", NAME, "iterations", its)


if __name__ == "__main__":
    main()
