"""The reference's own Solve against the oracle's (CPU).

oracle/_ref/libpspref.so runs psp::DistHelmholtz::Solve of the reference
(solve.hpp:12-611, compiled unchanged on one process; oracle/refshim): its
right-hand-side pull and push, its GMRES(m) with Givens updates and its
sweeping preconditioner (panel solves, sub- and superdiagonal couplings,
solve.hpp:681-1061) around its own global rows and Multiply.  Only
Clique's multifrontal panel factorization and solve, which are not in the
reference tree, come from the oracle (whose panel solves equal sparse LU
solves of the padded panel matrices, tests/test_oracle.py).  The oracle's
restatement of everything else must then take the same GMRES steps and
give the same wavefields.  Skipped where the reference tree was not
available to build the library.
"""
import os

import numpy as np
import pytest

from conftest import oracle_for, rel
from oracle import ref
from psp_b200 import workloads as W

pytestmark = pytest.mark.skipif(
    not (ref.available() or os.path.isdir(os.path.join(ref.REF_TREE, "include", "psp"))),
    reason="the reference's DistHelmholtz is not built here")

CASES = {
    "small": dict(),
    "uneven_leftover": dict(interior=(12, 13, 14), pml=5, freq=2.0, k=3, seed=7, top_pml=True),
    "dirichlet_top": dict(interior=(11, 9, 12), pml=4, freq=1.5, k=2, seed=11, top_pml=False),
    "seventeen_rhs": dict(interior=(9, 10, 11), pml=4, freq=1.5, k=17, seed=4, top_pml=True),
}


def _workload(name):
    if name == "layered":
        return W.CONFIGS["layered_faults_24"]()
    return W.small_case(**CASES[name])


@pytest.mark.parametrize("name", list(CASES) + ["layered"])
@pytest.mark.parametrize("tol", [1e-4, 1e-7])
def test_reference_solve_matches_oracle(name, tol):
    w = _workload(name)
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    Xo, sto = O.solve(w.rhs, 20, tol)
    R = ref.RefHelmholtz(w.disc)
    Xr, log, its = R.solve(w.velocity, O, w.rhs, 20, tol)
    assert "converged with relative tolerance" in log
    assert its == sto["iterations"]
    assert rel(Xr, Xo) < 1e-12


def test_reference_solve_restarts_like_oracle():
    """GMRES(5): several restart cycles, each restarting from the iterate."""
    w = _workload("uneven_leftover")
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    Xo, sto = O.solve(w.rhs, 5, 1e-7)
    Xr, log, its = ref.RefHelmholtz(w.disc).solve(w.velocity, O, w.rhs, 5, 1e-7)
    assert sto["iterations"] > 5 and its == sto["iterations"]
    assert log.count("starting iteration") == -(-its // 5)
    assert rel(Xr, Xo) < 1e-12


@pytest.mark.parametrize("name", list(CASES) + ["layered"])
def test_reference_operators_match_oracle(name):
    """Row by row of the scope table: the reference's own Multiply (A10),
    Precondition (A9: panel solves with the sub- and superdiagonal
    couplings, around the oracle's panel solves) and SolvePanel of every
    panel (A8's data movement: node layout, padding rows), each between its
    own PullRightHandSides and PushRightHandSides (A12), equal the oracle's
    operators."""
    w = _workload(name)
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    R = ref.RefHelmholtz(w.disc)
    assert rel(R.apply(w.velocity, O, w.rhs, "multiply"), O.multiply(w.rhs)) < 1e-14
    assert rel(R.apply(w.velocity, O, w.rhs, "precondition"), O.precondition(w.rhs)) < 1e-13
    for p in range(O.geometry().shape[0]):
        assert rel(R.apply(w.velocity, O, w.rhs, "panel", p), O.solve_panel(w.rhs, p)) < 1e-14, p
