"""The oracle against outputs of the reference's own code (CPU).

tests/golden/reference_dirichlet_top.npz was written by
tests/golden/make_reference_golden.py from the reference's psp::DistHelmholtz
compiled unchanged on one process (oracle/_ref, oracle/refshim): its
Multiply over its own global rows, its Precondition and its Solve (GMRES(20)
at 1e-8) on a seeded workload with a Dirichlet top face, around the oracle's
panel solves (Clique is not in the reference tree).  The fixture travels with
the tests, so these checks need neither the reference tree nor its library.
"""
import os

import numpy as np
import pytest

from conftest import oracle_for, rel
from oracle import ref
from psp_b200 import workloads as W

PATH = os.path.join(os.path.dirname(__file__), "golden", "reference_dirichlet_top.npz")
KEYS = ("interior", "pml", "freq", "k", "seed", "top_pml")


def load_fixture(path=PATH):
    """(fixture arrays, the workload they were made on)."""
    g = np.load(path)
    cfg = {k: (tuple(int(v) for v in g["cfg_" + k]) if k == "interior" else g["cfg_" + k].item()) for k in KEYS}
    return g, W.small_case(**cfg)


@pytest.fixture(scope="module")
def fixture():
    g, w = load_fixture()
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    return g, w, O


def test_fixture_inputs_are_the_seeded_workload(fixture):
    g, w, _ = fixture
    assert np.array_equal(w.velocity, g["velocity"])
    assert np.array_equal(w.rhs, g["rhs"])


def test_oracle_operators_match_reference_outputs(fixture):
    g, w, O = fixture
    assert rel(O.multiply(w.rhs), g["multiply"]) < 1e-14
    assert rel(O.precondition(w.rhs), g["precondition"]) < 1e-14


def test_oracle_solve_matches_reference_solve(fixture):
    g, w, O = fixture
    X, st = O.solve(w.rhs, 20, float(g["rel_tol"]))
    assert st["converged"]
    # several restart cycles of GMRES(20), the same steps as the reference
    assert st["iterations"] == int(g["iterations"]) > 40
    assert rel(X, g["solution"]) < 1e-12
    log = str(g["log"])
    assert log.count("starting iteration") == -(-st["iterations"] // 20)
    assert "converged with relative tolerance" in log


@pytest.mark.skipif(not ref.available(), reason="the reference's DistHelmholtz is not built here")
def test_reference_reproduces_fixture(fixture):
    """The fixture is current: the reference's Solve gives it again, bit
    for bit."""
    g, w, O = fixture
    X, _, its = ref.RefHelmholtz(w.disc).solve(w.velocity, O, w.rhs, 20, float(g["rel_tol"]))
    assert its == int(g["iterations"])
    assert np.array_equal(X, g["solution"])
