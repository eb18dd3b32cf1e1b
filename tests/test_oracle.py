"""The FP64 CPU oracle against independent restatements and direct solves.

The reference ships no golden vectors for this path (its numerical core,
Clique, is absent), so the oracle is pinned by: the global operator rebuilt
independently from the reference formulas, every panel solve against a
sparse LU of the padded panel subproblem, and the GMRES result against a
sparse direct solve of the global operator.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import helmholtz_np as hnp
from conftest import oracle_for, rel
from psp_b200 import DIRICHLET, workloads as W


CASES = [
    dict(interior=(12, 13, 14), pml=5, freq=2.0, k=3, seed=7, top_pml=True),
    dict(interior=(11, 9, 12), pml=4, freq=1.5, k=2, seed=11, top_pml=False),
]


@pytest.fixture(scope="module", params=range(len(CASES)))
def case(request):
    w = W.small_case(**CASES[request.param])
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    return w, O


def test_global_operator_matches_independent_restatement(case):
    w, O = case
    A = O.global_operator_natural()
    A_np = hnp.global_matrix(w.disc, w.velocity)
    assert abs(A - A_np).max() <= 1e-9 * abs(A_np).max()


def test_global_operator_is_complex_symmetric(case):
    _, O = case
    A = O.global_operator_natural()
    assert abs(A - A.T).max() == 0.0


def test_nd_order_is_a_permutation(case):
    w, O = case
    perm = O.nd_to_natural()
    assert np.array_equal(np.sort(perm), np.arange(perm.size))


def test_panel_solves_match_sparse_lu(case):
    w, O = case
    rng = np.random.default_rng(3)
    B = rng.standard_normal(w.rhs.shape) + 1j * rng.standard_normal(w.rhs.shape)
    for p, (low_v, depth, padding, _) in enumerate(O.geometry()):
        got = O.solve_panel(B, p)
        want = hnp.apply_panel_inverse(w.disc, w.velocity, B, low_v, depth, padding, 7.0)
        assert rel(got, want) < 1e-10, p


def test_gmres_converges_to_direct_solution(case):
    w, O = case
    X, st = O.solve(w.rhs, 20, 1e-10)
    assert st["converged"]
    A = O.global_operator_natural().tocsc()
    lu = spla.splu(A)
    Xd = np.stack([lu.solve(w.rhs[..., r].ravel()) for r in range(w.k)], -1)
    assert rel(X.reshape(-1, w.k), Xd) < 1e-8


def test_preconditioner_is_a_good_approximate_inverse(case):
    w, O = case
    MB = O.precondition(w.rhs)
    AMB = O.multiply(MB)
    # the moving-PML sweep approximates A^{-1}: ||b - A M^{-1} b|| < ||b||
    assert rel(AMB, w.rhs) < 0.9


def test_shallow_domain_is_a_logic_error():
    import oracle
    d = oracle.make_disc(10.0, 20, 20, 18, 1.0, 1.0, 1.0, pml=(5, 5, 5))
    with pytest.raises(ValueError, match="shallow"):
        oracle.Oracle(d)


def test_zero_rhs_raises_nan_error():
    w = W.small_case(**CASES[0])
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    with pytest.raises(RuntimeError, match="NaN"):
        O.solve(np.zeros_like(w.rhs), 20, 1e-4)


def test_golden_fixture_reproduced():
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "small_fp64.npz")
    g = np.load(path)
    w = W.small_case(**{k: (tuple(v) if k == "interior" else v.item()) for k, v in
                        ((k, g["cfg_" + k]) for k in ("interior", "pml", "freq", "k", "seed", "top_pml"))})
    assert np.array_equal(w.velocity, g["velocity"])
    assert np.array_equal(w.rhs, g["rhs"])
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    assert rel(O.precondition(w.rhs), g["precondition"]) < 1e-12
    X, st = O.solve(w.rhs, 20, float(g["rel_tol"]))
    assert st["iterations"] == int(g["iterations"])
    assert rel(X, g["solution"]) < 1e-10
