"""GMRES diagnostics of Solve: viewIterates (solve.hpp:579-585) and the
PRINT_RITZ_VALUES Ritz values of the first restart cycle (solve.hpp:257-261,
391-395, 422-426, 589-608).

The Hessenberg eigenvalue routine (the counterpart of Elemental's
lapack::HessenbergEig) is checked against numpy's LAPACK on the host; the
oracle's recorded first-cycle Hessenberg matrices against a numpy Arnoldi
process over the oracle's own operator and sweep; on the GPU, the Ritz
values of the CUDA path against the eigenvalues of the oracle's matrices
and the iterate volumes against the writer restatement.
"""
import os
import re

import numpy as np
import pytest

import psp_b200 as P
from conftest import oracle_for
from psp_b200 import workloads as W

CASE = dict(interior=(12, 13, 14), pml=5, freq=2.0, k=3, seed=7, top_pml=True)


def match_error(got, want):
    """Largest distance between paired eigenvalues (greedy nearest pairing)."""
    want = list(want)
    assert len(got) == len(want)
    err = 0.0
    for g in got:
        i = int(np.argmin([abs(g - w) for w in want]))
        err = max(err, abs(g - want.pop(i)))
    return err


# ---------------------------------------------------------------- host


@pytest.mark.parametrize("n", [1, 2, 3, 7, 20, 64])
def test_hessenberg_eigenvalues_match_lapack(product_lib, n):
    rng = np.random.default_rng(n)
    H = np.triu(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)), -1)
    want = np.linalg.eigvals(H)
    assert match_error(P.hessenberg_eigenvalues(H), want) <= 1e-12 * max(1.0, abs(want).max()) * n


def test_hessenberg_eigenvalues_special_matrices(product_lib):
    rot = np.array([[0.0, -1.0], [1.0, 0.0]])
    assert match_error(P.hessenberg_eigenvalues(rot), [1j, -1j]) < 1e-15
    # already triangular (every subdiagonal deflates at once)
    T = np.triu(np.arange(1, 26).reshape(5, 5) * (1 + 0.5j))
    assert match_error(P.hessenberg_eigenvalues(T), np.diag(T)) == 0.0
    # a defective eigenvalue and the zero matrix
    J = 2 * np.eye(5) + np.diag(np.ones(4), -1)
    assert match_error(P.hessenberg_eigenvalues(J), [2] * 5) < 1e-3
    assert np.array_equal(P.hessenberg_eigenvalues(np.zeros((4, 4))), np.zeros(4))
    assert P.hessenberg_eigenvalues(np.zeros((0, 0))).size == 0
    # entries below the first subdiagonal are ignored
    rng = np.random.default_rng(5)
    A = rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))
    assert match_error(P.hessenberg_eigenvalues(A), np.linalg.eigvals(np.triu(A, -1))) < 1e-12
    # a block that splits in two (zero subdiagonal in the middle)
    B = np.triu(A, -1)
    B[3, 2] = 0
    assert match_error(P.hessenberg_eigenvalues(B), np.linalg.eigvals(B)) < 1e-12


def test_hessenberg_eigenvalues_at_extreme_scales(product_lib):
    # the routine works on H scaled by a power of two, so the eigenvalues of
    # 2^e H are exactly 2^e times those of H, far beyond where unscaled
    # shift products would overflow or underflow
    rng = np.random.default_rng(11)
    H = np.triu(rng.standard_normal((17, 17)) + 1j * rng.standard_normal((17, 17)), -1)
    w = P.hessenberg_eigenvalues(H)
    for e in (-900, -600, 600, 900):
        assert np.array_equal(P.hessenberg_eigenvalues(H * 2.0 ** e), w * 2.0 ** e), e
    # tiny subdiagonal entries beside unit-size ones deflate
    T = np.triu(rng.standard_normal((6, 6)) + 0j, -1)
    T[3, 2] = 1e-300
    assert match_error(P.hessenberg_eigenvalues(T), np.linalg.eigvals(T)) < 1e-12


def test_hessenberg_eigenvalues_errors(product_lib):
    import ctypes
    H = np.zeros(8)
    w = np.zeros(4)
    dp = ctypes.POINTER(ctypes.c_double)
    # ldh < n
    assert P.lib().psp_cu_hessenberg_eigenvalues(2, H.ctypes.data_as(dp), 1, w.ctypes.data_as(dp)) == 1
    assert P.lib().psp_cu_hessenberg_eigenvalues(-1, None, 1, None) == 1
    with pytest.raises(P.PspRuntimeError, match="non-finite"):
        P.hessenberg_eigenvalues(np.array([[np.nan, 1.0], [1.0, 0.0]]))
    with pytest.raises(P.LogicError):
        P.hessenberg_eigenvalues(np.zeros((2, 3)))


def _arnoldi(O, b, steps):
    """Unrotated Hessenberg matrices of the left-preconditioned Arnoldi
    process of GMRES from x0 = 0 (solve.hpp:329-396), per right-hand side,
    by numpy modified Gram-Schmidt over O.multiply and O.precondition."""
    N, k = b.shape
    w = O.precondition(b).reshape(N, k)
    Hs = []
    for r in range(k):
        V = [w[:, r] / np.linalg.norm(w[:, r])]
        H = np.zeros((steps, steps), dtype=np.complex128)
        for j in range(steps):
            x = np.zeros((N, k), dtype=np.complex128)
            x[:, r] = V[j]
            u = O.precondition(O.multiply(x)).reshape(N, k)[:, r]
            for i in range(j + 1):
                H[i, j] = np.vdot(V[i], u)
                u = u - H[i, j] * V[i]
            d = np.linalg.norm(u)
            if j + 1 < steps:
                H[j + 1, j] = d
            V.append(u / d)
        Hs.append(H)
    return np.array(Hs)


def test_oracle_first_cycle_hessenberg_is_arnoldi():
    import oracle
    w = W.small_case(**CASE)
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    b = w.rhs.reshape(-1, w.k)
    O.solve(b, m=8, rel_tol=1e-14, max_its=5)
    H = oracle.first_cycle_hessenberg(O)
    assert H.shape == (w.k, 5, 5)
    assert np.all(np.tril(H, -2) == 0)
    want = _arnoldi(O, b, 5)
    assert np.abs(H - want).max() <= 1e-9 * np.abs(want).max()
    # a cycle that converges early records only its steps
    _, st = O.solve(b, m=20, rel_tol=1e-3)
    assert oracle.first_cycle_hessenberg(O).shape == (w.k, st["iterations"], st["iterations"])
    # with restarts only the first cycle is kept: its m steps, whose last
    # subdiagonal entry (outside the m x m block) is never stored
    _, st = O.solve(b, m=3, rel_tol=1e-6)
    assert st["iterations"] > 3
    H3 = oracle.first_cycle_hessenberg(O)
    assert H3.shape == (w.k, 3, 3)
    assert np.abs(H3 - want[:, :3, :3]).max() <= 1e-9 * np.abs(want).max()


# ---------------------------------------------------------------- GPU


@pytest.fixture(scope="module")
def problem(product_lib):
    w = W.small_case(**CASE)
    O = oracle_for(w.disc)
    O.initialize(w.velocity)
    H = P.DistHelmholtz(w.disc)
    H.Initialize(w.velocity_grid(), precision=P.FP64)
    return w, O, H


def _oracle_ritz(O):
    import oracle
    return [np.linalg.eigvals(h) for h in oracle.first_cycle_hessenberg(O)]


@pytest.mark.gpu
@pytest.mark.parametrize("m,rel_tol,max_its", [(8, 1e-14, 5), (20, 1e-6, 0), (3, 1e-6, 0)])
def test_ritz_values_match_oracle(problem, m, rel_tol, max_its):
    w, O, H = problem
    b = w.rhs.reshape(-1, w.k)
    X, sto = O.solve(b, m=m, rel_tol=rel_tol, max_its=max_its)
    want = _oracle_ritz(O)
    H.SetRitzValues(1)
    H.set_max_iterations(max_its)
    try:
        g = np.ascontiguousarray(b.copy())
        st = H.Solve(g, m, rel_tol)
    finally:
        H.set_max_iterations(0)
        H.SetRitzValues(0)
    assert st["iterations"] == sto["iterations"]
    got = H.RitzValues()
    assert got.shape == (w.k, len(want[0])) == (w.k, min(m, st["iterations"]))
    for r in range(w.k):
        assert match_error(got[r], want[r]) <= 1e-9 * abs(want[r]).max(), r


@pytest.mark.gpu
def test_ritz_values_printed_like_the_reference(problem, capfd):
    w, _, H = problem
    H.SetRitzValues(2)
    try:
        st = H.Solve(np.ascontiguousarray(w.rhs.reshape(-1, w.k).copy()), 20, 1e-6)
    finally:
        H.SetRitzValues(0)
    out = capfd.readouterr().out.splitlines()
    got = H.RitzValues()
    for r in range(w.k):
        i = out.index("Ritz values for %d'th right-hand side before first restart:" % r)
        vals = [complex(float(a), float(b)) for a, b in re.findall(r"\(([^,]+),([^)]+)\)", out[i + 1])]
        assert len(vals) == min(20, st["iterations"])
        assert np.allclose(vals, got[r], rtol=1e-5, atol=1e-6 * abs(got[r]).max())
    # mode 0: the next Solve records nothing
    H.Solve(np.ascontiguousarray(w.rhs.reshape(-1, w.k).copy()), 20, 1e-6)
    assert H.RitzValues().size == 0


def _numbers(text):
    body = text.split('format="ascii">\n', 1)[1].split("</DataArray>", 1)[0]
    return np.array([float(v) for v in body.split()])


@pytest.mark.gpu
def test_view_iterates_writes_each_unconverged_step(problem, tmp_path):
    from oracle import grid_io as G
    w, _, H = problem
    d = w.disc
    base = str(tmp_path / "iterates")
    g = np.ascontiguousarray(w.rhs.reshape(-1, w.k).copy())
    st = H.Solve(g, 20, 1e-6, viewIterates=base)
    its = st["iterations"]
    assert st["converged"] and its >= 3
    names = sorted(os.listdir(tmp_path))
    assert len([n for n in names if n.endswith(".pvti")]) == (its - 1) * w.k * 2
    assert not os.path.exists(base + "-%d_0_real.pvti" % (its - 1))
    # iterate 1 is the solution after two inner steps
    H.set_max_iterations(2)
    try:
        x2 = np.ascontiguousarray(w.rhs.reshape(-1, w.k).copy())
        H.Solve(x2, 20, 1e-6)
    finally:
        H.set_max_iterations(0)
    want = G.volume_texts(x2.reshape(d.nz, d.ny, d.nx, w.k), base + "-1")
    for name, text in want.items():
        got = open(name).read()
        if name.endswith(".pvti"):
            assert got == text
        else:
            a, b = _numbers(got), _numbers(text)
            assert a.shape == b.shape and np.allclose(a, b, rtol=2e-6, atol=1e-300)
    # switched off after the call
    H.Solve(np.ascontiguousarray(w.rhs.reshape(-1, w.k).copy()), 20, 1e-6)
    assert len(os.listdir(tmp_path)) == len(names)
