"""The reference's own DistHelmholtz members against the oracle and the
product (CPU).

oracle/_ref/libpspref.so holds include/psp/dist_helmholtz.hpp of the
reference compiled unchanged on one process against stand-ins for Clique
and Elemental (oracle/refshim): its constructor builds the panel geometry,
the global nested-dissection order and the elimination tree of every panel
class exactly as the reference does, and its FormGlobalRow and PML stretches
run as written.  Clique's symbolic analysis, factorization and solves are
not part of the reference tree and stay unpinned; the fill structure is
checked as the textbook closure of the reference's own trees (a node's
structure is its original lower structure plus its children's structures
minus its own pivots, which is what Clique's SymmetricAnalysis computes).
Skipped where the reference tree was not available to build the library.
"""
import os

import numpy as np
import pytest

import oracle
import psp_b200 as P
from oracle import ref
from psp_b200 import workloads as W

pytestmark = pytest.mark.skipif(
    not (ref.available() or os.path.isdir(os.path.join(ref.REF_TREE, "include", "psp"))),
    reason="the reference's DistHelmholtz is not built here")

SHAPES = [
    # (nx, ny, nz, pml, planesPerPanel, cutoff, topBC)
    (22, 25, 23, 5, 4, 12, P.PML),
    (31, 17, 26, 5, 3, 12, P.PML),
    (20, 20, 21, 4, 4, 12, P.DIRICHLET),
    (19, 27, 30, 5, 4, 20, P.PML),
    (50, 50, 50, 5, 4, 12, P.PML),
]


def _cases(shape):
    nx, ny, nz, b, planes, cutoff, top = shape
    bcs = (P.PML, P.PML, P.PML, P.PML, top)
    d = P.Discretization(9.0, nx, ny, nz, 1.0, 1.1, 1.2, bcs=bcs, pml=(b, b, b), sigma=1.5)
    od = oracle.make_disc(9.0, nx, ny, nz, 1.0, 1.1, 1.2, bcs=bcs, pml=(b, b, b), sigma=1.5)
    return d, oracle.Oracle(od, 7.0, planes, cutoff), ref.RefHelmholtz(d, 7.0, planes, cutoff), planes, cutoff


def _fill_sizes(info, lower):
    """Lower-structure sizes after the textbook symbolic factorization of
    the reference's tree (nodes in postorder)."""
    struct = [set(map(int, l)) for l in lower]
    for t in range(len(struct)):
        p = info[t, 2]
        if p >= 0:
            lo, hi = info[p, 0], info[p, 0] + info[p, 1]
            struct[p] |= {i for i in struct[t] if not lo <= i < hi}
    return np.array([len(s) for s in struct])


@pytest.mark.parametrize("shape", SHAPES)
def test_geometry_order_and_trees_match_reference(product_lib, shape):
    d, O, R, planes, cutoff = _cases(shape)
    geo = R.geometry()
    assert np.array_equal(geo, O.geometry()[:, :3])
    assert np.array_equal(geo, P.panel_geometry(d, planes)[:, :3])
    # the global nested-dissection order of the rows
    assert np.array_equal(R.local_to_natural(), O.nd_to_natural())
    # one elimination tree per panel class, as the product analyses it
    classes = sorted(set(O.geometry()[:, 3].tolist()))
    assert len(R.trees) == len(classes)
    for c, (info, lower) in zip(classes, R.trees):
        mine, _ = P.analyze_class(d, planes, cutoff, c)
        assert np.array_equal(info[:, 0], mine[:, 0]), c      # ND offsets
        assert np.array_equal(info[:, 1], mine[:, 1]), c      # pivot counts
        assert np.array_equal(info[:, 2], mine[:, 3]), c      # parents
        assert np.array_equal(_fill_sizes(info, lower), mine[:, 2]), c  # update sizes after fill
        assert np.array_equal(mine, O.tree(c)), c


@pytest.mark.parametrize("shape", SHAPES[:4])
def test_pml_stretches_match_reference(shape):
    d, O, R, _, _ = _cases(shape)
    for which, n in ((1, d.nx), (2, d.ny), (3, d.nz)):
        idx = np.arange(-1, n + 1)
        assert np.array_equal(R.stretch(which, idx), O.stretch(which, idx)), which
    idx = np.arange(-1, d.nz + 1)
    for v_offset in sorted(set(O.geometry()[:, 0].tolist())):
        assert np.array_equal(R.stretch(4, idx, v_offset), O.stretch(4, idx, v_offset)), v_offset


@pytest.mark.parametrize("name", ["small", "layered"])
def test_global_rows_match_reference(name):
    w = W.small_case() if name == "small" else W.CONFIGS["layered_faults_24"]()
    d = w.disc
    R = ref.RefHelmholtz(d)
    O = oracle.Oracle(oracle.make_disc(d.omega, d.nx, d.ny, d.nz, d.wx, d.wy, d.wz,
                                       bcs=(d.frontBC, d.rightBC, d.backBC, d.leftBC, d.topBC),
                                       pml=(d.bx, d.by, d.bz), sigma=d.sigmax))
    A = R.global_operator_natural(w.velocity)
    O.form_operator(w.velocity)
    B = O.global_operator_natural()
    assert A.nnz == B.nnz
    # the same formulas; the oracle's compiler may contract a multiply-add
    assert abs(A - B).max() <= 1e-14 * abs(B).max()


@pytest.mark.parametrize("name", ["small", "dirichlet_top", "layered"])
def test_panel_fronts_match_reference(name):
    """Every node of every panel, as the reference's Initialize fills it
    (GetPanelVelocity and FillPanelFronts with FormLowerColumnOfNode:
    damped frequency, artificial PML below the panel, the panel's velocity
    window), before any update: equal to the oracle's assembled fronts,
    whose panel factorization the product's panel solves match."""
    if name == "layered":
        w = W.CONFIGS["layered_faults_24"]()
    elif name == "dirichlet_top":
        w = W.small_case(interior=(11, 9, 12), pml=4, freq=1.5, k=2, seed=11, top_pml=False)
    else:
        w = W.small_case()
    d = w.disc
    R = ref.RefHelmholtz(d)
    O = oracle.Oracle(oracle.make_disc(d.omega, d.nx, d.ny, d.nz, d.wx, d.wy, d.wz,
                                       bcs=(d.frontBC, d.rightBC, d.backBC, d.leftBC, d.topBC),
                                       pml=(d.bx, d.by, d.bz), sigma=d.sigmax))
    geo = O.geometry()
    for p in range(geo.shape[0]):
        for t in range(O.tree(geo[p, 3]).shape[0]):
            a, b = R.panel_front(w.velocity, p, t), O.panel_front(w.velocity, p, t)
            assert a.shape == b.shape, (p, t)
            assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max(), (p, t)
