"""Host-side symbolic analysis of the product against the oracle's
restatement of PSP's nested dissection (main.hpp:1423-1477, 1709-1900) and
Clique's fill structure; runs without a GPU."""
import numpy as np
import pytest

import oracle
import psp_b200 as P

SHAPES = [
    # (nx, ny, nz, pml, planesPerPanel, cutoff, topBC)
    (22, 25, 23, 5, 4, 12, P.PML),
    (31, 17, 26, 5, 3, 12, P.PML),
    (20, 20, 21, 4, 4, 12, P.DIRICHLET),
    (19, 27, 30, 5, 4, 20, P.PML),
    (50, 50, 50, 5, 4, 12, P.PML),
]


@pytest.mark.parametrize("shape", SHAPES)
def test_trees_and_orderings_match_oracle(product_lib, shape):
    nx, ny, nz, b, planes, cutoff, top = shape
    bcs = (P.PML, P.PML, P.PML, P.PML, top)
    d = P.Discretization(9.0, nx, ny, nz, 1.0, 1.1, 1.2, bcs=bcs, pml=(b, b, b), sigma=1.5)
    od = oracle.make_disc(9.0, nx, ny, nz, 1.0, 1.1, 1.2, bcs=bcs, pml=(b, b, b), sigma=1.5)
    O = oracle.Oracle(od, 7.0, planes, cutoff)
    classes = sorted(set(O.geometry()[:, 3].tolist()))
    for c in classes:
        info, nd = P.analyze_class(d, planes, cutoff, c)
        assert np.array_equal(info, O.tree(c)), c
        # ND -> panel-natural map is a bijection and ND offsets tile [0, nSub)
        assert np.array_equal(np.sort(nd), np.arange(nd.size))
        assert info[0, 0] == 0
        assert np.array_equal(info[1:, 0], np.cumsum(info[:-1, 1]))
        assert info[:, 1].sum() == nd.size
        # postorder: parents come after children, exactly one root
        parents = info[:, 3]
        assert (parents == -1).sum() == 1
        assert all(p > i for i, p in enumerate(parents) if p >= 0)


def test_panel_geometry_matches_oracle(product_lib):
    for nz, planes, top in [(30, 4, P.PML), (31, 3, P.PML), (25, 4, P.DIRICHLET)]:
        bcs = (P.PML,) * 4 + (top,)
        od = oracle.make_disc(9.0, 20, 20, nz, 1.0, 1.0, 1.0, bcs=bcs, pml=(5, 5, 5))
        O = oracle.Oracle(od, 7.0, planes, 12)
        geo = O.geometry()
        # panels cover the sweep direction once, bottom panel unpadded
        assert geo[0, 0] == 0 and geo[0, 2] == 0
        assert (geo[1:, 2] == 5).all()
        assert np.array_equal(geo[1:, 0], geo[:-1, 0] + geo[:-1, 1])
        assert geo[-1, 0] + geo[-1, 1] == nz


def test_shallow_domain_rejected_without_gpu(product_lib):
    d = P.Discretization(10.0, 20, 20, 18, 1.0, 1.0, 1.0, pml=(5, 5, 5))
    with pytest.raises(P.LogicError, match="shallow"):
        P.analyze_class(d, 4, 12, 0)
    with pytest.raises(P.LogicError, match="shallow"):
        P.DistHelmholtz(d)
