"""Host-side constraint set-up of the mirror (constraints.ts:23-52,
constraintSet.ts:64-120, 333-344) against the oracle, on CPU."""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as O
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F


def curves():
    yield F.trefoil(128, jitter=0.01, seed=1)
    yield F.random_walk_knot(256, seed=2)
    v, e = F.trefoil(64, jitter=0.0, seed=3)
    yield v, e[:40]  # an open polyline: edges do not cover every vertex


@pytest.mark.parametrize("i", range(3))
def test_targets_match_the_oracle(i):
    v, e = list(curves())[i]
    x0 = T.barycenterTarget(v, e)
    assert np.allclose(x0, O.barycenter_target(v, e), rtol=0, atol=1e-14 * max(1.0, np.abs(x0).max()))
    L = T.totalLength(v, e)
    assert abs(L - O.total_length(v, e)) <= 1e-14 * L
    ell = T.edgeLengths(v, e)
    assert np.allclose(ell, O.edge_lengths(v, e), rtol=1e-15, atol=0)


def test_degenerate_curve_barycenter_is_the_vertex_mean():
    v = np.zeros((4, 3))
    v[:, 0] = 1.0
    e = np.array([[0, 1], [1, 2], [2, 3], [3, 0]], dtype=np.int32)
    assert np.array_equal(T.barycenterTarget(v, e), O.barycenter_target(v, e))
    assert np.array_equal(T.barycenterTarget(v, e), np.array([1.0, 0.0, 0.0]))


def test_total_and_edge_lengths_are_mutually_exclusive():
    v, e = F.trefoil(16, jitter=0.0, seed=4)
    T.assertValidConstraintSet([T.barycenterBlock([0, 0, 0]), T.totalLengthBlock(1.0)])
    T.assertValidConstraintSet([T.edgeLengthsBlock(T.edgeLengths(v, e)), T.pointBlock(0, v[0])])
    with pytest.raises(ValueError, match="mutually exclusive"):
        T.assertValidConstraintSet([T.totalLengthBlock(1.0), T.edgeLengthsBlock(T.edgeLengths(v, e))])


def _oracle_pairs(e):
    import ctypes as C
    from repulsive_test2_b200 import abi
    e = np.ascontiguousarray(np.asarray(e, dtype=np.int32))
    E = len(e)
    n = O.lib().tpeo_disjoint_pairs(e.ctypes.data_as(abi.ip), E, None, None, 0)
    off = np.zeros(E + 1, dtype=np.int32)
    part = np.zeros(max(n, 1), dtype=np.int32)
    O.lib().tpeo_disjoint_pairs(e.ctypes.data_as(abi.ip), E, off.ctypes.data_as(abi.ip),
                                part.ctypes.data_as(abi.ip), n)
    return [part[off[i]:off[i + 1]].tolist() for i in range(E)]


def test_disjoint_pairs_listing_matches_the_oracle():
    """tangentPointEnergy.ts:33-47: for each edge, the edges sharing no vertex, in index order."""
    closed = F.trefoil(24, jitter=0.0, seed=7)[1]
    y = np.array([[0, 1], [1, 2], [2, 3], [1, 4], [4, 5], [5, 0], [3, 3]], dtype=np.int32)
    for e in (closed, y):
        got = T.calculateDisjointPairs(e)
        assert got == _oracle_pairs(e)
    # a closed polygon: every edge is disjoint from all but itself and its two neighbours
    assert all(len(p) == len(closed) - 3 for p in T.calculateDisjointPairs(closed))
