"""Host logic of the hierarchical path, on the CPU: api.bctApplyB's glue around
the block-cluster-tree products (the edge averages or tangential differences of
u, K1 y - K y, the spread back to the vertices, after the stage-2 oracle's
bct_apply_B_scalar, oracle/tpe_stage2_oracle.py:742-805). The two products are
replaced by a dense numpy restatement of the exact edge kernels
(exact_edge_kernel_pair, :712-740), which is what the device products return at
theta = 0; the result must then be B u and B0 u of the C oracle's assembly
(innerProduct.ts assembleBHighFlat / assembleBLowFlat)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as O
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

EPS = 1e-10


def _dense_kernel(v, e, kind):
    """K[I][J] for disjoint edges I != J (0 otherwise)."""
    p = 7.0 / 3.0
    E = len(e)
    a, b = e[:, 0], e[:, 1]
    d = v[b] - v[a]
    lr = np.linalg.norm(d, axis=1)
    ell = lr + EPS
    Tn = np.where(lr[:, None] >= 1e-14, d / np.where(lr[:, None] > 0, lr[:, None], 1.0), 0.0)
    K = np.zeros((E, E))
    for I in range(E):
        for J in range(E):
            if I == J or len({a[I], b[I]} & {a[J], b[J]}):
                continue
            s1 = s2 = 0.0
            for vi in (a[I], b[I]):
                for vj in (a[J], b[J]):
                    q = v[vi] - v[vj]
                    dn = np.linalg.norm(q) + EPS
                    if kind == "high":
                        s1 += 1.0 / dn ** p
                    else:
                        s1 += (np.linalg.norm(np.cross(Tn[I], q)) + EPS) ** 2 / dn ** (4 + p)
                        s2 += (np.linalg.norm(np.cross(Tn[J], -q)) + EPS) ** 2 / dn ** (4 + p)
            K[I, J] = 2 * 0.25 * ell[I] * ell[J] * s1 if kind == "high" else 0.25 * ell[I] * ell[J] * (s1 + s2)
    return K


@pytest.mark.parametrize("kind", ["high", "low"])
def test_apply_B_glue_against_dense_assembly(kind, monkeypatch):
    v, e = F.random_walk_knot(48, seed=21)
    e = np.asarray(e)
    K = _dense_kernel(v, e, kind)

    def fake_bct(vertices, edges, psi, kind_, epsilon=1e-10, theta=0.5, leafSize=8, thetaT=None):
        assert kind_ == kind
        stats = {"leaves": 1, "admissible_blocks": 0, "direct_blocks": 1, "direct_pairs": 0}
        return K @ np.asarray(psi), stats

    monkeypatch.setattr(T, "bctMatvec", fake_bct)
    u = np.sin(np.arange(len(v)) * 0.7)
    out, st = T.bctApplyB(v, e, u, kind, theta=0.0)
    M = np.asarray(O.assemble(v, e, "B" if kind == "high" else "B0")).reshape(len(v), len(v))
    want = M @ u
    assert np.linalg.norm(out - want) <= 1e-12 * np.linalg.norm(M) * np.linalg.norm(u)
    assert set(st) == {f"{p}_{k}" for p in ("K1", "Ky") for k in
                       ("leaves", "admissible_blocks", "direct_blocks", "direct_pairs")}


TREES = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                   "golden", "bh_trees.npz")


@pytest.mark.parametrize("name", ["trefoil120_leaf4", "network_leaf4", "walk20000_leaf8"])
def test_edge_tree_is_the_oracle_tree(name):
    """tpe_edge_tree (the host builder the device traversals use, threaded below its top
    levels for the 20000-edge walk) against the oracle's build_edge_bvh: the same nodes with
    the same edges (in the same order in every leaf), and bit-equal centers, mean tangents,
    masses and radii (the numpy summation orders are reproduced)."""
    import ctypes as C

    from repulsive_test2_b200 import abi

    z = np.load(TREES)
    v = np.ascontiguousarray(z[name + "/vertices"])
    e = np.ascontiguousarray(z[name + "/edges"], dtype=np.int32)
    leaf = int(z[name + "/leaf"][0])
    f_o, links, off, idx = z[name + "/f"], z[name + "/links"], z[name + "/idx_off"], z[name + "/idx"]
    E = len(e)
    maxn = 4 * E + 8
    node_f = np.zeros((maxn, 9))
    node_i = np.zeros((maxn, 4), dtype=np.int32)
    perm = np.zeros(E, dtype=np.int32)
    nn = C.c_int32(0)
    lib = abi.load_library()
    rc = lib.tpe_edge_tree(v.ctypes.data_as(abi.dp), len(v), e.ctypes.data_as(abi.ip), E, EPS, leaf, maxn,
                           node_f.ctypes.data_as(abi.dp), node_i.ctypes.data_as(abi.ip),
                           perm.ctypes.data_as(abi.ip), C.byref(nn))
    assert rc == 0
    assert nn.value == len(f_o)
    stack = [(0, 0)]
    seen = 0
    while stack:
        mine, theirs = stack.pop()
        seen += 1
        b, cnt, l, r = node_i[mine]
        want = idx[off[theirs]:off[theirs + 1]]
        if l < 0:  # a leaf keeps its edges in the oracle's order
            np.testing.assert_array_equal(perm[b:b + cnt], want)
        else:  # an inner node's range is reordered by its children
            np.testing.assert_array_equal(np.sort(perm[b:b + cnt]), np.sort(want))
        np.testing.assert_array_equal(node_f[mine], f_o[theirs])
        assert (l < 0) == (links[theirs][0] < 0)
        if l >= 0:
            stack.append((l, links[theirs][0]))
            stack.append((r, links[theirs][1]))
    assert seen == len(f_o)


MG = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                "golden", "mg_levels.npz")


@pytest.mark.parametrize("name", ["trefoil120", "network_pins4", "walk512_pins3"])
def test_mg_hierarchy_is_the_oracle_hierarchy(name):
    """api.mgHierarchy (tpe_mg_coarsen per level) against the oracle's build_hierarchy: the
    same number of levels and, level by level, the same coarse edges, original vertices,
    original edge paths and prolongation to the finer level."""
    z = np.load(MG)
    levels = T.mgHierarchy(z[name + "/vertices"], z[name + "/edges"], pinned=z[name + "/pins"])
    assert len(levels) == int(z[name + "/nlevels"][0])
    for li, L in enumerate(levels):
        key = f"{name}/L{li}"
        np.testing.assert_array_equal(L["edges"], z[key + "/edges"])
        np.testing.assert_array_equal(L["orig_vertices"], z[key + "/orig"])
        off, pe = z[key + "/path_off"], z[key + "/path_edges"]
        assert [list(p) for p in L["edge_paths"]] == [list(pe[off[j]:off[j + 1]]) for j in range(len(off) - 1)]
        if li > 0:
            np.testing.assert_array_equal(L["P_to_fine"], z[key + "/P"])
