"""Regenerates tests/golden/bh_cases.npz and bct_cases.npz: Barnes-Hut energies
and block-cluster-tree kernel products of the reference's own stage-2 oracle
(oracle/tpe_stage2_oracle.py bh_energy, bct_matvec_kernel) with their counts.

Run where a checkout of the reference repository exists, naming its root in
REFERENCE_ROOT (required; there is no default); the GPU tests only read the
file this writes:

    REFERENCE_ROOT=<reference checkout> python tests/golden/make_bh.py

Cases: the closed trefoil of the oracle's own check script (oracle/check_bh_stage2.py:
N points on t in [0, 2 pi), scale 0.25) at N = 60 with theta = 0 (leaf 2 and 8:
the exact energy, no cluster admitted) and at N = 120 with (theta, theta_t,
leaf) = (0.5, 0.75, 4) and (0.25, 0.5, 4); a seeded random-walk knot (V = 512)
at the default (0.5, 0.75, 8) and at (0.5, 0.75, 4); and a small loop network
(3 loops of 64 joined at 2 junctions: vertices of degree 3, not one closed loop).
Each case stores vertices, edges, (alpha, beta, epsilon, theta, theta_t, leaf),
the energy, the exact energy (calculate_energy) and the counts (visits,
approximated edge references, direct pairs). The kernel-product cases (high and
low kernels, theta = 0 on the 60-point trefoil, a three-column psi) store psi,
phi, the dense product exact_edge_kernel_sym @ psi and the block counts
(leaves, admissible blocks, direct blocks, direct pairs). bh_trees.npz holds the
oracle's trees (build_edge_bvh) node by node: center, mean tangent, mass, radii,
children and edge lists, for a trefoil, the loop network and a 20000-edge walk.
mg_levels.npz holds the oracle's multigrid hierarchies (build_hierarchy): every
level's edges, original vertices, edge paths and prolongation, for a trefoil, the
loop network with 4 pins and a random walk with 3 pins.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("REFERENCE_ROOT", "")
sys.path.insert(0, REPO)

from repulsive_test2_b200 import fixtures  # noqa: E402

ALPHA, BETA, EPS = 3.0, 6.0, 1e-10


def trefoil(n):
    t = np.linspace(0.0, 2.0 * np.pi, n, endpoint=False)
    v = np.stack([np.sin(t) + 2.0 * np.sin(2.0 * t), np.cos(t) - 2.0 * np.cos(2.0 * t), -np.sin(3.0 * t)],
                 axis=1) * 0.25
    e = np.asarray([[i, (i + 1) % n] for i in range(n)], dtype=np.int64)
    return v, e


def main():
    if not REF:
        sys.exit("set REFERENCE_ROOT to the reference checkout")
    sys.path.insert(0, os.path.join(REF, "oracle"))
    import tpe_stage2_oracle as O

    v60, e60 = trefoil(60)
    v120, e120 = trefoil(120)
    vrw, erw = fixtures.random_walk_knot(512, seed=3)
    vnet, enet = fixtures.loop_network(loops=3, n=64, junctions=2, seed=7)
    cases = [
        ("trefoil60_exact_leaf2", v60, e60, 0.0, 0.0, 2),
        ("trefoil60_exact_leaf8", v60, e60, 0.0, 0.0, 8),
        ("trefoil120_0.5", v120, e120, 0.5, 0.75, 4),
        ("trefoil120_0.25", v120, e120, 0.25, 0.5, 4),
        ("walk512_default", vrw, erw, 0.5, 0.75, 8),
        ("walk512_leaf4", vrw, erw, 0.5, 0.75, 4),
        ("network_0.5", vnet, enet, 0.5, 0.75, 4),
    ]
    out = {}
    for name, v, e, th, tht, leaf in cases:
        v = np.asarray(v, dtype=np.float64)
        e = np.asarray(e, dtype=np.int64)
        en, st = O.bh_energy(v, e, ALPHA, BETA, EPS, theta=th, leaf_size=leaf, theta_t=tht)
        ex = O.calculate_energy(v, e, ALPHA, BETA, EPS)
        out[name + "/vertices"] = v
        out[name + "/edges"] = e.astype(np.int32)
        out[name + "/params"] = np.array([ALPHA, BETA, EPS, th, tht, leaf], dtype=np.float64)
        out[name + "/energy"] = np.array([en, ex])
        out[name + "/stats"] = np.array([st["visits"], st["approximated_edge_refs"], st["direct_pairs"]],
                                        dtype=np.int64)
        print(f"{name}: E={len(e)} bh={en:.17g} exact={ex:.17g} rel={abs(en - ex) / abs(ex):.2e} {st}")
    np.savez_compressed(os.path.join(HERE, "bh_cases.npz"), **out)

    # block-cluster-tree kernel products (bct_matvec_kernel)
    bct = {}
    vec = np.stack([np.sin(np.arange(120) * 0.61) + 0.2, np.cos(np.arange(120) * 0.37),
                    np.sin(np.arange(120) * 0.11) - 0.5], axis=1)
    bcases = [
        ("trefoil60_exact_leaf2_high", v60, e60, "high", 0.0, 0.0, 2, None),
        ("trefoil60_exact_leaf8_low", v60, e60, "low", 0.0, 0.0, 8, None),
        ("trefoil120_high", v120, e120, "high", 0.5, 0.75, 4, None),
        ("trefoil120_low", v120, e120, "low", 0.5, 0.75, 4, None),
        ("trefoil120_high_vec", v120, e120, "high", 0.5, 0.75, 4, vec),
        ("walk512_high", vrw, erw, "high", 0.5, 0.75, 8, None),
        ("walk512_low", vrw, erw, "low", 0.5, 0.75, 8, None),
        ("network_low", vnet, enet, "low", 0.5, 0.75, 4, None),
    ]
    for name, v, e, kind, th, tht, leaf, psi in bcases:
        v = np.asarray(v, dtype=np.float64)
        e = np.asarray(e, dtype=np.int64)
        if psi is None:
            psi = np.sin(np.arange(len(e)) * 0.61) + 0.2
        phi, st = O.bct_matvec_kernel(v, e, EPS, psi, kind, theta=th, leaf_size=leaf, theta_t=tht)
        exact = O.exact_edge_kernel_sym(v, e, EPS, kind) @ psi
        bct[name + "/vertices"] = v
        bct[name + "/edges"] = e.astype(np.int32)
        bct[name + "/params"] = np.array([EPS, th, tht, leaf, 0 if kind == "high" else 1], dtype=np.float64)
        bct[name + "/psi"] = np.asarray(psi, dtype=np.float64)
        bct[name + "/phi"] = phi
        bct[name + "/exact"] = exact
        bct[name + "/stats"] = np.array([st["leaves"], st["admissible_blocks"], st["direct_blocks"],
                                         st["direct_pairs"]], dtype=np.int64)
        rel = np.linalg.norm(phi - exact) / max(1.0, np.linalg.norm(exact))
        print(f"{name}: E={len(e)} rel_vs_exact={rel:.2e} {st}")
    # the oracle's trees themselves (build_edge_bvh), node by node in its preorder
    trees = {}
    vbig, ebig = fixtures.random_walk_knot(20000, seed=13)
    for name, v, e, leaf in (("trefoil120_leaf4", v120, e120, 4), ("network_leaf4", vnet, enet, 4),
                             ("walk20000_leaf8", vbig, ebig, 8)):
        v = np.asarray(v, dtype=np.float64)
        e = np.asarray(e, dtype=np.int64)
        nodes, _, _, _ = O.build_edge_bvh(v, e, EPS, leaf)
        trees[name + "/vertices"] = v
        trees[name + "/edges"] = e.astype(np.int32)
        trees[name + "/leaf"] = np.array([leaf])
        trees[name + "/f"] = np.array([np.concatenate([nd.center, nd.tangent, [nd.mass, nd.rx, nd.rT]])
                                       for nd in nodes])
        trees[name + "/links"] = np.array([[-1 if nd.left is None else nd.left,
                                            -1 if nd.right is None else nd.right] for nd in nodes], dtype=np.int32)
        trees[name + "/idx_off"] = np.cumsum([0] + [len(nd.indices) for nd in nodes]).astype(np.int64)
        trees[name + "/idx"] = np.concatenate([nd.indices for nd in nodes]).astype(np.int32)
        print(f"tree {name}: {len(nodes)} nodes")
    np.savez_compressed(os.path.join(HERE, "bh_trees.npz"), **trees)

    # the multigrid hierarchy (build_hierarchy / build_coarse_level)
    mg = {}
    vw, ew = fixtures.random_walk_knot(512, seed=17)
    pins_net = [int(p) for p in fixtures.seeded_pins(len(vnet), 4, seed=2)]
    for name, v, e, pins in (("trefoil120", v120, e120, []), ("network_pins4", vnet, enet, pins_net),
                             ("walk512_pins3", vw, ew, [5, 200, 401])):
        v = np.asarray(v, dtype=np.float64)
        e = np.asarray(e, dtype=np.int64)
        spec = O.ConstraintSpec(points=tuple((p, tuple(v[p])) for p in pins))
        levels = O.build_hierarchy(v, e, spec)
        mg[name + "/vertices"] = v
        mg[name + "/edges"] = e.astype(np.int32)
        mg[name + "/pins"] = np.asarray(pins, dtype=np.int32)
        mg[name + "/nlevels"] = np.array([len(levels)])
        for li, L in enumerate(levels):
            key = f"{name}/L{li}"
            mg[key + "/edges"] = np.asarray(L.edges, dtype=np.int32)
            mg[key + "/orig"] = np.asarray(L.orig_vertices, dtype=np.int32)
            mg[key + "/path_off"] = np.cumsum([0] + [len(p) for p in L.edge_paths]).astype(np.int32)
            mg[key + "/path_edges"] = np.concatenate([np.asarray(p, dtype=np.int32) for p in L.edge_paths])
            if L.P_to_fine is not None:
                mg[key + "/P"] = L.P_to_fine
        print(f"hierarchy {name}: levels {[len(L.vertices) for L in levels]}")
    np.savez_compressed(os.path.join(HERE, "mg_levels.npz"), **mg)

    # the Sobolev operators through the products (bct_apply_B_scalar)
    u = np.sin(np.arange(120) * 0.7)
    for kind in ("high", "low"):
        name = f"applyB_trefoil120_{kind}"
        o, st = O.bct_apply_B_scalar(v120, e120, EPS, u, kind, 0.5, 4, theta_t=0.75)
        bct[name + "/vertices"] = v120
        bct[name + "/edges"] = e120.astype(np.int32)
        bct[name + "/params"] = np.array([EPS, 0.5, 0.75, 4, 0 if kind == "high" else 1], dtype=np.float64)
        bct[name + "/u"] = u
        bct[name + "/out"] = o
        bct[name + "/stats"] = np.array([st[k] for k in sorted(st)], dtype=np.int64)
        print(f"{name}: {st}")
    np.savez_compressed(os.path.join(HERE, "bct_cases.npz"), **bct)


if __name__ == "__main__":
    main()
