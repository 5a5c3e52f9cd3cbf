"""The hierarchical path of the reference's stage-2 oracle
(oracle/tpe_stage2_oracle.py): the Barnes-Hut energy (tpe_energy_bh, bh_energy)
and the block-cluster-tree kernel product (tpe_bct_matvec, bct_matvec_kernel).

Against the oracle's own outputs (tests/golden/bh_cases.npz, written by
tests/golden/make_bh.py from the reference's Python oracle): the energy within
1e-12 and the tree visits, approximated edge references and direct pairs
exactly, which pins the tree (same splits, same order) and every admissibility
decision. Then the oracle check script's gates (oracle/check_bh_stage2.py) at
sizes the Python oracle cannot reach: theta = 0 is the exact energy, clusters
are admitted, and the error shrinks with theta."""
from __future__ import annotations

import os

import numpy as np
import pytest

from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bh_cases.npz")


def _cases():
    z = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in z.files})
    return [(n, z) for n in names]


@pytest.mark.parametrize("name", [n for n, _ in _cases()])
def test_bh_matches_reference_oracle(name):
    z = np.load(GOLDEN)
    v, e = z[name + "/vertices"], z[name + "/edges"]
    alpha, beta, eps, th, tht, leaf = z[name + "/params"]
    want, exact = z[name + "/energy"]
    st_want = z[name + "/stats"]
    got, st = T.bhEnergy(v, e, alpha, beta, eps, theta=th, leafSize=int(leaf), thetaT=tht)
    assert abs(got - want) <= 1e-12 * abs(want), (got, want)
    assert [st["visits"], st["approximated_edge_refs"], st["direct_pairs"]] == list(st_want)
    if th == 0.0:
        assert st["approximated_edge_refs"] == 0
        assert abs(got - T.calculateEnergy(v, e)) <= 1e-12 * abs(exact)


def test_bh_gates_at_large_sizes():
    """check_bh_stage2.py's three gates on curves of 2048 and 16384 edges."""
    v, e = F.random_walk_knot(2048, seed=4)
    exact = T.calculateEnergy(v, e)
    for leaf in (2, 8):
        got, st = T.bhEnergy(v, e, theta=0.0, leafSize=leaf)
        assert st["approximated_edge_refs"] == 0
        assert abs(got - exact) <= 1e-12 * abs(exact)
    n = 16384
    t = np.linspace(0.0, 2.0 * np.pi, n, endpoint=False)
    v = np.stack([np.sin(t) + 2.0 * np.sin(2.0 * t), np.cos(t) - 2.0 * np.cos(2.0 * t), -np.sin(3.0 * t)],
                 axis=1) * 0.25
    e = np.asarray([[i, (i + 1) % n] for i in range(n)], dtype=np.int32)
    exact = T.calculateEnergy(v, e)
    e05, st05 = T.bhEnergy(v, e, theta=0.5, leafSize=8, thetaT=0.75)
    e025, st025 = T.bhEnergy(v, e, theta=0.25, leafSize=8, thetaT=0.5)
    rel05, rel025 = abs(e05 - exact) / abs(exact), abs(e025 - exact) / abs(exact)
    assert st05["approximated_edge_refs"] > 0
    assert rel05 <= 5e-2 and rel025 <= rel05
    # the tree replaces most of the n^2 pairs
    assert st05["direct_pairs"] < 0.1 * n * n


BCT_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bct_cases.npz")


def _bct_names(prefix=""):
    return sorted({k.split("/")[0] for k in np.load(BCT_GOLDEN).files if k.endswith("/params")
                   and k.startswith(prefix) and not k.startswith("applyB")} if not prefix else
                  {k.split("/")[0] for k in np.load(BCT_GOLDEN).files if k.startswith(prefix)})


@pytest.mark.parametrize("name", _bct_names())
def test_bct_matvec_matches_reference_oracle(name):
    """tpe_bct_matvec against the oracle's bct_matvec_kernel: phi within 1e-12 of
    its norm and the block counts exactly (same tree, same block recursion)."""
    z = np.load(BCT_GOLDEN)
    v, e, psi = z[name + "/vertices"], z[name + "/edges"], z[name + "/psi"]
    eps, th, tht, leaf, kind = z[name + "/params"]
    want, exact = z[name + "/phi"], z[name + "/exact"]
    phi, st = T.bctMatvec(v, e, psi, "high" if kind == 0 else "low", epsilon=eps, theta=th,
                          leafSize=int(leaf), thetaT=tht)
    assert np.linalg.norm(phi - want) <= 1e-12 * np.linalg.norm(want)
    assert [st["leaves"], st["admissible_blocks"], st["direct_blocks"], st["direct_pairs"]] == \
        list(z[name + "/stats"])
    if th == 0.0:
        assert np.linalg.norm(phi - exact) <= 1e-12 * np.linalg.norm(exact)


def test_bct_matvec_large_sizes():
    """theta = 0 is the exact product and the error shrinks with theta, at 8192 edges."""
    n = 8192
    t = np.linspace(0.0, 2.0 * np.pi, n, endpoint=False)
    v = np.stack([np.sin(t) + 2.0 * np.sin(2.0 * t), np.cos(t) - 2.0 * np.cos(2.0 * t), -np.sin(3.0 * t)],
                 axis=1) * 0.25
    e = np.asarray([[i, (i + 1) % n] for i in range(n)], dtype=np.int32)
    psi = np.sin(np.arange(n) * 0.61) + 0.2
    for kind in ("high", "low"):
        ex, st0 = T.bctMatvec(v, e, psi, kind, theta=0.0, leafSize=8)
        assert st0["admissible_blocks"] == 0 and st0["direct_pairs"] == n * (n - 3)
        p05, st05 = T.bctMatvec(v, e, psi, kind, theta=0.5, leafSize=8, thetaT=0.75)
        p025, _ = T.bctMatvec(v, e, psi, kind, theta=0.25, leafSize=8, thetaT=0.5)
        r05 = np.linalg.norm(p05 - ex) / np.linalg.norm(ex)
        r025 = np.linalg.norm(p025 - ex) / np.linalg.norm(ex)
        assert st05["admissible_blocks"] > 0 and st05["direct_pairs"] < 0.2 * n * n
        assert r025 <= r05


@pytest.mark.parametrize("name", _bct_names("applyB"))
def test_bct_apply_B_matches_reference_oracle(name):
    """The Sobolev operators through the products (bct_apply_B_scalar) at theta 0.5."""
    z = np.load(BCT_GOLDEN)
    v, e, u = z[name + "/vertices"], z[name + "/edges"], z[name + "/u"]
    eps, th, tht, leaf, kind = z[name + "/params"]
    out, st = T.bctApplyB(v, e, u, "high" if kind == 0 else "low", epsilon=eps, theta=th,
                          leafSize=int(leaf), thetaT=tht)
    want = z[name + "/out"]
    # K1 y - K y cancels: the bound is on the size of the two products' difference
    assert np.linalg.norm(out - want) <= 1e-11 * np.linalg.norm(want)
    assert [st[k] for k in sorted(st)] == list(z[name + "/stats"])


def test_bct_apply_B_theta0_is_the_dense_gram_product():
    """theta = 0: B u and B0 u from the hierarchical products equal the products with the
    dense matrices of the step's own assembly kernels (assembleBHighFlat / assembleBLowFlat)."""
    v, e = F.random_walk_knot(512, seed=9)
    u = np.sin(np.arange(512) * 0.7)
    for kind, assemble in (("high", T.assembleBHighFlat), ("low", T.assembleBLowFlat)):
        M = np.asarray(assemble(v, e)).reshape(512, 512)
        out, st = T.bctApplyB(v, e, u, kind, theta=0.0, leafSize=8)
        want = M @ u
        assert st["Ky_admissible_blocks"] == 0
        assert np.linalg.norm(out - want) <= 1e-12 * np.linalg.norm(M) * np.linalg.norm(u)
