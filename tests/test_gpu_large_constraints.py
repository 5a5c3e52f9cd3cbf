"""Large constraint sets: one edge-length row per edge (k = E + 3 with the
barycenter) take the device Schur path (explicit FP64 inverses of A_rho and of
the k x k Schur complement, Y and S by sparse gathers).

The mixed request forms both inverses with their products on the int8 tensor
cores (a recursive Cholesky and triangular inverse in halves, FP64 kernels on
the diagonal blocks of at most 1024, FP64-class products from exact digit
GEMMs); TPE_INT8_BASE lowers that block size so the recursion runs at orders
the oracle finishes in seconds.

Against the FP64 oracle (which factors the full (3V + k)^2 saddle matrix) at
sizes it finishes in seconds, with the parity tolerances of the small-k path,
in both precisions; at larger sizes through properties: the saddle residual,
the edge lengths held by the projection, the energy decrease, and agreement of
the mixed step with the FP64 step.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as O
from repulsive_test2_b200 import abi
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu


def _per_edge(v, e):
    return [T.barycenterBlock(T.barycenterTarget(v, e)), T.edgeLengthsBlock(T.edgeLengths(v, e))]


@pytest.mark.parametrize("V,seed,precision", [(72, 11, "fp64"), (512, 2, "fp64"), (512, 2, "mixed"),
                                              (300, 4, "mixed")])
def test_per_edge_step_vs_oracle(V, seed, precision, monkeypatch):
    monkeypatch.setenv("TPE_INT8_BASE", "128")  # recursion depth 2 at V=512
    v, e = F.random_walk_knot(V, seed=seed)
    blocks = _per_edge(v, e)
    r = T.sobolevStepSet(v, e, None, blocks, {"projectionMode": "frozen", "collectField": True,
                                              "precision": precision})
    rc, out, st, g = O.sobolev_step(v, e, blocks, O.default_opts(projection_mode=abi.PROJECTION_FROZEN))
    assert rc == 0
    assert r["accepted"] == bool(st.accepted)
    assert r["stats"]["tau"] == st.tau
    assert r["stats"]["projectionIterations"] == st.projection_iterations
    assert abs(r["energy"] - st.energy) <= 1e-10 * abs(st.energy)
    assert np.linalg.norm(r["vertices"] - out) <= 1e-9 * np.linalg.norm(out)
    assert r["stats"]["residual"] <= 1e-10


def test_per_edge_saddle_solve_vs_oracle():
    """The constrained gradient alone (no line search) at V=256: g~ and lambda."""
    v, e = F.random_walk_knot(256, seed=7)
    blocks = _per_edge(v, e)
    dE = O.gradient(v, e)
    rg = T.solveConstrainedGradientSet(v, e, None, 3.0, 6.0, 1e-10, dE, blocks)
    st, g, lam, res = O.solve_constrained_gradient(v, e, blocks, dE)
    assert st == 0
    assert np.linalg.norm(rg["gTilde"] - g) <= 1e-9 * np.linalg.norm(g)
    assert np.linalg.norm(rg["lambda"] - lam) <= 1e-8 * np.linalg.norm(lam)
    assert rg["residual"] <= 1e-10


def test_per_edge_2048_properties():
    V = 2048
    v, e = F.random_walk_knot(V, seed=1)
    ell = T.edgeLengths(v, e)
    blocks = _per_edge(v, e)
    proj = {"tolAbs": 1e-10, "tolRel": 1e-10}
    r64 = T.sobolevStepSet(v, e, None, blocks, {"projectionMode": "frozen", "precision": "fp64",
                                                "projection": proj})
    rmx = T.sobolevStepSet(v, e, None, blocks, {"projectionMode": "frozen", "precision": "mixed",
                                                "projection": proj})
    assert r64["accepted"]
    assert r64["stats"]["residual"] <= 1e-10
    assert r64["energy"] < T.calculateEnergy(v, e)
    # the projection holds the edge lengths to its tolerance: the block norm of
    # Phi within max(tolAbs, tolRel * max(1, total length))
    ell1 = T.edgeLengths(r64["vertices"], e)
    assert np.linalg.norm(ell1 - ell) <= 1e-10 * max(1.0, float(np.sum(ell)))
    # the int8-tensor-core inverses agree with the FP64 ones to FP64-class accuracy
    assert rmx["accepted"] and rmx["stats"]["residual"] <= 1e-10
    assert rmx["stats"]["tau"] == r64["stats"]["tau"]
    assert rmx["stats"]["projectionIterations"] == r64["stats"]["projectionIterations"]
    assert abs(rmx["energy"] - r64["energy"]) <= 1e-10 * abs(r64["energy"])
    assert np.linalg.norm(rmx["vertices"] - r64["vertices"]) <= 1e-9 * np.linalg.norm(r64["vertices"])
    assert not np.array_equal(rmx["vertices"], r64["vertices"])  # a different solve ran


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_per_edge_repeated_steps_are_bit_identical(precision, monkeypatch):
    monkeypatch.setenv("TPE_INT8_BASE", "128")
    v, e = F.random_walk_knot(512, seed=12)
    blocks = _per_edge(v, e)
    o = {"projectionMode": "frozen", "trials": 8, "collectField": True, "precision": precision}
    runs = [T.sobolevStepSet(v, e, None, blocks, o) for _ in range(2)]
    assert runs[1]["energy"] == runs[0]["energy"]
    assert np.array_equal(runs[1]["vertices"], runs[0]["vertices"])
    assert np.array_equal(runs[1]["descentField"], runs[0]["descentField"])


def test_per_edge_mixed_saddle_solve_vs_oracle(monkeypatch):
    """The mixed constrained gradient at V=600 (ragged halves: 640 -> 320 + 283 ...)."""
    monkeypatch.setenv("TPE_INT8_BASE", "128")
    v, e = F.random_walk_knot(600, seed=8)
    blocks = _per_edge(v, e)
    dE = O.gradient(v, e)
    st, g, lam, res = O.solve_constrained_gradient(v, e, blocks, dE)
    assert st == 0
    r = T.sobolevStepSet(v, e, None, blocks, {"projectionMode": "frozen", "precision": "mixed",
                                              "collectField": True})
    rc, out, sto, gt = O.sobolev_step(v, e, blocks, O.default_opts(projection_mode=abi.PROJECTION_FROZEN))
    assert rc == 0 and r["stats"]["tau"] == sto.tau
    assert np.linalg.norm(r["descentField"] - gt) <= 1e-9 * np.linalg.norm(gt)
    assert np.linalg.norm(r["vertices"] - out) <= 1e-9 * np.linalg.norm(out)
