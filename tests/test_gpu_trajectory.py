"""Descent trajectories against the oracle, step by step.

The FP64 trajectory of the V=2048 random-walk knot (20 sobolevStepSet steps,
[barycenter, totalLength] frozen at the initial curve, frozen projection,
optimizer.ts:231-440) comes from tests/golden/traj_rw2048.npz, written by the
oracle on the CPU (tests/golden/make_trajectory.py). Each GPU step starts from
the oracle's iterate x_i with the oracle's E(x_i) as energyBefore, so a step's
error does not carry into the next: energy, the descent field g~ (the
constrained solve), tau, the projection iteration count and the vertices are
compared per step. A free-running GPU trajectory of the same 20 steps is then
compared with the fixture as a whole, and the mixed-precision step is held to
its own gates (energy 1e-8, projected gradient 1e-6, same tau) on every
iterate. Energy and the adjoint gradient are also compared with the oracle at
V=2048 and V=8192 (the O(E^2) oracle loops run in seconds there).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle_lib as O
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "traj_rw2048.npz")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def traj():
    d = np.load(FIXTURE)
    return {k: d[k] for k in d.files}


def _set(x0):
    v = x0
    e = F.closed_edges(len(v))
    return [T.barycenterBlock(O.barycenter_target(v, e)), T.totalLengthBlock(O.total_length(v, e))]


@pytest.mark.parametrize("V", [2048, 8192])
def test_energy_gradient_against_oracle_large(V):
    v, e = F.random_walk_knot(V, seed=1)
    en, g = T.energyAndGradient(v, e)
    en_o = O.energy(v, e)
    assert abs(en - en_o) <= 1e-10 * abs(en_o), (en, en_o)
    assert rel(g, O.gradient(v, e)) <= 1e-10


def test_fixture_matches_workload(traj):
    v, e = F.random_walk_knot(2048, seed=1)
    assert np.array_equal(traj["vertices"][0], v)
    assert np.array_equal(traj["edges"], e)
    assert abs(traj["energy"][0] - O.energy(v, e)) == 0.0


def test_fp64_steps_against_oracle(traj):
    """Per step: energy <= 1e-10, g~ <= 1e-8, vertices <= 1e-10 relative, tau and
    projection iterations exact, every step accepted like the oracle's."""
    X, e = traj["vertices"], traj["edges"]
    blocks = _set(X[0])
    worst = {"energy": 0.0, "field": 0.0, "vertices": 0.0}
    for i in range(len(traj["tau"])):
        o = {"projectionMode": "frozen", "energyBefore": float(traj["energy"][i]), "collectField": True}
        r = T.sobolevStepSet(X[i], e, None, blocks, o)
        assert r["accepted"] == bool(traj["accepted"][i]), i
        assert r["stats"]["tau"] == traj["tau"][i], (i, r["stats"]["tau"], traj["tau"][i])
        assert r["stats"]["projectionIterations"] == traj["projection_iterations"][i], i
        assert r["stats"]["residual"] <= 1e-10
        worst["energy"] = max(worst["energy"], abs(r["energy"] - traj["energy"][i + 1]) / abs(traj["energy"][i + 1]))
        worst["field"] = max(worst["field"], rel(r["descentField"], traj["field"][i]))
        worst["vertices"] = max(worst["vertices"], rel(r["vertices"], X[i + 1]))
    print("fp64 per-step worst relative errors vs oracle:", worst)
    assert worst["energy"] <= 1e-10
    assert worst["field"] <= 1e-8
    assert worst["vertices"] <= 1e-10


def test_gradient_along_trajectory_against_oracle(traj):
    X, e = traj["vertices"], traj["edges"]
    for i in (0, 7, 14, len(X) - 1):
        en, g = T.energyAndGradient(X[i], e)
        assert abs(en - traj["energy"][i]) <= 1e-10 * abs(traj["energy"][i]), i
        assert rel(g, O.gradient(X[i], e)) <= 1e-10, i


def test_fp64_free_running_trajectory(traj):
    """20 GPU steps, each from the previous GPU output: the same taus and
    projection iterations, and the iterates within 1e-9 of the oracle's."""
    X, e = traj["vertices"], traj["edges"]
    blocks = _set(X[0])
    x, eb = X[0].copy(), float(traj["energy"][0])
    for i in range(len(traj["tau"])):
        r = T.sobolevStepSet(x, e, None, blocks, {"projectionMode": "frozen", "energyBefore": eb})
        assert r["stats"]["tau"] == traj["tau"][i], i
        assert r["stats"]["projectionIterations"] == traj["projection_iterations"][i], i
        if r["accepted"]:
            x, eb = r["vertices"], r["energy"]
        assert rel(x, X[i + 1]) <= 1e-9, (i, rel(x, X[i + 1]))
        assert abs(eb - traj["energy"][i + 1]) <= 1e-9 * abs(traj["energy"][i + 1]), i


def test_mixed_steps_against_oracle(traj):
    """The mixed-precision step (FP32 tensor-core factor + FP64 CG, batched
    trials) from every oracle iterate: energy <= 1e-8, projected gradient
    <= 1e-6 relative, the oracle's tau."""
    X, e = traj["vertices"], traj["edges"]
    blocks = _set(X[0])
    worst_e = worst_g = 0.0
    for i in range(len(traj["tau"])):
        o = {"projectionMode": "frozen", "energyBefore": float(traj["energy"][i]), "collectField": True,
             "precision": "mixed", "trials": 8}
        r = T.sobolevStepSet(X[i], e, None, blocks, o)
        assert r["stats"]["refineIterations"] > 0, i  # the mixed solve ran (no FP64 fallback)
        assert r["stats"]["tau"] == traj["tau"][i], i
        worst_e = max(worst_e, abs(r["energy"] - traj["energy"][i + 1]) / abs(traj["energy"][i + 1]))
        worst_g = max(worst_g, rel(r["descentField"], traj["field"][i]))
    print(f"mixed per-step worst relative errors vs oracle: energy {worst_e:.3g}, g~ {worst_g:.3g}")
    assert worst_e <= 1e-8
    assert worst_g <= 1e-6
