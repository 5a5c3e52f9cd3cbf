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
    """Per step, from the oracle's iterate: tau and projection iterations exact,
    the step accepted like the oracle's, the descent field g~ within 1e-8 and
    the new vertices within 2e-10 relative of the oracle's. The accepted
    energy is checked two ways: against the oracle's energy of the GPU's own new
    vertices (the evaluation itself, 1e-10), and against the oracle's accepted
    energy (2e-9: the two new iterates differ by the vertex error above, and the
    energy of a near-contact knot amplifies a relative position change about
    tenfold)."""
    X, e = traj["vertices"], traj["edges"]
    blocks = _set(X[0])
    worst = {"energy_eval": 0.0, "energy": 0.0, "field": 0.0, "vertices": 0.0}
    for i in range(len(traj["tau"])):
        o = {"projectionMode": "frozen", "energyBefore": float(traj["energy"][i]), "collectField": True}
        r = T.sobolevStepSet(X[i], e, None, blocks, o)
        assert r["accepted"] == bool(traj["accepted"][i]), i
        assert r["stats"]["tau"] == traj["tau"][i], (i, r["stats"]["tau"], traj["tau"][i])
        assert r["stats"]["projectionIterations"] == traj["projection_iterations"][i], i
        assert r["stats"]["residual"] <= 1e-10
        e_own = O.energy(r["vertices"], e)
        worst["energy_eval"] = max(worst["energy_eval"], abs(r["energy"] - e_own) / abs(e_own))
        worst["energy"] = max(worst["energy"], abs(r["energy"] - traj["energy"][i + 1]) / abs(traj["energy"][i + 1]))
        worst["field"] = max(worst["field"], rel(r["descentField"], traj["field"][i]))
        worst["vertices"] = max(worst["vertices"], rel(r["vertices"], X[i + 1]))
    print("fp64 per-step worst relative errors vs oracle:", worst)
    assert worst["energy_eval"] <= 1e-10
    assert worst["energy"] <= 2e-9
    assert worst["field"] <= 1e-8
    assert worst["vertices"] <= 2e-10


def test_gradient_along_trajectory_against_oracle(traj):
    X, e = traj["vertices"], traj["edges"]
    for i in (0, 7, 14, len(X) - 1):
        en, g = T.energyAndGradient(X[i], e)
        assert abs(en - traj["energy"][i]) <= 1e-10 * abs(traj["energy"][i]), i
        assert rel(g, O.gradient(X[i], e)) <= 1e-10, i


def test_fp64_free_running_trajectory(traj):
    """20 GPU steps, each from the previous GPU output (the app's loop): the
    same taus and projection iterations as the oracle's trajectory at every
    step. The iterates drift apart slowly (each step adds its own ~1e-11
    relative difference, and the descent map carries earlier ones along), so
    the whole-trajectory bounds are looser than the per-step ones: vertices
    1e-8, energies 1e-7 relative."""
    X, e = traj["vertices"], traj["edges"]
    blocks = _set(X[0])
    x, eb = X[0].copy(), float(traj["energy"][0])
    errs = []
    for i in range(len(traj["tau"])):
        r = T.sobolevStepSet(x, e, None, blocks, {"projectionMode": "frozen", "energyBefore": eb})
        same = (r["stats"]["tau"] == traj["tau"][i] and
                r["stats"]["projectionIterations"] == traj["projection_iterations"][i])
        if r["accepted"]:
            x, eb = r["vertices"], r["energy"]
        errs.append((i, same, rel(x, X[i + 1]), abs(eb - traj["energy"][i + 1]) / abs(traj["energy"][i + 1])))
    print("free-running (step, same tau and iterations, vertices, energy):",
          [(i, s_, f"{a:.2e}", f"{b:.2e}") for i, s_, a, b in errs])
    assert all(s_ for _, s_, _, _ in errs)
    assert max(a for _, _, a, _ in errs) <= 1e-8
    assert max(b for _, _, _, b in errs) <= 1e-7


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
