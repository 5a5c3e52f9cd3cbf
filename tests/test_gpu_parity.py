"""CUDA path (libtpe through its C ABI) against the oracle and the reference goldens.

Tolerances: the reference's own (energy/B/A 1e-12 rel, g~/lambda/vertices 1e-9,
tau and projection iterations exact, residual <= 1e-10) plus 1e-10 relative for
energy and gradient against the FP64 oracle on the same inputs.
"""
from __future__ import annotations

import numpy as np
import pytest

import goldens as G
import oracle_lib as O
from repulsive_test2_b200 import abi
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu

STAGE1_PROJECTION = {"tolAbs": 1e-10, "tolRel": 1e-10}


def relerr(a, b):
    return G.rel(a, b)


def test_energy_gradient_golden_cases():
    for c in G.load("energy_bitexact.json"):
        v = np.asarray(c["vertices"], dtype=np.float64)
        e = np.asarray(c["edges"], dtype=np.int32)
        en, g = T.energyAndGradient(v, e, c["alpha"], c["beta"], c["epsilon"])
        assert abs(en - c["energy"]) <= 1e-12 * abs(c["energy"]), c["name"]
        assert relerr(g, c["gradient"]) <= 1e-12, c["name"]
        assert abs(T.calculateEnergy(v, e, None, c["alpha"], c["beta"], c["epsilon"]) - c["energy"]) <= \
            1e-12 * abs(c["energy"])


@pytest.mark.parametrize("name", G.STAGE1)
def test_stage1_energy_assembly(name):
    fx, gd, v, e = G.ref(name)
    a, b, eps = fx["alpha"], fx["beta"], fx["epsilon"]
    assert abs(T.calculateEnergy(v, e, None, a, b, eps) - gd["energy"]) <= 1e-12 * abs(gd["energy"])
    for which, fn in (("B", T.assembleBHighFlat), ("B0", T.assembleBLowFlat), ("A", T.assembleAFlat)):
        M = fn(v, e, None, a, b, eps)
        assert relerr(M, gd[which]) <= 1e-12, which
        assert np.array_equal(M, M.T)
    g = T.gradientAnalytical(v, e, None, a, b, eps)
    assert relerr(g, O.gradient(v, e, a, b, eps)) <= 1e-10
    fd = T.gradientFiniteDiff(v, e, None, a, b, eps, 1e-6)
    assert relerr(fd, gd["dE"]) <= 1e-6


@pytest.mark.parametrize("name", G.STAGE1)
def test_stage1_solve_and_line_search(name):
    fx, gd, v, e = G.ref(name)
    a, b, eps = fx["alpha"], fx["beta"], fx["epsilon"]
    s = [T.barycenterBlock(gd["x0_barycenter_target"])]
    r = T.solveConstrainedGradientSet(v, e, None, a, b, eps, gd["dE"], s)
    assert relerr(r["gTilde"], gd["g_tilde"]) <= 1e-9
    assert np.linalg.norm(r["lambda"] - gd["lambda"]) / max(1, np.linalg.norm(gd["lambda"])) <= 1e-9
    assert r["residual"] <= 1e-10
    ls = T.lineSearchStepSet(v, e, None, a, b, eps, gd["dE"], gd["g_tilde"], s,
                             {"projection": STAGE1_PROJECTION})
    gold = gd["line_search_step"]
    assert ls["accepted"] and ls["tau"] == gold["tau"]
    assert ls["projectionIterations"] == gold["projection_iterations"]
    assert abs(ls["energyAfter"] - gold["energy_after"]) <= 1e-12 * abs(gold["energy_after"])
    assert relerr(ls["vertices"], gold["vertices"]) <= 1e-9


@pytest.mark.parametrize("name,projection", G.SETS)
def test_constraint_set_goldens(name, projection):
    fx, gd, v, e = G.ref(name)
    a, b, eps = fx["alpha"], fx["beta"], fx["epsilon"]
    blocks = G.blocks_of(gd)
    ev = T.evaluateConstraintSet(blocks, v, e)
    assert relerr(ev["C"], gd["C_stacked"]) <= 1e-12
    assert np.allclose(ev["phi"], gd["Phi_stacked"], atol=1e-12)
    r = T.solveConstrainedGradientSet(v, e, None, a, b, eps, gd["dE"], blocks)
    assert relerr(r["gTilde"], gd["g_tilde"]) <= 1e-9
    assert r["residual"] <= 1e-10
    opts = {}
    pen = G.penalties_of(gd)
    if pen:
        opts["penalties"] = {"totalLength": pen["w_length"], "lengthDiff": pen["w_diff"],
                             "field": {"weight": pen["w_field"], "X": pen["X"]}}
    if projection == "frozen":
        opts["projectionMode"] = "frozen"
    ls = T.lineSearchStepSet(v, e, None, a, b, eps, gd["dE"], gd["g_tilde"], blocks, opts)
    gold = gd["line_search_step"]
    assert ls["accepted"]
    assert ls["tau"] == gold["tau"]
    assert ls["projectionIterations"] == gold["projection_iterations"]
    assert abs(ls["energyBefore"] - gold["energy_before"]) <= 1e-12 * abs(gold["energy_before"])
    assert abs(ls["energyAfter"] - gold["energy_after"]) <= 1e-12 * abs(gold["energy_after"])
    assert relerr(ls["vertices"], gold["vertices"]) <= 1e-9


@pytest.mark.parametrize("name", ["crossing-bary-pen-length", "helix-bary-pen-field",
                                  "junction-y-bary-pen-diff", "crossing-length-pen-combo"])
def test_penalties(name):
    fx, gd, v, e = G.ref(name)
    p = G.penalties_of(gd)
    cfg = {"totalLength": p["w_length"], "lengthDiff": p["w_diff"], "field": {"weight": p["w_field"], "X": p["X"]}}
    assert abs(T.penaltyEnergy(v, e, cfg) - gd["penalty_energy_initial"]) <= 1e-12 * max(1, gd["penalty_energy_initial"])
    pg = T.penaltyGradient(v, e, cfg)
    assert relerr(np.concatenate([pg[:, 0], pg[:, 1], pg[:, 2]]), gd["dE_penalty_flat"]) <= 1e-12


def _step_compare(v, e, blocks, opts_gpu, opts_oracle, e_tol=1e-10, v_tol=1e-9):
    r = T.sobolevStepSet(v, e, None, blocks, opts_gpu)
    rc, out, st, _ = O.sobolev_step(v, e, blocks, opts_oracle)
    assert rc == 0
    assert r["accepted"] == bool(st.accepted)
    assert r["converged"] == bool(st.converged)
    assert r["stats"]["tau"] == st.tau
    assert (r["stats"]["projectionIterations"] if r["stats"]["projectionIterations"] is not None else -1) == \
        st.projection_iterations
    assert abs(r["energy"] - st.energy) <= e_tol * abs(st.energy)
    assert relerr(r["vertices"], out) <= v_tol
    return r, st


@pytest.mark.parametrize("mode", ["reassemble", "frozen"])
def test_step_trefoil128(mode):
    """Config 1: trefoil V=E=128 + N(0, 0.01^2) jitter, [barycenter, totalLength], one step."""
    v, e = F.trefoil(128, jitter=0.01, seed=128)
    x0 = T.barycenterTarget(v, e)
    L0 = T.totalLength(v, e)
    blocks = [T.barycenterBlock(x0), T.totalLengthBlock(L0)]
    o = O.default_opts(projection_mode=abi.PROJECTION_FROZEN if mode == "frozen" else abi.PROJECTION_REASSEMBLE)
    r, st = _step_compare(v, e, blocks, {"projectionMode": mode}, o)
    assert r["accepted"]


def test_flow_crossing_five_steps():
    fx, gd, v, e = G.ref("crossing")
    x0 = T.barycenterTarget(v, e)
    L0 = T.totalLength(v, e)
    blocks = [T.barycenterBlock(x0), T.totalLengthBlock(L0)]
    prev = T.calculateEnergy(v, e)
    cur = v
    for _ in range(5):
        r = T.sobolevStepSet(cur, e, None, blocks)
        assert r["accepted"] and r["energy"] < prev
        prev = r["energy"]
        cur = r["vertices"]
        L1 = T.totalLength(cur, e)
        assert abs(L1 - L0) <= 1e-4 * max(1, L1)


def test_empty_set_step():
    fx, gd, v, e = G.ref("crossing")
    r = T.sobolevStepSet(v, e, None, [])
    assert r["accepted"] and r["energy"] < T.calculateEnergy(v, e)
    assert r["stats"]["projectionIterations"] == 0
    assert r["stats"]["residual"] <= 1e-10


def test_isolated_vertex_singular():
    fx, gd, v, e = G.ref("crossing")
    v2 = np.vstack([v, [[5.0, 5.0, 5.0]]])
    x0 = T.barycenterTarget(v2, e)
    r = T.sobolevStepSet(v2, e, None, [T.barycenterBlock(x0)])
    assert not r["accepted"] and not r["converged"]
    assert r["stats"]["reason"] == "singular_system"
    assert r["stats"]["tau"] == 0 and np.array_equal(r["vertices"], v2)


def test_nonfinite_saddle_is_singular():
    fx, gd, v, e = G.ref("crossing")
    A = np.asarray(gd["A"], dtype=np.float64)
    n = len(A)
    Cm = np.asarray(gd["C_barycenter"])
    with pytest.raises(T.SingularSystemError):
        T.solveSaddleFromA(A, n, Cm, np.full(3 * n, np.nan))
    A2 = A.copy()
    A2[0, 1] = A2[1, 0] = np.nan
    with pytest.raises(T.SingularSystemError):
        T.solveSaddleFromA(A2, n, Cm, np.zeros(3 * n))


@pytest.mark.parametrize("name", G.STAGE1)
def test_solve_saddle_from_a_vs_oracle(name):
    fx, gd, v, e = G.ref(name)
    A = np.asarray(gd["A"], dtype=np.float64)
    n = len(A)
    Cm = np.asarray(gd["C_barycenter"])
    rhs = np.asarray(gd["dE_flat"])
    r = T.solveSaddleFromA(A, n, Cm, rhs)
    st, x, lam, res = O.solve_saddle(A, n, Cm, rhs)
    assert st == 0
    assert relerr(r["x"], x) <= 1e-9 and r["residual"] <= 1e-10
    # projection form: bottom block -Phi
    rb = -np.asarray(gd["Phi_barycenter"]) + 0.01
    r = T.solveSaddleFromA(A, n, Cm, np.zeros(3 * n), rb)
    st, x, lam, res = O.solve_saddle(A, n, Cm, np.zeros(3 * n), rb)
    assert relerr(r["x"], x) <= 1e-9 and r["residual"] <= 1e-10


def test_random_walk_energy_gradient_vs_oracle():
    """Config 2 construction at V=512: energy and gradient within 1e-10 of the oracle."""
    v, e = F.random_walk_knot(512, seed=2)
    en, g = T.energyAndGradient(v, e)
    assert abs(en - O.energy(v, e)) <= 1e-10 * abs(en)
    assert relerr(g, O.gradient(v, e)) <= 1e-10
    A = T.assembleAFlat(v, e)
    assert relerr(A, O.assemble(v, e, "A")) <= 1e-12


def test_central_fd_directions():
    """Adjoint gradient vs central differences along 64 seeded random directions, with
    test_gradient.ts's gate |fd - an| <= 1e-6 + 1e-5 max|an| (h = 1e-6)."""
    v, e = F.random_walk_knot(256, seed=7)
    en, g = T.energyAndGradient(v, e)
    dirs = F.normals(99, 64 * v.size).reshape(64, -1, 3)
    h = 1e-6
    curves = np.concatenate([v[None] + h * dirs, v[None] - h * dirs], axis=0)
    es = T.energyBatch(curves, e)
    fd = (es[:64] - es[64:]) / (2 * h)
    an = np.einsum("kvc,vc->k", dirs, g)
    assert np.max(np.abs(fd - an)) <= 1e-5 * np.max(np.abs(an)) + 1e-6


def test_step_random_walk_256_vs_oracle():
    v, e = F.random_walk_knot(256, seed=3)
    x0 = T.barycenterTarget(v, e)
    blocks = [T.barycenterBlock(x0), T.totalLengthBlock(T.totalLength(v, e))]
    o = O.default_opts(projection_mode=abi.PROJECTION_FROZEN)
    _step_compare(v, e, blocks, {"projectionMode": "frozen"}, o)


def test_step_random_walk_odd_size_vs_oracle():
    """V = 301: rows of the V x V factor start on 8- but not 16-byte boundaries
    (the trailing update then stages them by 8-byte copies); ragged last block."""
    v, e = F.random_walk_knot(301, seed=4)
    x0 = T.barycenterTarget(v, e)
    blocks = [T.barycenterBlock(x0), T.totalLengthBlock(T.totalLength(v, e))]
    o = O.default_opts(projection_mode=abi.PROJECTION_FROZEN)
    _step_compare(v, e, blocks, {"projectionMode": "frozen", "precision": "fp64"}, o)


def test_step_edge_lengths_and_pins_vs_oracle():
    v, e = F.trefoil(96, jitter=0.01, seed=5)
    x0 = T.barycenterTarget(v, e)
    blocks = [T.barycenterBlock(x0), T.edgeLengthsBlock(T.edgeLengths(v, e)), T.pointBlock(7, v[7])]
    o = O.default_opts(projection_mode=abi.PROJECTION_FROZEN)
    _step_compare(v, e, blocks, {"projectionMode": "frozen"}, o)


def test_step_penalties_network_vs_oracle():
    v, e = F.loop_network(loops=3, n=48, junctions=2, seed=9)
    x0 = T.barycenterTarget(v, e)
    blocks = [T.barycenterBlock(x0), T.pointBlock(3, v[3])]
    cfg = {"totalLength": 1.0, "lengthDiff": 10.0, "field": {"weight": 5.0, "X": [0.5, 1.0, 0.0]}}
    o = O.default_opts(projection_mode=abi.PROJECTION_FROZEN)
    o.has_penalties = 1
    o.penalties = O.penalties_struct(1.0, 10.0, 5.0, (0.5, 1.0, 0.0))
    _step_compare(v, e, blocks, {"projectionMode": "frozen", "penalties": cfg}, o)


def test_backstops_never_raise():
    fx, gd, v, e = G.ref("crossing")
    ev = T.evaluateConstraintSet([T.edgeLengthsBlock([1.0])], v, e)
    assert not np.isnan(ev["phi"][0]) and np.isnan(ev["phi"][1:]).all()
    ev = T.evaluateConstraintSet([T.pointBlock(999, [0, 0, 0])], v, e)
    assert np.isnan(ev["phi"]).all() and (ev["C"] == 0).all()
    # mismatched ell0 inside a step: same outcome as the oracle, no exception
    x0 = T.barycenterTarget(v, e)
    blocks = [T.barycenterBlock(x0), T.edgeLengthsBlock([1.0])]
    r = T.sobolevStepSet(v, e, None, blocks)
    rc, out, st, _ = O.sobolev_step(v, e, blocks)
    assert r["accepted"] == bool(st.accepted) and r["stats"].get("reason") == abi.REASONS[st.reason]


@pytest.mark.parametrize("mode", ["analytical", "finiteDiff"])
def test_raw_gradient_step(mode):
    """optimizer.ts:37-71 on the device: grad, v - stepSize*grad, energy(next)."""
    v, e = F.trefoil(64, jitter=0.01, seed=64)
    s = 1e-3
    r = T.step(v, e, None, {"mode": mode, "stepSize": s, "collectField": True})
    g = O.gradient(v, e) if mode == "analytical" else O.gradient_fd(v, e)
    assert relerr(r["field"], g) <= (1e-10 if mode == "analytical" else 1e-6)
    assert np.array_equal(r["vertices"], v - s * r["field"])
    en = O.energy(r["vertices"], e)
    assert abs(r["energy"] - en) <= 1e-10 * abs(en)
    assert "field" not in T.step(v, e, None, {"mode": mode, "stepSize": s})


@pytest.mark.parametrize("V", [8, 33, 301, 1000])
def test_closed_loop_assembly_vs_oracle(V):
    """A of a single closed loop (edge I = (I, I+1 mod V)) comes from the fused
    stencil kernel; the same loop with its edges listed in another order takes
    the general pair-matrix path. Both against the oracle's assembleAFlat."""
    v, e = F.random_walk_knot(V, seed=60 + V)
    want = O.assemble(v, e, "A")
    A = T.assembleAFlat(v, e)
    assert relerr(A, want) <= 1e-12
    assert np.array_equal(A, A.T)
    perm = np.roll(np.arange(V), 3)
    e2 = np.ascontiguousarray(e[perm])
    A2 = T.assembleAFlat(v, e2)
    assert relerr(A2, O.assemble(v, e2, "A")) <= 1e-12
    assert relerr(A, A2) <= 1e-12
