"""Pins the CPU oracle to the reference's own golden vectors (CPU only).

Mirrors the reference's bun tests: test/golden.test.ts (bit-exact energy and
gradient), test/sobolev/{innerProduct,lowOrder,gradient,lineSearch,
constraintSetFlow,frozenProjection,penalties}.test.ts and
oracle/compare_energy.ts, with the tolerances written in those files.
"""
from __future__ import annotations

import numpy as np
import pytest

import goldens as G
import oracle_lib as O
from repulsive_test2_b200 import abi

STAGE1_PROJECTION = dict(proj_tol_abs=1e-10, proj_tol_rel=1e-10)  # lineSearch.test.ts:31


def test_energy_gradient_bit_exact():
    """test/golden.test.ts: energy and every gradient component with Object.is."""
    for c in G.load("energy_bitexact.json"):
        v = np.asarray(c["vertices"], dtype=np.float64)
        e = np.asarray(c["edges"], dtype=np.int32)
        en = O.energy(v, e, c["alpha"], c["beta"], c["epsilon"])
        g = O.gradient(v, e, c["alpha"], c["beta"], c["epsilon"])
        assert en == c["energy"], c["name"]
        want = np.asarray(c["gradient"], dtype=np.float64)
        assert np.array_equal(g.view(np.int64), want.view(np.int64)), c["name"]


@pytest.mark.parametrize("name", G.STAGE1)
def test_stage1_energy_assembly(name):
    fx, gd, v, e = G.ref(name)
    a, b, eps = fx["alpha"], fx["beta"], fx["epsilon"]
    assert abs(O.energy(v, e, a, b, eps) - gd["energy"]) <= 1e-12 * abs(gd["energy"])
    for which in ("B", "B0", "A"):
        M = O.assemble(v, e, which, a, b, eps)
        assert G.rel(M, gd[which]) <= 1e-12, which
        assert np.array_equal(M, M.T)  # explicit symmetrisation: exact
        assert np.linalg.norm(M.sum(axis=1)) <= 1e-10 * np.linalg.norm(M)  # constants in the kernel


@pytest.mark.parametrize("name", G.STAGE1)
def test_stage1_gradient_vs_fd(name):
    """oracle/compare_energy.ts: FD-vs-FD 1e-6, analytic-vs-FD 1e-4 (norm-relative)."""
    fx, gd, v, e = G.ref(name)
    a, b, eps = fx["alpha"], fx["beta"], fx["epsilon"]
    fd = O.gradient_fd(v, e, a, b, eps, 1e-6)
    an = O.gradient(v, e, a, b, eps)
    assert G.rel(fd, gd["dE"]) <= 1e-6
    assert G.rel(an, gd["dE"]) <= 1e-4


@pytest.mark.parametrize("name", G.STAGE1)
def test_stage1_constraint_and_solve(name):
    fx, gd, v, e = G.ref(name)
    x0 = O.barycenter_target(v, e)
    assert G.rel(x0, gd["x0_barycenter_target"]) <= 1e-12 or np.allclose(x0, gd["x0_barycenter_target"],
                                                                          atol=1e-14)
    blocks = [{"kind": "barycenter", "target": gd["x0_barycenter_target"]}]
    phi, Cm = O.evaluate_constraints(blocks, v, e)
    assert np.allclose(phi, gd["Phi_barycenter"], atol=1e-12)
    assert G.rel(Cm, gd["C_barycenter"]) <= 1e-12
    st, g, lam, res = O.solve_constrained_gradient(v, e, blocks, np.asarray(gd["dE"]))
    assert st == 0
    assert G.rel(g, gd["g_tilde"]) <= 1e-9
    assert np.linalg.norm(lam - gd["lambda"]) / max(1, np.linalg.norm(gd["lambda"])) <= 1e-9
    assert res <= 1e-10
    dEflat = np.asarray(gd["dE_flat"])
    gflat = np.concatenate([g[:, 0], g[:, 1], g[:, 2]])
    assert dEflat @ gflat > 0
    assert np.linalg.norm(Cm @ gflat) / max(1, np.linalg.norm(gflat)) <= 1e-10
    assert abs(O.l2_curve_norm(gd["g_tilde"], v, e) - gd["gradient_l2_norm"]) <= 1e-12 * gd["gradient_l2_norm"]


@pytest.mark.parametrize("factor", [abi.FACTOR_LDLT, abi.FACTOR_LU])
@pytest.mark.parametrize("name", G.STAGE1)
def test_stage1_line_search(name, factor):
    """lineSearch.test.ts: accepted, tau exact, iterations exact, energy 1e-12, vertices 1e-9."""
    fx, gd, v, e = G.ref(name)
    gold = gd["line_search_step"]
    blocks = [{"kind": "barycenter", "target": gd["x0_barycenter_target"]}]
    opts = O.default_opts(factor_mode=factor, **STAGE1_PROJECTION)
    rc, out, st = O.line_search_step(v, e, np.asarray(gd["dE"]), np.asarray(gd["g_tilde"]), blocks, opts)
    assert rc == 0 and st.accepted == 1 and gold["accepted"]
    assert st.tau == gold["tau"]
    assert st.projection_iterations == gold["projection_iterations"]
    assert abs(st.energy - gold["energy_after"]) <= 1e-12 * abs(gold["energy_after"])
    assert G.rel(out, gold["vertices"]) <= 1e-9
    assert st.energy <= st.energy_before - 1e-4 * st.tau * st.slope


@pytest.mark.parametrize("name,projection", G.SETS)
def test_constraint_set_goldens(name, projection):
    """constraintSetFlow / constraintSetM2Flow / frozenProjection / penalties tests."""
    fx, gd, v, e = G.ref(name)
    blocks = G.blocks_of(gd)
    pen = G.penalties_of(gd)
    phi, Cm = O.evaluate_constraints(blocks, v, e)
    assert G.rel(Cm, gd["C_stacked"]) <= 1e-12
    assert np.allclose(phi, gd["Phi_stacked"], atol=1e-12)
    st, g, lam, res = O.solve_constrained_gradient(v, e, blocks, np.asarray(gd["dE"]))
    assert st == 0
    assert G.rel(g, gd["g_tilde"]) <= 1e-9
    assert np.linalg.norm(lam - gd["lambda"]) / max(1, np.linalg.norm(gd["lambda"])) <= 1e-9
    assert res <= 1e-10
    kw = {}
    if projection == "frozen":
        kw["projection_mode"] = abi.PROJECTION_FROZEN
    opts = O.default_opts(**kw)
    if pen:
        opts.has_penalties = 1
        opts.penalties = O.penalties_struct(**pen)
    rc, out, s = O.line_search_step(v, e, np.asarray(gd["dE"]), np.asarray(gd["g_tilde"]), blocks, opts)
    gold = gd["line_search_step"]
    assert rc == 0 and s.accepted == 1
    assert s.tau == gold["tau"]
    assert s.projection_iterations == gold["projection_iterations"]
    assert abs(s.energy_before - gold["energy_before"]) <= 1e-12 * abs(gold["energy_before"])
    assert abs(s.energy - gold["energy_after"]) <= 1e-12 * abs(gold["energy_after"])
    assert G.rel(out, gold["vertices"]) <= 1e-9


@pytest.mark.parametrize("name", ["crossing-bary-pen-length", "helix-bary-pen-field",
                                  "junction-y-bary-pen-diff", "crossing-length-pen-combo"])
def test_penalties_vs_golden(name):
    """penalties.test.ts: penalty energy and gradient vs the oracle at 1e-12."""
    fx, gd, v, e = G.ref(name)
    pen = O.penalties_struct(**G.penalties_of(gd))
    pe = O.penalty_energy(v, e, pen)
    assert abs(pe - gd["penalty_energy_initial"]) <= 1e-12 * max(1.0, abs(gd["penalty_energy_initial"]))
    pg = O.penalty_gradient(v, e, pen)
    pgf = np.concatenate([pg[:, 0], pg[:, 1], pg[:, 2]])
    assert G.rel(pgf, gd["dE_penalty_flat"]) <= 1e-12


def test_flow_five_steps_crossing():
    """constraintSetFlow.test.ts:234: 5 accepted steps, energy decreasing, length drift bounded."""
    fx, gd, v, e = G.ref("crossing")
    x0 = O.barycenter_target(v, e)
    L0 = O.total_length(v, e)
    blocks = [{"kind": "barycenter", "target": x0}, {"kind": "totalLength", "L0": L0}]
    prev = O.energy(v, e)
    cur = v
    for _ in range(5):
        rc, cur, st, _f = O.sobolev_step(cur, e, blocks)
        assert rc == 0 and st.accepted == 1
        assert st.energy < prev
        prev = st.energy
        L1 = O.total_length(cur, e)
        assert abs(L1 - L0) <= 1e-4 * max(1.0, L1)


def test_empty_set_step():
    """constraintSetFlow.test.ts:274: k = 0 still takes an accepted descending step."""
    fx, gd, v, e = G.ref("crossing")
    rc, out, st, _f = O.sobolev_step(v, e, [])
    assert rc == 0 and st.accepted == 1
    assert st.energy < O.energy(v, e)
    assert st.projection_iterations == 0
    assert st.residual <= 1e-10


def test_isolated_vertex_singular():
    """optimizer-sobolev.test.ts:83: singular saddle -> singular_system, input echoed."""
    fx, gd, v, e = G.ref("crossing")
    v2 = np.vstack([v, [[5.0, 5.0, 5.0]]])
    x0 = O.barycenter_target(v2, e)
    rc, out, st, _f = O.sobolev_step(v2, e, [{"kind": "barycenter", "target": x0}])
    assert rc == 0 and st.accepted == 0 and st.converged == 0
    assert abi.REASONS[st.reason] == "singular_system"
    assert st.tau == 0 and np.array_equal(out, v2)


def _mulberry_system(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((n, n))
    return M + M.T + np.diag(rng.standard_normal(n))


@pytest.mark.parametrize("n", [1, 2, 5, 17, 40])
def test_dense_factorizations(n):
    """linsolveFlat.test.ts / ldlt.test.ts: reconstruction-free solve accuracy on
    symmetric indefinite systems, both factor kinds."""
    import ctypes as C
    K = _mulberry_system(n, n)
    x_true = np.linspace(-1, 1, n)
    rhs = K @ x_true
    for factor, solve in (("lu", "tpeo_lu"), ("ldlt", "tpeo_ldlt")):
        Kf = K.copy()
        piv = np.zeros(n, dtype=np.int32)
        st = getattr(O.lib(), f"{solve}_factor")(Kf.ctypes.data_as(abi.dp), n, piv.ctypes.data_as(abi.ip))
        assert st == 0
        x = np.zeros(n)
        st = getattr(O.lib(), f"{solve}_solve")(Kf.ctypes.data_as(abi.dp), n, piv.ctypes.data_as(abi.ip),
                                               rhs.ctypes.data_as(abi.dp), x.ctypes.data_as(abi.dp))
        assert st == 0
        assert np.linalg.norm(K @ x - rhs) <= 1e-10 * max(1, np.linalg.norm(rhs)), factor
    Kbad = K.copy()
    Kbad[0, n - 1] = np.nan
    piv = np.zeros(n, dtype=np.int32)
    assert O.lib().tpeo_ldlt_factor(Kbad.ctypes.data_as(abi.dp), n, piv.ctypes.data_as(abi.ip)) == \
        abi.TPE_ERR_SINGULAR
    del C


def test_constraint_backstops():
    """constraintSetM2.test.ts:211,222: NaN rows instead of throwing."""
    fx, gd, v, e = G.ref("crossing")
    phi, Cm = O.evaluate_constraints([{"kind": "edgeLengths", "ell0": [1.0]}], v, e)
    assert not np.isnan(phi[0]) and np.isnan(phi[1:]).all() and np.isfinite(Cm).all()
    phi, Cm = O.evaluate_constraints([{"kind": "point", "vertex": 999, "target": [0, 0, 0]}], v, e)
    assert np.isnan(phi).all() and (Cm == 0).all()
