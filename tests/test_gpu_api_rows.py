"""Entry points with no other direct test: l2CurveNorm (lineSearch.ts:53-75)
against the oracle, the phase-timing ledger (phaseTimings.ts:9-78, the checks of
the reference's test/sobolev/phaseTimings.test.ts), the device-resident step
against the host-buffer step, and the FP32-pair energy of tpe_energy_batch
against the FP64 energy."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import goldens as G
import oracle_lib as O
from repulsive_test2_b200 import abi
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("V", [5, 300, 2048])
def test_l2_curve_norm_against_oracle(V):
    v, e = F.random_walk_knot(V, seed=40 + V)
    rng = np.random.default_rng(V)
    vals = rng.standard_normal((V, 3))
    got = T.l2CurveNorm(vals, v, e)
    want = O.l2_curve_norm(vals, v, e)
    assert abs(got - want) <= 1e-13 * abs(want), (got, want)


def test_l2_curve_norm_network_against_oracle():
    # a vertex of degree 3 and an isolated vertex (mass 0)
    _, gd, v, e = G.ref("junction-y")
    v = np.vstack([v, [[5.0, 5.0, 5.0]]])
    vals = np.random.default_rng(7).standard_normal(v.shape)
    got = T.l2CurveNorm(vals, v, e)
    want = O.l2_curve_norm(vals, v, e)
    assert abs(got - want) <= 1e-13 * abs(want), (got, want)


def _crossing_set(v, e):
    return [T.barycenterBlock(T.barycenterTarget(v, e)), T.totalLengthBlock(T.totalLength(v, e))]


def test_timings_off_by_default():
    fx, _, v, e = G.ref("crossing")
    r = T.sobolevStepSet(v, e, None, _crossing_set(v, e),
                         {"alpha": fx["alpha"], "beta": fx["beta"], "epsilon": fx["epsilon"]})
    assert "timings" not in r


def test_timings_ledger_shape_and_calls():
    """Every present key is a reference phase key (or the appended 'refine'),
    ms >= 0 and calls >= 1; step.calls == 1, energy.calls >= 2 (E0 + a trial),
    assembleA.calls >= 2 (the gradient solve + a projection iterate, reassemble
    mode) and saddle.calls == assembleA.calls."""
    fx, _, v, e = G.ref("crossing")
    o = {"alpha": fx["alpha"], "beta": fx["beta"], "epsilon": fx["epsilon"], "collectTimings": True}
    t = T.sobolevStepSet(v, e, None, _crossing_set(v, e), o)["timings"]
    ref_keys = {"dE", "energy", "bHigh", "bLow", "assembleA", "expand", "saddle", "factor",
                "projection", "lineSearch", "step"}
    assert set(t) <= ref_keys | {"refine"}
    for s in t.values():
        assert s["ms"] >= 0 and s["calls"] >= 1
    assert t["step"]["calls"] == 1
    assert t["energy"]["calls"] >= 2
    assert t["assembleA"]["calls"] >= 2
    assert t["saddle"]["calls"] == t["assembleA"]["calls"]


@pytest.mark.parametrize("mode", ["reassemble", "frozen"])
def test_timings_do_not_perturb_numerics(mode):
    fx, _, v, e = G.ref("crossing")
    o = {"alpha": fx["alpha"], "beta": fx["beta"], "epsilon": fx["epsilon"], "projectionMode": mode}
    off = T.sobolevStepSet(v, e, None, _crossing_set(v, e), o)
    on = T.sobolevStepSet(v, e, None, _crossing_set(v, e), dict(o, collectTimings=True))
    assert np.array_equal(on["vertices"], off["vertices"])
    assert on["energy"] == off["energy"]
    assert on["stats"] == off["stats"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_step_equals_host_step(precision):
    import torch

    v, e = F.random_walk_knot(1024, seed=41)
    blocks = _crossing_set(v, e)
    o = {"projectionMode": "frozen", "precision": precision, "trials": 8}
    host = T.sobolevStepSet(v, e, None, blocks, o)
    ctx = T.context()
    ctx.topology(v, e)
    arr, keep = abi.make_set(blocks)
    dev = torch.device("cuda", 0)
    d_in = torch.from_numpy(v.copy()).to(dev)
    d_out = torch.zeros_like(d_in)
    st = abi.tpe_step_stats()
    oo = T._opts(o)
    ctx.check(ctx.lib.tpe_sobolev_step_device(ctx.ptr, d_in.data_ptr(), arr, len(blocks), C.byref(oo),
                                              d_out.data_ptr(), C.byref(st), None),
              "tpe_sobolev_step_device")
    assert np.array_equal(d_out.cpu().numpy(), host["vertices"])
    assert T._stats_dict(st) == host["stats"]
    # the input stays untouched
    assert np.array_equal(d_in.cpu().numpy(), v)


def test_fp32_pair_energy_error_against_fp64():
    """The FP32-pair energy (tpe_energy_batch, precision mixed): two-float
    positions, FP32 pair terms, FP64 sums. Its error against the FP64 energy on
    the random-walk knots is about 1e-7 relative (the per-term FP32 rounding of
    the dominant near-contact pairs), which is why the descent step keeps FP64
    pair terms; the bound checked here is 1e-6."""
    ctx = T.context()
    for V in (2048, 8192):
        v, e = F.random_walk_knot(V, seed=1)
        ctx.topology(v, e)
        curves = np.ascontiguousarray(np.stack([v, v * 1.001]))
        out = {}
        for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
            en = np.zeros(2)
            ctx.check(ctx.lib.tpe_energy_batch(ctx.ptr, curves.ctypes.data_as(abi.dp), 2,
                                               C.byref(T._params(3.0, 6.0, 1e-10)), prec,
                                               en.ctypes.data_as(abi.dp)), "tpe_energy_batch")
            out[prec] = en
        rel = np.abs(out[abi.PRECISION_MIXED] - out[abi.PRECISION_FP64]) / np.abs(out[abi.PRECISION_FP64])
        assert np.all(rel <= 1e-6), (V, rel)
        assert np.all(rel > 0.0)  # it is a different (lower-accuracy) evaluation
