"""Mixed-precision solve and batched line-search trials against the FP64 path.

The mixed mode factors the Jacobi-scaled A_rho in FP32 on the tensor cores and
restores FP64 accuracy with preconditioned CG; the pair kernels and A stay
FP64. Tolerances (the ones the mixed mode is specified to): energy relative
error <= 1e-8 and projected-gradient relative error <= 1e-6 against the FP64
step, the same accepted tau, and the CG relative residual at refineTol.
Batched trials (several step sizes projected together) must reproduce the
one-at-a-time line search exactly: same tau, bit-identical vertices.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as O
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu


def _set(v, e, per_edge=False):
    x0 = T.barycenterTarget(v, e)
    if per_edge:
        return [T.barycenterBlock(x0), T.edgeLengthsBlock(T.edgeLengths(v, e))]
    return [T.barycenterBlock(x0), T.totalLengthBlock(T.totalLength(v, e))]


def _step(v, e, blocks, **opts):
    o = {"projectionMode": "frozen", "collectField": True}
    o.update(opts)
    return T.sobolevStepSet(v, e, None, blocks, o)


# 300, 2500 and 4097 are not multiples of 128 times a power of two: the factor
# is padded to the next multiple of 128 and the inverse splits unevenly
@pytest.mark.parametrize("V", [256, 300, 1024, 2048, 2500, 4097])
def test_mixed_matches_fp64_step(V):
    v, e = F.random_walk_knot(V, seed=1)
    blocks = _set(v, e)
    r64 = _step(v, e, blocks, precision="fp64")
    r32 = _step(v, e, blocks, precision="mixed")
    assert r32["stats"]["refineIterations"] > 0  # the tensor-core factor was used
    assert r32["accepted"] == r64["accepted"]
    assert r32["stats"]["tau"] == r64["stats"]["tau"]
    g64, g32 = r64["descentField"], r32["descentField"]
    assert np.linalg.norm(g32 - g64) / np.linalg.norm(g64) <= 1e-6
    assert abs(r32["energy"] - r64["energy"]) <= 1e-8 * abs(r64["energy"])
    assert r32["stats"]["residual"] <= 1e-10
    assert np.linalg.norm(r32["vertices"] - r64["vertices"]) <= 1e-6 * np.linalg.norm(r64["vertices"])


def test_mixed_against_oracle_small():
    """Trefoil V=128 (one padded 128-block): mixed step against the FP64 oracle."""
    v, e = F.trefoil(128, jitter=0.01, seed=128)
    blocks = _set(v, e)
    r = _step(v, e, blocks, precision="mixed")
    rc, out, st, _ = O.sobolev_step(v, e, blocks, O.default_opts(projection_mode=1))
    assert rc == 0
    assert r["stats"]["refineIterations"] > 0
    assert r["stats"]["tau"] == st.tau
    assert np.linalg.norm(r["vertices"] - out) <= 1e-9 * np.linalg.norm(out)
    assert abs(r["energy"] - st.energy) <= 1e-8 * abs(st.energy)


def test_mixed_non_power_of_two_size():
    """V=300 pads to 512 with an identity block; results must not see the pad."""
    v, e = F.random_walk_knot(300, seed=5)
    blocks = _set(v, e)
    r64 = _step(v, e, blocks, precision="fp64")
    r32 = _step(v, e, blocks, precision="mixed")
    assert r32["stats"]["refineIterations"] > 0
    assert r32["stats"]["tau"] == r64["stats"]["tau"]
    g64, g32 = r64["descentField"], r32["descentField"]
    assert np.linalg.norm(g32 - g64) / np.linalg.norm(g64) <= 1e-6


def test_mixed_refine_cap_falls_back_to_fp64():
    """A CG cap of one iteration cannot reach refineTol: the step falls back to
    the FP64 factorization (refineIterations = -1) and equals the FP64 step."""
    v, e = F.random_walk_knot(512, seed=2)
    blocks = _set(v, e)
    r64 = _step(v, e, blocks, precision="fp64")
    r = _step(v, e, blocks, precision="mixed", refineMaxIter=1, refineTol=1e-14)
    assert r["stats"]["refineIterations"] == -1
    assert r["stats"]["tau"] == r64["stats"]["tau"]
    assert np.array_equal(r["vertices"], r64["vertices"])


@pytest.mark.parametrize("V,trials", [(512, 8), (2048, 4), (2048, 16)])
def test_batched_trials_reproduce_sequential(V, trials):
    """The random-walk knots reject several large step sizes (projection
    failures) before one is accepted: batching must not change any of it."""
    v, e = F.random_walk_knot(V, seed=1)
    blocks = _set(v, e)
    seq = _step(v, e, blocks, trials=1)
    bat = _step(v, e, blocks, trials=trials)
    assert seq["stats"]["tau"] < 0.5  # several trials were rejected
    assert bat["stats"]["tau"] == seq["stats"]["tau"]
    assert bat["accepted"] == seq["accepted"]
    assert bat["stats"]["projectionIterations"] == seq["stats"]["projectionIterations"]
    assert bat["energy"] == seq["energy"]
    assert np.array_equal(bat["vertices"], seq["vertices"])


def test_batched_trials_per_edge_constraints():
    v, e = F.random_walk_knot(256, seed=3)
    blocks = _set(v, e, per_edge=True)
    seq = _step(v, e, blocks, trials=1)
    bat = _step(v, e, blocks, trials=8)
    assert bat["stats"]["tau"] == seq["stats"]["tau"]
    assert np.array_equal(bat["vertices"], seq["vertices"])


@pytest.mark.parametrize("precision,V", [("mixed", 2048), ("fp64", 1024)])
def test_repeated_steps_are_bit_identical(precision, V):
    """The factorization runs on several streams (panel tails, trailing updates,
    half of the inverse, the gradient beside it) and its persistent kernels take
    tiles from counters in whatever order the GPU schedules them: the result may
    not depend on any of that."""
    v, e = F.random_walk_knot(V, seed=9)
    blocks = _set(v, e)
    runs = [_step(v, e, blocks, precision=precision) for _ in range(3)]
    for r in runs[1:]:
        assert r["energy"] == runs[0]["energy"]
        assert r["stats"]["tau"] == runs[0]["stats"]["tau"]
        assert r["stats"]["refineIterations"] == runs[0]["stats"]["refineIterations"]
        assert np.array_equal(r["vertices"], runs[0]["vertices"])
        assert np.array_equal(r["descentField"], runs[0]["descentField"])
