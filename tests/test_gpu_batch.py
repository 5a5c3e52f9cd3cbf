"""Multi-curve batch (tpe_step_batch): uneven curves stepped concurrently, one
context per curve. Every curve's result must be bit-identical to stepping it
alone with tpe_sobolev_step (same kernels on the same data), whatever the
number of host threads driving the batch."""
from __future__ import annotations

import numpy as np
import pytest

from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu


def _sets(curves, per_edge_every=0):
    sets = []
    for i, (v, e) in enumerate(curves):
        b = [T.barycenterBlock(T.barycenterTarget(v, e))]
        if per_edge_every and i % per_edge_every == per_edge_every - 1:
            b.append(T.edgeLengthsBlock(T.edgeLengths(v, e)))
        else:
            b.append(T.totalLengthBlock(T.totalLength(v, e)))
        sets.append(b)
    return sets


@pytest.mark.parametrize("threads", [1, 4, 0])
def test_batch_matches_single_steps(threads):
    curves = F.batch_curves(count=9, vmin=128, vmax=1024, seed=3)
    sets = _sets(curves, per_edge_every=4)
    opts = [{"projectionMode": "frozen", "precision": "mixed" if i % 2 else "fp64"} for i in range(len(curves))]
    b = T.Batch(curves)
    res = b.step([v for v, _ in curves], sets, opts, max_threads=threads)
    for (v, e), s, o, r in zip(curves, sets, opts, res):
        ref = T.sobolevStepSet(v, e, None, s, o)
        assert r["accepted"] == ref["accepted"]
        assert r["stats"]["tau"] == ref["stats"]["tau"]
        assert r["energy"] == ref["energy"]
        assert np.array_equal(r["vertices"], ref["vertices"])
    b.close()


def test_batch_two_steps_continue():
    """The batch keeps per-curve state apart across calls: step twice from each
    output, compare against two single steps."""
    curves = F.batch_curves(count=5, vmin=200, vmax=600, seed=8)
    sets = _sets(curves)
    o = {"projectionMode": "frozen"}
    b = T.Batch(curves)
    r1 = b.step([v for v, _ in curves], sets, o)
    r2 = b.step([r["vertices"] for r in r1], sets, o)
    for (v, e), s, x2 in zip(curves, sets, r2):
        a = T.sobolevStepSet(v, e, None, s, o)
        a2 = T.sobolevStepSet(a["vertices"], e, None, s, o)
        assert np.array_equal(x2["vertices"], a2["vertices"])
    b.close()
