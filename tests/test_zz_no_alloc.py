"""tpe_energy_noalloc, the entry point for callers that cannot allocate device
memory (an application whose device memory comes only from its own pool, or a
real-time loop that must never enter the driver's allocator): it allocates
nothing and keeps its scratch in a static device array. Checked against the
regular tpe_energy on two calls in a row with different curves (the second call
reuses the scratch the first one left behind), at the largest edge count the
scratch serves, with a non-integer exponent pair, and with an edge index out of
range (NaN energy, nothing read outside the positions). Collected last so that a
failure here stops a -x run only after every other test has run."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from repulsive_test2_b200 import abi
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu

MAX_EDGES = 16384


def _noalloc(v, e, params):
    import torch

    lib = abi.load_library()
    dev = torch.device("cuda", 0)
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    dv = torch.from_numpy(np.ascontiguousarray(v)).to(dev)
    de = torch.from_numpy(np.ascontiguousarray(e, dtype=np.int32)).to(dev)
    rc = lib.tpe_energy_noalloc(dv.data_ptr(), de.data_ptr(), len(v), len(e), C.byref(params),
                                out.data_ptr(), C.c_void_p(stream.cuda_stream))
    stream.synchronize()
    return rc, float(out.item())


def test_noalloc_energy_matches_tpe_energy_twice():
    params = abi.tpe_params(3.0, 6.0, 1e-10)
    curves = [F.random_walk_knot(2048, seed=21), F.trefoil(1500, jitter=0.01, seed=22)]
    for v, e in curves:
        want = T.calculateEnergy(v, e)
        rc, got = _noalloc(v, e, params)
        assert rc == abi.TPE_OK
        assert abs(got - want) <= 1e-12 * abs(want), (got, want)


def test_noalloc_general_exponents():
    v, e = F.trefoil(700, jitter=0.01, seed=23)
    want = T.calculateEnergy(v, e, alpha=2.0, beta=4.5)
    rc, got = _noalloc(v, e, abi.tpe_params(2.0, 4.5, 1e-10))
    assert rc == abi.TPE_OK
    assert abs(got - want) <= 1e-12 * abs(want), (got, want)


def test_noalloc_at_the_edge_limit():
    v, e = F.random_walk_knot(MAX_EDGES, seed=24)
    assert len(e) == MAX_EDGES
    want = T.calculateEnergy(v, e)
    rc, got = _noalloc(v, e, abi.tpe_params(3.0, 6.0, 1e-10))
    assert rc == abi.TPE_OK
    assert abs(got - want) <= 1e-12 * abs(want), (got, want)


def test_noalloc_index_out_of_range_gives_nan():
    v, e = F.random_walk_knot(256, seed=25)
    e = e.copy()
    e[17, 1] = len(v)  # one past the last vertex: checked on the device, never loaded
    rc, got = _noalloc(v, e, abi.tpe_params(3.0, 6.0, 1e-10))
    assert rc == abi.TPE_OK and math.isnan(got)
    # the next call with valid indices is unaffected (the flag is cleared per call)
    v2, e2 = F.random_walk_knot(256, seed=26)
    rc, got = _noalloc(v2, e2, abi.tpe_params(3.0, 6.0, 1e-10))
    want = T.calculateEnergy(v2, e2)
    assert rc == abi.TPE_OK and abs(got - want) <= 1e-12 * abs(want)


def test_noalloc_rejects_oversize_without_launching():
    import torch

    lib = abi.load_library()
    dev = torch.device("cuda", 0)
    params = abi.tpe_params(3.0, 6.0, 1e-10)
    dummy = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = lib.tpe_energy_noalloc(dummy.data_ptr(), dummy.data_ptr(), MAX_EDGES + 1, MAX_EDGES + 1,
                                C.byref(params), dummy.data_ptr(), None)
    assert rc == abi.TPE_ERR_TOO_LARGE
