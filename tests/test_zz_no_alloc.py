"""tpe_energy_noalloc, the entry point for callers that cannot allocate device
memory (for example a loop being captured into a CUDA graph, or an application
whose device memory comes only from its own pool): it allocates nothing and
keeps its scratch in a static device array. Checked against the regular
tpe_energy on two calls in a row with different curves (the second call reuses
the scratch the first one left behind). Collected last so that a failure here
stops a -x run only after every other test has run."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from repulsive_test2_b200 import abi
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F

pytestmark = pytest.mark.gpu


def test_noalloc_energy_matches_tpe_energy_twice():
    import torch

    lib = abi.load_library()
    dev = torch.device("cuda", 0)
    params = abi.tpe_params(3.0, 6.0, 1e-10)
    curves = [F.random_walk_knot(2048, seed=21), F.trefoil(1500, jitter=0.01, seed=22)]
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for v, e in curves:
        want = T.calculateEnergy(v, e)
        dv = torch.from_numpy(np.ascontiguousarray(v)).to(dev)
        de = torch.from_numpy(np.ascontiguousarray(e, dtype=np.int32)).to(dev)
        rc = lib.tpe_energy_noalloc(dv.data_ptr(), de.data_ptr(), len(v), len(e), C.byref(params),
                                    out.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert rc == abi.TPE_OK
        stream.synchronize()
        got = float(out.item())
        assert abs(got - want) <= 1e-12 * abs(want), (got, want)


def test_noalloc_rejects_oversize_without_launching():
    import torch

    lib = abi.load_library()
    dev = torch.device("cuda", 0)
    params = abi.tpe_params(3.0, 6.0, 1e-10)
    dummy = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = lib.tpe_energy_noalloc(dummy.data_ptr(), dummy.data_ptr(), 20000, 20000, C.byref(params),
                                dummy.data_ptr(), None)
    assert rc == abi.TPE_ERR_TOO_LARGE
