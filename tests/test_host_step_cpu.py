"""Host logic of the raw gradient step (optimizer.ts:37-71) on CPU.

The device calls it composes (gradient, energy) are replaced by the oracle here,
as the checker; the GPU test of the same function runs them on the device."""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as O
from repulsive_test2_b200 import api as T
from repulsive_test2_b200 import fixtures as F


@pytest.fixture
def oracle_device(monkeypatch):
    calls = []

    def grad_an(v, e, dp, a, b, eps):
        calls.append(("analytical", a, b, eps))
        return O.gradient(v, e, a, b, eps)

    def grad_fd(v, e, dp, a, b, eps, h):
        calls.append(("finiteDiff", a, b, eps, h))
        return O.gradient_fd(v, e, a, b, eps, h)

    def energy(v, e, dp, a, b, eps):
        calls.append(("energy", a, b, eps))
        return O.energy(v, e, a, b, eps)

    monkeypatch.setattr(T, "gradientAnalytical", grad_an)
    monkeypatch.setattr(T, "gradientFiniteDiff", grad_fd)
    monkeypatch.setattr(T, "calculateEnergy", energy)
    return calls


@pytest.mark.parametrize("mode", ["analytical", "finiteDiff", "anything else"])
def test_step_dispatch_and_arithmetic(oracle_device, mode):
    v, e = F.trefoil(32, jitter=0.01, seed=5)
    v0 = v.copy()
    r = T.step(v, e, None, {"mode": mode, "stepSize": 1e-3, "collectField": True})
    kind = "analytical" if mode == "analytical" else "finiteDiff"
    assert oracle_device[0][0] == kind and oracle_device[1][0] == "energy"
    # the reference's defaults (optimizer.ts:18) when the options leave them out
    assert oracle_device[0][1:4] == (3.0, 6.0, 1e-10)
    if kind == "finiteDiff":
        assert oracle_device[0][4] == 1e-6
    g = r["field"]
    assert np.array_equal(r["vertices"], v0 - 1e-3 * g)
    assert r["energy"] == O.energy(r["vertices"], e)
    assert np.array_equal(v, v0)


def test_step_options_and_field(oracle_device):
    v, e = F.trefoil(32, jitter=0.01, seed=6)
    r = T.step(v, e, None, {"mode": "finiteDiff", "stepSize": 0.5, "alpha": 2.0, "beta": 4.5,
                            "epsilon": 1e-9, "h": 1e-5})
    assert "field" not in r
    assert oracle_device[0] == ("finiteDiff", 2.0, 4.5, 1e-9, 1e-5)
    assert oracle_device[1] == ("energy", 2.0, 4.5, 1e-9)
