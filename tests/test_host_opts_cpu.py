"""SobolevStepOptions (optimizer.ts:95-184) → tpe_step_opts on CPU: the host
mirror's option mapping and the library's defaults (a host-only entry point)."""
from __future__ import annotations

import pytest

from repulsive_test2_b200 import abi
from repulsive_test2_b200 import api as T


@pytest.fixture(scope="module", autouse=True)
def lib():
    return abi.load_library()


def test_defaults_are_the_reference_defaults():
    o = T._opts()
    assert (o.mode, o.alpha, o.beta, o.epsilon, o.h) == (abi.DE_ANALYTICAL, 3.0, 6.0, 1e-10, 1e-6)
    assert o.projection_mode == abi.PROJECTION_REASSEMBLE  # the function default (optimizer.ts)
    assert (o.c1, o.shrink, o.tau0, o.tau_min) == (1e-4, 0.5, 1.0, 1e-12)
    assert (o.proj_tol_abs, o.proj_tol_rel, o.proj_max_iter) == (1e-4, 1e-4, 8)
    assert o.precision == abi.PRECISION_FP64 and o.has_energy_before == 0 and o.has_penalties == 0
    assert (o.refine_max_iter, o.refine_tol) == (60, 1e-12)


def test_every_option_reaches_its_field():
    o = T._opts({"mode": "finiteDiff", "alpha": 2.0, "beta": 4.5, "epsilon": 1e-9, "h": 1e-5,
                 "energyBefore": 12.5, "projectionMode": "frozen", "factorMode": "lu",
                 "penalties": {"totalLength": 1.0, "lengthDiff": 10.0,
                               "field": {"weight": 5.0, "X": [0.5, 1.0, 0.0]}},
                 "c1": 1e-3, "shrink": 0.25, "tau0": 2.0, "tauMin": 1e-9,
                 "projection": {"tolAbs": 1e-10, "tolRel": 1e-11, "maxIter": 5},
                 "precision": "mixed", "refineTol": 1e-13, "refineMaxIter": 40, "trials": 4,
                 "collectField": True})
    assert (o.mode, o.alpha, o.beta, o.epsilon, o.h) == (abi.DE_FINITE_DIFF, 2.0, 4.5, 1e-9, 1e-5)
    assert o.has_energy_before == 1 and o.energy_before == 12.5
    assert o.projection_mode == abi.PROJECTION_FROZEN and o.factor_mode == abi.FACTOR_LU
    p = o.penalties
    assert o.has_penalties == 1 and (p.total_length, p.length_diff, p.field_weight) == (1.0, 10.0, 5.0)
    assert list(p.field_X) == [0.5, 1.0, 0.0]
    assert (o.c1, o.shrink, o.tau0, o.tau_min) == (1e-3, 0.25, 2.0, 1e-9)
    assert (o.proj_tol_abs, o.proj_tol_rel, o.proj_max_iter) == (1e-10, 1e-11, 5)
    assert o.precision == abi.PRECISION_MIXED and (o.refine_tol, o.refine_max_iter) == (1e-13, 40)
    assert o.trials == 4 and o.collect_field == 1


def test_keyword_options_override_the_dict():
    o = T._opts({"mode": "finiteDiff", "trials": 2}, mode="analytical", trials=6)
    assert o.mode == abi.DE_ANALYTICAL and o.trials == 6
