"""CPU-only checks of the C ABI: the library loads, exports every symbol that
include/tpe.h declares, and the ctypes mirror matches the C struct layouts.
No compute entry point is called (there is no GPU here)."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from repulsive_test2_b200 import abi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "tpe.h")


def header_functions():
    src = open(HEADER, encoding="utf-8").read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tpe_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(abi.LIB_PATH):
        from repulsive_test2_b200 import build
        build.build()
    return C.CDLL(abi.LIB_PATH)


def test_every_declared_symbol_is_exported(lib):
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(abi.SIGNATURES), set(names) ^ set(abi.SIGNATURES)


def test_pure_host_entry_points(lib):
    lib.tpe_abi_version.restype = C.c_int32
    assert lib.tpe_abi_version() == 1
    o = abi.tpe_step_opts()
    lib.tpe_default_step_opts(C.byref(o))
    assert o.struct_size == C.sizeof(abi.tpe_step_opts)
    assert (o.alpha, o.beta, o.epsilon, o.h) == (3.0, 6.0, 1e-10, 1e-6)
    assert (o.c1, o.shrink, o.tau0, o.tau_min) == (1e-4, 0.5, 1.0, 1e-12)
    assert (o.proj_tol_abs, o.proj_tol_rel, o.proj_max_iter) == (1e-4, 1e-4, 8)


PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "tpe.h"
#define F(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  printf("tpe_constraint %zu\ntpe_params %zu\ntpe_penalties %zu\ntpe_step_opts %zu\ntpe_step_stats %zu\n",
         sizeof(tpe_constraint), sizeof(tpe_params), sizeof(tpe_penalties), sizeof(tpe_step_opts),
         sizeof(tpe_step_stats));
  F(tpe_constraint, ell0) F(tpe_constraint, n_ell0) F(tpe_step_opts, energy_before)
  F(tpe_step_opts, penalties) F(tpe_step_opts, c1) F(tpe_step_opts, proj_max_iter)
  F(tpe_step_opts, refine_tol) F(tpe_step_stats, accepted) F(tpe_step_stats, trials_evaluated)
  return 0;
}
"""


def test_struct_layouts_match_header():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write(PROBE)
        subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line.strip())
    want = {
        "tpe_constraint": C.sizeof(abi.tpe_constraint),
        "tpe_params": C.sizeof(abi.tpe_params),
        "tpe_penalties": C.sizeof(abi.tpe_penalties),
        "tpe_step_opts": C.sizeof(abi.tpe_step_opts),
        "tpe_step_stats": C.sizeof(abi.tpe_step_stats),
        "tpe_constraint.ell0": abi.tpe_constraint.ell0.offset,
        "tpe_constraint.n_ell0": abi.tpe_constraint.n_ell0.offset,
        "tpe_step_opts.energy_before": abi.tpe_step_opts.energy_before.offset,
        "tpe_step_opts.penalties": abi.tpe_step_opts.penalties.offset,
        "tpe_step_opts.c1": abi.tpe_step_opts.c1.offset,
        "tpe_step_opts.proj_max_iter": abi.tpe_step_opts.proj_max_iter.offset,
        "tpe_step_opts.refine_tol": abi.tpe_step_opts.refine_tol.offset,
        "tpe_step_stats.accepted": abi.tpe_step_stats.accepted.offset,
        "tpe_step_stats.trials_evaluated": abi.tpe_step_stats.trials_evaluated.offset,
    }
    for k, v in want.items():
        assert int(got[k]) == v, k


def test_no_cpu_fallback_in_product():
    """The product package never imports the oracle."""
    pkg = os.path.join(REPO, "repulsive_test2_b200")
    for root, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".h", ".cpp", ".cuh")):
                txt = open(os.path.join(root, f), encoding="utf-8").read()
                assert "tpe_oracle" not in txt and "oracle_lib" not in txt, f
