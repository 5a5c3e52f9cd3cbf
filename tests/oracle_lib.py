"""ctypes front end of the CPU oracle (oracle/libtpe_oracle.so) for the tests.

The oracle is the checker: tests compare the CUDA library against it and pin
it to the reference's golden vectors. It is never on the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from repulsive_test2_b200 import abi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "libtpe_oracle.so")

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(ORACLE_DIR, "tpe_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    L = C.CDLL(ORACLE_SO)
    dp, ip = abi.dp, abi.ip
    sig = {
        "tpeo_js_pow": (C.c_double, [C.c_double, C.c_double]),
        "tpeo_disjoint_pairs": (C.c_int64, [ip, C.c_int32, ip, ip, C.c_int64]),
        "tpeo_energy": (C.c_double, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double]),
        "tpeo_energy_rows": (C.c_double, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double,
                                          C.c_int32, C.c_int32]),
        "tpeo_gradient": (None, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double, dp]),
        "tpeo_gradient_rows": (None, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double,
                                      C.c_int32, C.c_int32, dp]),
        "tpeo_gradient_fd": (None, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double,
                                    C.c_double, dp]),
        "tpeo_assemble_bhigh": (None, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double, dp]),
        "tpeo_assemble_blow": (None, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double, dp]),
        "tpeo_assemble_a": (None, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double, dp]),
        "tpeo_assemble_a_rows": (None, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_double, C.c_double,
                                        C.c_int32, C.c_int32, dp]),
        "tpeo_barycenter_target": (None, [dp, C.c_int32, ip, C.c_int32, dp]),
        "tpeo_total_length": (C.c_double, [dp, ip, C.c_int32]),
        "tpeo_edge_lengths": (None, [dp, ip, C.c_int32, dp]),
        "tpeo_l2_curve_norm": (C.c_double, [dp, dp, ip, C.c_int32]),
        "tpeo_constraint_rows": (C.c_int32, [C.POINTER(abi.tpe_constraint), C.c_int32, C.c_int32]),
        "tpeo_evaluate_constraint_set": (None, [C.POINTER(abi.tpe_constraint), C.c_int32, dp, C.c_int32,
                                                ip, C.c_int32, dp, dp]),
        "tpeo_block_scale": (C.c_double, [C.POINTER(abi.tpe_constraint), dp, C.c_int32, ip, C.c_int32]),
        "tpeo_lu_factor": (C.c_int32, [dp, C.c_int32, ip]),
        "tpeo_lu_solve": (C.c_int32, [dp, C.c_int32, ip, dp, dp]),
        "tpeo_ldlt_factor": (C.c_int32, [dp, C.c_int32, ip]),
        "tpeo_ldlt_solve": (C.c_int32, [dp, C.c_int32, ip, dp, dp]),
        "tpeo_solve_saddle_from_a": (C.c_int32, [dp, C.c_int32, dp, C.c_int32, dp, dp, C.c_int32, dp, dp, dp]),
        "tpeo_penalties_active": (C.c_int32, [C.POINTER(abi.tpe_penalties)]),
        "tpeo_penalty_energy": (C.c_double, [dp, C.c_int32, ip, C.c_int32, C.POINTER(abi.tpe_penalties)]),
        "tpeo_penalty_gradient": (None, [dp, C.c_int32, ip, C.c_int32, C.POINTER(abi.tpe_penalties), dp]),
        "tpeo_solve_constrained_gradient": (C.c_int32, [dp, C.c_int32, ip, C.c_int32,
                                                        C.POINTER(abi.tpe_constraint), C.c_int32,
                                                        C.POINTER(abi.tpe_step_opts), dp, dp, dp, dp]),
        "tpeo_project": (C.c_int32, [dp, C.c_int32, ip, C.c_int32, C.POINTER(abi.tpe_constraint), C.c_int32,
                                     C.POINTER(abi.tpe_step_opts), dp, dp, ip, ip, dp]),
        "tpeo_line_search_step": (C.c_int32, [dp, C.c_int32, ip, C.c_int32, dp, dp,
                                              C.POINTER(abi.tpe_constraint), C.c_int32,
                                              C.POINTER(abi.tpe_step_opts), dp, C.POINTER(abi.tpe_step_stats)]),
        "tpeo_sobolev_step": (C.c_int32, [dp, C.c_int32, ip, C.c_int32, C.POINTER(abi.tpe_constraint),
                                          C.c_int32, C.POINTER(abi.tpe_step_opts), dp,
                                          C.POINTER(abi.tpe_step_stats), dp]),
        "tpeo_default_step_opts": (None, [C.POINTER(abi.tpe_step_opts)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(abi.dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(abi.ip)


def default_opts(**kw) -> abi.tpe_step_opts:
    o = abi.tpe_step_opts()
    lib().tpeo_default_step_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def energy(v, e, alpha=3.0, beta=6.0, eps=1e-10):
    v, vp = _d(v)
    e, ep = _i(e)
    return lib().tpeo_energy(vp, len(v), ep, len(e), alpha, beta, eps)


def gradient(v, e, alpha=3.0, beta=6.0, eps=1e-10):
    v, vp = _d(v)
    e, ep = _i(e)
    g = np.zeros((len(v), 3))
    lib().tpeo_gradient(vp, len(v), ep, len(e), alpha, beta, eps, g.ctypes.data_as(abi.dp))
    return g


def gradient_fd(v, e, alpha=3.0, beta=6.0, eps=1e-10, h=1e-6):
    v, vp = _d(v)
    e, ep = _i(e)
    g = np.zeros((len(v), 3))
    lib().tpeo_gradient_fd(vp, len(v), ep, len(e), alpha, beta, eps, h, g.ctypes.data_as(abi.dp))
    return g


def assemble(v, e, which="A", alpha=3.0, beta=6.0, eps=1e-10):
    v, vp = _d(v)
    e, ep = _i(e)
    out = np.zeros((len(v), len(v)))
    fn = {"A": lib().tpeo_assemble_a, "B": lib().tpeo_assemble_bhigh, "B0": lib().tpeo_assemble_blow}[which]
    fn(vp, len(v), ep, len(e), alpha, beta, eps, out.ctypes.data_as(abi.dp))
    return out


def barycenter_target(v, e):
    v, vp = _d(v)
    e, ep = _i(e)
    x0 = np.zeros(3)
    lib().tpeo_barycenter_target(vp, len(v), ep, len(e), x0.ctypes.data_as(abi.dp))
    return x0


def total_length(v, e):
    v, vp = _d(v)
    e, ep = _i(e)
    return lib().tpeo_total_length(vp, ep, len(e))


def edge_lengths(v, e):
    v, vp = _d(v)
    e, ep = _i(e)
    out = np.zeros(len(e))
    lib().tpeo_edge_lengths(vp, ep, len(e), out.ctypes.data_as(abi.dp))
    return out


def l2_curve_norm(values, v, e):
    values, valp = _d(values)
    v, vp = _d(v)
    e, ep = _i(e)
    return lib().tpeo_l2_curve_norm(valp, vp, ep, len(e))


def evaluate_constraints(blocks, v, e):
    arr, keep = abi.make_set(blocks)
    v, vp = _d(v)
    e, ep = _i(e)
    k = lib().tpeo_constraint_rows(arr, len(blocks), len(e))
    phi = np.zeros(max(k, 1))
    Cm = np.zeros((max(k, 1), 3 * len(v)))
    lib().tpeo_evaluate_constraint_set(arr, len(blocks), vp, len(v), ep, len(e),
                                       phi.ctypes.data_as(abi.dp), Cm.ctypes.data_as(abi.dp))
    return phi[:k], Cm[:k]


def solve_saddle(A, n, Cm, rhs_top, rhs_bottom=None, factor_mode=abi.FACTOR_LDLT):
    A, Ap = _d(A)
    k = 0 if Cm is None else len(Cm)
    Cm, Cp = _d(Cm if k else np.zeros((1, 3 * n)))
    rt, rtp = _d(rhs_top)
    rb = None
    rbp = None
    if rhs_bottom is not None:
        rb, rbp = _d(rhs_bottom)
    x = np.zeros(3 * n)
    lam = np.zeros(max(k, 1))
    res = C.c_double(0)
    st = lib().tpeo_solve_saddle_from_a(Ap, n, Cp, k, rtp, rbp, factor_mode, x.ctypes.data_as(abi.dp),
                                        lam.ctypes.data_as(abi.dp), C.byref(res))
    return st, x, lam[:k], res.value


def solve_constrained_gradient(v, e, blocks, dE, opts=None):
    arr, keep = abi.make_set(blocks)
    v, vp = _d(v)
    e, ep = _i(e)
    dE, dp_ = _d(dE)
    o = opts or default_opts()
    k = lib().tpeo_constraint_rows(arr, len(blocks), len(e))
    g = np.zeros((len(v), 3))
    lam = np.zeros(max(k, 1))
    res = C.c_double(0)
    st = lib().tpeo_solve_constrained_gradient(vp, len(v), ep, len(e), arr, len(blocks), C.byref(o), dp_,
                                               g.ctypes.data_as(abi.dp), lam.ctypes.data_as(abi.dp),
                                               C.byref(res))
    return st, g, lam[:k], res.value


def line_search_step(v, e, dE, g, blocks, opts=None):
    arr, keep = abi.make_set(blocks)
    v, vp = _d(v)
    e, ep = _i(e)
    dE, dEp = _d(dE)
    g, gp = _d(g)
    o = opts or default_opts()
    out = np.zeros_like(v)
    st = abi.tpe_step_stats()
    rc = lib().tpeo_line_search_step(vp, len(v), ep, len(e), dEp, gp, arr, len(blocks), C.byref(o),
                                     out.ctypes.data_as(abi.dp), C.byref(st))
    return rc, out, st


def sobolev_step(v, e, blocks, opts=None):
    arr, keep = abi.make_set(blocks)
    v, vp = _d(v)
    e, ep = _i(e)
    o = opts or default_opts()
    out = np.zeros_like(v)
    field = np.zeros_like(v)
    st = abi.tpe_step_stats()
    rc = lib().tpeo_sobolev_step(vp, len(v), ep, len(e), arr, len(blocks), C.byref(o),
                                 out.ctypes.data_as(abi.dp), C.byref(st), field.ctypes.data_as(abi.dp))
    return rc, out, st, field


def penalties_struct(w_length=0.0, w_diff=0.0, w_field=0.0, X=(0.0, 0.0, 0.0)):
    p = abi.tpe_penalties()
    p.total_length = w_length
    p.length_diff = w_diff
    p.field_weight = w_field
    for c in range(3):
        p.field_X[c] = X[c]
    return p


def penalty_energy(v, e, pen):
    v, vp = _d(v)
    e, ep = _i(e)
    return lib().tpeo_penalty_energy(vp, len(v), ep, len(e), C.byref(pen))


def penalty_gradient(v, e, pen):
    v, vp = _d(v)
    e, ep = _i(e)
    g = np.zeros((len(v), 3))
    lib().tpeo_penalty_gradient(vp, len(v), ep, len(e), C.byref(pen), g.ctypes.data_as(abi.dp))
    return g
