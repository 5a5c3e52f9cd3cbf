"""ctypes mirror of include/tpe.h and the loader for the in-tree libtpe.so.

The library is loaded from this package directory only; there is no fallback.
If libtpe.so is missing, or cannot be loaded, or reports no CUDA device,
``load_library`` raises -- nothing on the product path computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtpe.so")

# ---- status / reason / enum values (tpe.h) ---------------------------------
TPE_OK = 0
TPE_ERR_BAD_ARG = 1
TPE_ERR_CUDA = 2
TPE_ERR_SINGULAR = 3
TPE_ERR_NONFINITE_INPUT = 4
TPE_ERR_NO_TOPOLOGY = 5
TPE_ERR_OUT_OF_MEMORY = 6
TPE_ERR_INVALID_SET = 7
TPE_ERR_REFINE_NOT_CONVERGED = 8
TPE_ERR_DEVICE_TIMEOUT = 9
TPE_ERR_TOO_LARGE = 10
TPE_ERR_INTERNAL = 11

REASONS = {
    0: None,
    1: "zero_or_nonfinite_gradient_norm",
    2: "not_a_descent_direction",
    3: "armijo_failed",
    4: "projection_failed",
    5: "tau_below_min",
    6: "singular_system",
}

BLOCK_BARYCENTER, BLOCK_TOTAL_LENGTH, BLOCK_EDGE_LENGTHS, BLOCK_POINT = 0, 1, 2, 3
BLOCK_KINDS = {"barycenter": 0, "totalLength": 1, "edgeLengths": 2, "point": 3}
DE_ANALYTICAL, DE_FINITE_DIFF = 0, 1
PROJECTION_REASSEMBLE, PROJECTION_FROZEN = 0, 1
FACTOR_LDLT, FACTOR_LU = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
GEMM_FP64, GEMM_INT8_EMULATED = 0, 1
BCT_HIGH, BCT_LOW = 0, 1

PHASE_KEYS = ["dE", "energy", "bHigh", "bLow", "assembleA", "expand", "saddle", "factor",
              "projection", "lineSearch", "step", "refine"]
PHASE_COUNT = len(PHASE_KEYS)


class tpe_constraint(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("vertex", C.c_int32),
        ("target", C.c_double * 3),
        ("L0", C.c_double),
        ("ell0", C.POINTER(C.c_double)),
        ("n_ell0", C.c_int32),
        ("reserved", C.c_int32),
    ]


class tpe_params(C.Structure):
    _fields_ = [("alpha", C.c_double), ("beta", C.c_double), ("epsilon", C.c_double)]


class tpe_penalties(C.Structure):
    _fields_ = [
        ("total_length", C.c_double),
        ("length_diff", C.c_double),
        ("field_weight", C.c_double),
        ("field_X", C.c_double * 3),
    ]


class tpe_step_opts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32),
        ("mode", C.c_int32),
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("epsilon", C.c_double),
        ("h", C.c_double),
        ("has_energy_before", C.c_int32),
        ("projection_mode", C.c_int32),
        ("energy_before", C.c_double),
        ("factor_mode", C.c_int32),
        ("has_penalties", C.c_int32),
        ("penalties", tpe_penalties),
        ("c1", C.c_double),
        ("shrink", C.c_double),
        ("tau0", C.c_double),
        ("tau_min", C.c_double),
        ("proj_tol_abs", C.c_double),
        ("proj_tol_rel", C.c_double),
        ("proj_max_iter", C.c_int32),
        ("precision", C.c_int32),
        ("trials", C.c_int32),
        ("collect_field", C.c_int32),
        ("refine_max_iter", C.c_int32),
        ("reserved", C.c_int32),
        ("refine_tol", C.c_double),
    ]


class tpe_step_stats(C.Structure):
    _fields_ = [
        ("energy", C.c_double),
        ("energy_before", C.c_double),
        ("tau", C.c_double),
        ("residual", C.c_double),
        ("gradient_l2_norm", C.c_double),
        ("slope", C.c_double),
        ("projection_phi_norm", C.c_double),
        ("accepted", C.c_int32),
        ("converged", C.c_int32),
        ("projection_iterations", C.c_int32),
        ("reason", C.c_int32),
        ("refine_iterations", C.c_int32),
        ("trials_evaluated", C.c_int32),
    ]


dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)
vp = C.c_void_p

# name -> (restype, argtypes): every symbol declared in include/tpe.h.
SIGNATURES = {
    "tpe_abi_version": (C.c_int32, []),
    "tpe_default_step_opts": (None, [C.POINTER(tpe_step_opts)]),
    "tpe_create": (vp, [C.c_int32, ip]),
    "tpe_destroy": (None, [vp]),
    "tpe_last_error": (C.c_char_p, [vp]),
    "tpe_set_topology": (C.c_int32, [vp, ip, C.c_int32, C.c_int32]),
    "tpe_disjoint_pairs": (C.c_int32, [vp, ip, ip, C.c_int64]),
    "tpe_energy": (C.c_int32, [vp, dp, C.POINTER(tpe_params), dp]),
    "tpe_energy_grad": (C.c_int32, [vp, dp, C.POINTER(tpe_params), dp, dp]),
    "tpe_gradient_fd": (C.c_int32, [vp, dp, C.POINTER(tpe_params), C.c_double, dp]),
    "tpe_assemble": (C.c_int32, [vp, dp, C.POINTER(tpe_params), dp, dp, dp]),
    "tpe_constraint_rows": (C.c_int32, [vp, C.POINTER(tpe_constraint), C.c_int32]),
    "tpe_evaluate_constraints": (C.c_int32, [vp, dp, C.POINTER(tpe_constraint), C.c_int32, dp, dp]),
    "tpe_l2_curve_norm": (C.c_int32, [vp, dp, dp, dp]),
    "tpe_solve_saddle": (C.c_int32, [vp, dp, C.c_int32, dp, C.c_int32, dp, dp, C.c_int32, dp, dp, dp]),
    "tpe_solve_constrained_gradient": (C.c_int32, [vp, dp, dp, C.POINTER(tpe_constraint), C.c_int32,
                                                   C.POINTER(tpe_step_opts), dp, dp, dp]),
    "tpe_project": (C.c_int32, [vp, dp, C.POINTER(tpe_constraint), C.c_int32, C.POINTER(tpe_step_opts),
                                dp, dp, ip, ip, dp]),
    "tpe_line_search_step": (C.c_int32, [vp, dp, dp, dp, C.POINTER(tpe_constraint), C.c_int32,
                                         C.POINTER(tpe_step_opts), dp, C.POINTER(tpe_step_stats)]),
    "tpe_sobolev_step": (C.c_int32, [vp, dp, C.POINTER(tpe_constraint), C.c_int32,
                                     C.POINTER(tpe_step_opts), dp, C.POINTER(tpe_step_stats), dp, dp]),
    "tpe_penalty_energy": (C.c_int32, [vp, dp, C.POINTER(tpe_penalties), dp]),
    "tpe_penalty_gradient": (C.c_int32, [vp, dp, C.POINTER(tpe_penalties), dp]),
    "tpe_energy_batch": (C.c_int32, [vp, dp, C.c_int32, C.POINTER(tpe_params), C.c_int32, dp]),
    "tpe_bct_matvec": (C.c_int32, [vp, dp, C.c_int32, dp, C.c_int32, C.c_double, C.c_double, C.c_double,
                                   C.c_int32, dp, C.POINTER(C.c_int64)]),
    "tpe_mg_coarsen": (C.c_int32, [C.c_int32, ip, C.c_int32, ip, ip, ip, ip, C.c_int32, C.c_int32, ip, ip, dp,
                                   ip, ip, ip, ip, ip]),
    "tpe_edge_tree": (C.c_int32, [dp, C.c_int32, ip, C.c_int32, C.c_double, C.c_int32, C.c_int32, dp, ip, ip,
                                  ip]),
    "tpe_energy_bh": (C.c_int32, [vp, dp, C.POINTER(tpe_params), C.c_double, C.c_double, C.c_int32, dp,
                                  C.POINTER(C.c_int64)]),
    "tpe_sobolev_step_device": (C.c_int32, [vp, C.c_void_p, C.POINTER(tpe_constraint), C.c_int32,
                                            C.POINTER(tpe_step_opts), C.c_void_p,
                                            C.POINTER(tpe_step_stats), dp]),
    "tpe_stream": (C.c_void_p, [vp]),
    "tpe_gemm_nt_device": (C.c_int32, [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                       C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                       C.c_double, C.c_double, C.c_int32]),
    "tpe_energy_noalloc": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(tpe_params),
                                       C.c_void_p, C.c_void_p]),
    "tpe_profile": (C.c_int32, [vp, C.c_int32]),
    "tpe_batch_create": (vp, [C.c_int32, C.c_int32, ip]),
    "tpe_batch_destroy": (None, [vp]),
    "tpe_batch_context": (vp, [vp, C.c_int32]),
    "tpe_batch_set_topology": (C.c_int32, [vp, C.c_int32, ip, C.c_int32, C.c_int32]),
    "tpe_step_batch": (C.c_int32, [vp, C.POINTER(dp), C.POINTER(C.POINTER(tpe_constraint)), ip,
                                   C.POINTER(tpe_step_opts), C.POINTER(dp), C.POINTER(tpe_step_stats), ip,
                                   C.c_int32]),
    "tpe_profile_read": (C.c_int32, [vp, dp, C.POINTER(C.c_int64)]),
}

KGROUPS = ["energy", "gradient", "pair_weights", "gather_A", "cholesky", "trsv", "other"]

_LIB = None


def load_library(path: str = LIB_PATH):
    """Load libtpe.so (no fallback: raises if it is absent or unloadable)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(
            f"libtpe.so not found at {path}; build it with `python __graft_entry__.py build` "
            "(the CUDA library is the only implementation of this path)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def default_opts(lib=None) -> tpe_step_opts:
    o = tpe_step_opts()
    (lib or load_library()).tpe_default_step_opts(C.byref(o))
    return o


def make_set(blocks):
    """blocks: list of dicts {kind, target/x0, L0, ell0, vertex}. Returns
    (ctypes array, keepalive list)."""
    arr = (tpe_constraint * max(1, len(blocks)))()
    keep = []
    for i, b in enumerate(blocks):
        kind = b["kind"]
        kind = BLOCK_KINDS[kind] if isinstance(kind, str) else int(kind)
        arr[i].kind = kind
        arr[i].vertex = int(b.get("vertex", 0))
        tgt = b.get("target", b.get("x0", (0.0, 0.0, 0.0)))
        for c in range(3):
            arr[i].target[c] = float(tgt[c])
        arr[i].L0 = float(b.get("L0", float("nan")))
        ell0 = b.get("ell0")
        if ell0 is not None:
            buf = (C.c_double * max(1, len(ell0)))(*[float(x) for x in ell0])
            keep.append(buf)
            arr[i].ell0 = C.cast(buf, dp)
            arr[i].n_ell0 = len(ell0)
        else:
            arr[i].ell0 = None
            arr[i].n_ell0 = 0
    return arr, keep
