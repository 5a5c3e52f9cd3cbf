"""Host-side mirror of the reference's TypeScript API for the descent step.

Same names, argument meaning and failure behaviour as src/core/tangentPointEnergy.ts,
src/core/sobolev/*.ts and src/core/optimizer.ts; every call goes through the
C ABI of libtpe.so (include/tpe.h) to the CUDA implementation. There is no CPU
fallback: without the library or a CUDA device the first call raises.

Vertices are ``(V, 3)`` float arrays (``Vec3[]``), edges ``(E, 2)`` int arrays
(``Edge[]``). A constraint block is a plain dict ``{"kind": ..., target}`` --
the closure-captured target of the TypeScript ``ConstraintBlock`` made
explicit, as the FFI needs it.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Any, Dict, List, Optional, Sequence

import numpy as np

from . import abi

DEFAULTS = {"alpha": 3.0, "beta": 6.0, "epsilon": 1e-10, "h": 1e-6}  # optimizer.ts:18
SOBOLEV_CONVERGENCE_TOL = 1e-4  # optimizer.ts:78


class SingularSystemError(RuntimeError):
    """The saddle system is singular (the reference throws an Error mentioning "singular")."""


class TpeError(RuntimeError):
    pass


# ---- context management ------------------------------------------------------

class Context:
    """One libtpe context (one CUDA stream) with its topology."""

    def __init__(self, device: int = 0):
        self.lib = abi.load_library()
        st = C.c_int32(0)
        self.ptr = self.lib.tpe_create(device, C.byref(st))
        if not self.ptr:
            raise TpeError(f"tpe_create(device={device}) failed with status {st.value} "
                           "(no CUDA device?)")
        self._edges_key: Optional[bytes] = None
        self.V = 0
        self.E = 0

    def close(self):
        if self.ptr:
            self.lib.tpe_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, status: int, what: str):
        if status == abi.TPE_OK:
            return
        msg = self.lib.tpe_last_error(self.ptr)
        msg = msg.decode() if msg else ""
        if status in (abi.TPE_ERR_SINGULAR, abi.TPE_ERR_NONFINITE_INPUT):
            raise SingularSystemError(f"{what}: {msg} (treating as singular)")
        raise TpeError(f"{what} failed with status {status}: {msg}")

    def topology(self, vertices: np.ndarray, edges: np.ndarray):
        e = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1, 2))
        V = int(np.asarray(vertices).reshape(-1, 3).shape[0])
        key = e.tobytes() + V.to_bytes(8, "little")
        if key != self._edges_key:
            self.check(self.lib.tpe_set_topology(self.ptr, e.ctypes.data_as(abi.ip), len(e), V),
                       "tpe_set_topology")
            self._edges_key = key
            self.V, self.E = V, len(e)
        return e


_CTX: Optional[Context] = None


def context() -> Context:
    global _CTX
    if _CTX is None:
        _CTX = Context(0)
    return _CTX


def _v(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, 3))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(abi.dp)


def _params(alpha, beta, epsilon):
    p = abi.tpe_params()
    p.alpha, p.beta, p.epsilon = float(alpha), float(beta), float(epsilon)
    return p


# ---- tangentPointEnergy.ts ------------------------------------------------------

def calculateDisjointPairs(edges) -> List[List[int]]:
    """tangentPointEnergy.ts:33-47 (host-side listing; the kernels never need it)."""
    e = np.asarray(edges, dtype=np.int32).reshape(-1, 2)
    out = []
    for i in range(len(e)):
        a1, a2 = e[i]
        m = (e[:, 0] != a1) & (e[:, 0] != a2) & (e[:, 1] != a1) & (e[:, 1] != a2)
        m[i] = False
        out.append(np.nonzero(m)[0].tolist())
    return out


def calculateEnergy(vertices, edges, disjointPairs=None, alpha=3.0, beta=6.0, epsilon=1e-10) -> float:
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    out = C.c_double(0)
    ctx.check(ctx.lib.tpe_energy(ctx.ptr, _dp(v), C.byref(_params(alpha, beta, epsilon)), C.byref(out)),
              "calculateEnergy")
    return out.value


def energyAndGradient(vertices, edges, alpha=3.0, beta=6.0, epsilon=1e-10):
    """One FFI call: the forward energy and the adjoint gradient."""
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    g = np.zeros_like(v)
    en = C.c_double(0)
    ctx.check(ctx.lib.tpe_energy_grad(ctx.ptr, _dp(v), C.byref(_params(alpha, beta, epsilon)),
                                      C.byref(en), _dp(g)), "energyAndGradient")
    return en.value, g


def gradientAnalytical(vertices, edges, disjointPairs=None, alpha=3.0, beta=6.0, epsilon=1e-10):
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    g = np.zeros_like(v)
    ctx.check(ctx.lib.tpe_energy_grad(ctx.ptr, _dp(v), C.byref(_params(alpha, beta, epsilon)), None,
                                      _dp(g)), "gradientAnalytical")
    return g


def gradientFiniteDiff(vertices, edges, disjointPairs=None, alpha=3.0, beta=6.0, epsilon=1e-10,
                       h=1e-6):
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    g = np.zeros_like(v)
    ctx.check(ctx.lib.tpe_gradient_fd(ctx.ptr, _dp(v), C.byref(_params(alpha, beta, epsilon)), h,
                                      _dp(g)), "gradientFiniteDiff")
    return g


def energyBatch(curves: np.ndarray, edges, alpha=3.0, beta=6.0, epsilon=1e-10) -> np.ndarray:
    """Energies of several curves sharing one topology, one launch."""
    ctx = context()
    c = np.ascontiguousarray(np.asarray(curves, dtype=np.float64))
    n = c.shape[0]
    ctx.topology(c[0], edges)
    out = np.zeros(n)
    ctx.check(ctx.lib.tpe_energy_batch(ctx.ptr, _dp(c), n, C.byref(_params(alpha, beta, epsilon)),
                                       abi.PRECISION_FP64, _dp(out)), "energyBatch")
    return out


def bhEnergy(vertices, edges, alpha=3.0, beta=6.0, epsilon=1e-10, theta=0.5, leafSize=8,
             thetaT=None):
    """Barnes-Hut energy, the stage-2 oracle's bh_energy (oracle/tpe_stage2_oracle.py:532-589):
    (energy, {"visits", "approximated_edge_refs", "direct_pairs"}). thetaT defaults to
    1.5 * theta; theta = 0 is the exact energy."""
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    out = C.c_double(0.0)
    st = (C.c_int64 * 3)()
    ctx.check(ctx.lib.tpe_energy_bh(ctx.ptr, _dp(v), C.byref(_params(alpha, beta, epsilon)), float(theta),
                                    -1.0 if thetaT is None else float(thetaT), int(leafSize),
                                    C.byref(out), st), "bhEnergy")
    return out.value, {"visits": int(st[0]), "approximated_edge_refs": int(st[1]), "direct_pairs": int(st[2])}


def bctMatvec(vertices, edges, psi, kind="high", epsilon=1e-10, theta=0.5, leafSize=8, thetaT=None):
    """phi = K psi for the high- or low-order edge kernel by the block cluster tree, the
    stage-2 oracle's bct_matvec_kernel (oracle/tpe_stage2_oracle.py:649-703): (phi, {"leaves",
    "admissible_blocks", "direct_blocks", "direct_pairs"}). psi is E or E x 3."""
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    ps = np.ascontiguousarray(np.asarray(psi, dtype=np.float64))
    ncols = 1 if ps.ndim == 1 else ps.shape[1]
    phi = np.zeros_like(ps)
    st = (C.c_int64 * 4)()
    ctx.check(ctx.lib.tpe_bct_matvec(ctx.ptr, _dp(v), abi.BCT_HIGH if kind == "high" else abi.BCT_LOW,
                                     _dp(ps), ncols, float(epsilon), float(theta),
                                     -1.0 if thetaT is None else float(thetaT), int(leafSize), _dp(phi), st),
              "bctMatvec")
    return phi, {"leaves": int(st[0]), "admissible_blocks": int(st[1]), "direct_blocks": int(st[2]),
                 "direct_pairs": int(st[3])}


def bctApplyB(vertices, edges, u, kind="high", epsilon=1e-10, theta=0.5, leafSize=8, thetaT=None):
    """The high-order (B) or low-order (B0) Sobolev operator applied to a vertex function u
    through block-cluster-tree kernel products, the stage-2 oracle's bct_apply_B_scalar
    (oracle/tpe_stage2_oracle.py:742-805): low: z = (K1 y - K y) for y the edge averages of u,
    spread half to each endpoint; high: y = D u (edge differences along the unit tangents),
    z = K1 y - K y, out = D^T z; K1 = K 1. theta = 0 gives B u (B0 u) of the dense assembly
    (innerProduct.ts assembleBHighFlat / assembleBLowFlat). Returns (out, stats) with the two
    products' counts prefixed K1_ and Ky_."""
    v = _v(vertices)
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    u = np.asarray(u, dtype=np.float64)
    a, b = e[:, 0], e[:, 1]
    ed = v[b] - v[a]
    ell_raw = np.linalg.norm(ed, axis=1)
    ell_eps = ell_raw + epsilon
    T_ = np.zeros_like(ed)
    mask = ell_raw >= 1e-14
    T_[mask] = ed[mask] / ell_raw[mask, None]
    ones = np.ones(len(e))
    if kind == "low":
        y = 0.5 * (u[a] + u[b])
        K1, s1 = bctMatvec(v, e, ones, "low", epsilon, theta, leafSize, thetaT)
        Ky, s2 = bctMatvec(v, e, y, "low", epsilon, theta, leafSize, thetaT)
        z = K1 * y - Ky
        out = np.zeros(len(v))
        np.add.at(out, a, 0.5 * z)
        np.add.at(out, b, 0.5 * z)
    elif kind == "high":
        y = ((u[b] - u[a]) / ell_eps)[:, None] * T_
        K1, s1 = bctMatvec(v, e, ones, "high", epsilon, theta, leafSize, thetaT)
        Ky, s2 = bctMatvec(v, e, y, "high", epsilon, theta, leafSize, thetaT)
        z = K1[:, None] * y - Ky
        coeff = np.einsum("ij,ij->i", z, T_) / ell_eps
        out = np.zeros(len(v))
        np.add.at(out, a, -coeff)
        np.add.at(out, b, coeff)
    else:
        raise ValueError(kind)
    stats = {"K1_" + k: x for k, x in s1.items()}
    stats.update({"Ky_" + k: x for k, x in s2.items()})
    return out, stats


def mgHierarchy(vertices, edges, pinned=(), maxLevels=16, minVertices=8):
    """The stage-2 multigrid's level hierarchy (build_hierarchy / build_coarse_level,
    oracle/tpe_stage2_oracle.py:816-955), coarsened on the host by tpe_mg_coarsen: a list of
    levels, each {"vertices", "edges", "orig_vertices", "edge_paths"} and, below the finest,
    "P_to_fine" (the dense prolongation to the next finer level). pinned lists original
    vertex indices (the point constraints)."""
    lib = abi.load_library()
    v0 = _v(vertices)
    e0 = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1, 2))
    pin = np.ascontiguousarray(np.asarray(sorted(set(int(p) for p in pinned)), dtype=np.int32))
    levels = [{"vertices": v0.copy(), "edges": e0.copy(), "orig_vertices": list(range(len(v0))),
               "edge_paths": [[i] for i in range(len(e0))]}]
    while len(levels) < maxLevels:
        L = levels[-1]
        V, E = len(L["vertices"]), len(L["edges"])
        orig = np.ascontiguousarray(np.asarray(L["orig_vertices"], dtype=np.int32))
        off = np.ascontiguousarray(np.cumsum([0] + [len(p) for p in L["edge_paths"]]).astype(np.int32))
        pe = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.int32) for p in L["edge_paths"]])
                                  if E else np.zeros(1, dtype=np.int32))
        le = np.ascontiguousarray(L["edges"], dtype=np.int32)
        black = np.zeros(max(V, 1), dtype=np.int32)
        p_idx = np.zeros(max(2 * V, 1), dtype=np.int32)
        p_w = np.zeros(max(2 * V, 1))
        ce = np.zeros(max(2 * E, 2), dtype=np.int32)
        coff = np.zeros(E + 2, dtype=np.int32)
        cpe = np.zeros(max(int(off[-1]), 1), dtype=np.int32)
        vc, ec = C.c_int32(0), C.c_int32(0)
        rc = lib.tpe_mg_coarsen(V, le.ctypes.data_as(abi.ip), E, orig.ctypes.data_as(abi.ip),
                                off.ctypes.data_as(abi.ip), pe.ctypes.data_as(abi.ip),
                                pin.ctypes.data_as(abi.ip), len(pin), int(minVertices),
                                black.ctypes.data_as(abi.ip), p_idx.ctypes.data_as(abi.ip), _dp(p_w),
                                ce.ctypes.data_as(abi.ip), coff.ctypes.data_as(abi.ip),
                                cpe.ctypes.data_as(abi.ip), C.byref(vc), C.byref(ec))
        if rc != abi.TPE_OK:
            raise TpeError(f"tpe_mg_coarsen failed with status {rc}")
        if vc.value == 0:
            break
        nc, nec = vc.value, ec.value
        P = np.zeros((V, nc))
        for i in range(V):
            for s in range(2):
                if p_idx[2 * i + s] >= 0:
                    P[i, p_idx[2 * i + s]] = p_w[2 * i + s]
        blk = black[:nc]
        levels.append({"vertices": L["vertices"][blk].copy(), "edges": ce[:2 * nec].reshape(-1, 2).copy(),
                       "orig_vertices": [L["orig_vertices"][i] for i in blk],
                       "edge_paths": [cpe[coff[j]:coff[j + 1]].tolist() for j in range(nec)],
                       "P_to_fine": P})
    return levels


# ---- innerProduct.ts --------------------------------------------------------------

def _assemble(vertices, edges, which, alpha, beta, epsilon):
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    n = len(v)
    out = np.zeros((n, n))
    args = [None, None, None]
    args[{"B": 0, "B0": 1, "A": 2}[which]] = _dp(out)
    ctx.check(ctx.lib.tpe_assemble(ctx.ptr, _dp(v), C.byref(_params(alpha, beta, epsilon)), *args),
              f"assemble {which}")
    return out


def assembleBHighFlat(vertices, edges, disjointPairs=None, alpha=3.0, beta=6.0, epsilon=1e-10):
    return _assemble(vertices, edges, "B", alpha, beta, epsilon)


def assembleBLowFlat(vertices, edges, disjointPairs=None, alpha=3.0, beta=6.0, epsilon=1e-10):
    return _assemble(vertices, edges, "B0", alpha, beta, epsilon)


def assembleAFlat(vertices, edges, disjointPairs=None, alpha=3.0, beta=6.0, epsilon=1e-10):
    return _assemble(vertices, edges, "A", alpha, beta, epsilon)


# ---- constraintSet.ts / constraints.ts ---------------------------------------------

def barycenterBlock(x0) -> Dict[str, Any]:
    return {"kind": "barycenter", "target": [float(x) for x in x0]}


def totalLengthBlock(L0: float) -> Dict[str, Any]:
    return {"kind": "totalLength", "L0": float(L0)}


def edgeLengthsBlock(ell0: Sequence[float]) -> Dict[str, Any]:
    return {"kind": "edgeLengths", "ell0": [float(x) for x in ell0]}


def pointBlock(vertexIndex: int, target) -> Dict[str, Any]:
    return {"kind": "point", "vertex": int(vertexIndex), "target": [float(x) for x in target]}


def assertValidConstraintSet(set_: List[Dict[str, Any]]) -> None:
    """constraintSet.ts:333-344: totalLength and edgeLengths are mutually exclusive."""
    kinds = {b["kind"] for b in set_}
    if "totalLength" in kinds and "edgeLengths" in kinds:
        raise ValueError("ConstraintSet: totalLength and edgeLengths are mutually exclusive -- "
                         "the total-length row is exactly the sum of the edge-length rows (§3.4)")


def barycenterTarget(vertices, edges):
    """constraints.ts:23-52 (set-up, host)."""
    v = _v(vertices)
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    d = v[e[:, 1]] - v[e[:, 0]]
    ell = np.sqrt((d * d).sum(axis=1))
    tot = ell.sum()
    if tot < 1e-14:
        return v.mean(axis=0)
    return (ell[:, None] * 0.5 * (v[e[:, 0]] + v[e[:, 1]])).sum(axis=0) / tot


def totalLength(vertices, edges) -> float:
    v = _v(vertices)
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    d = v[e[:, 1]] - v[e[:, 0]]
    return float(np.sqrt((d * d).sum(axis=1)).sum())


def edgeLengths(vertices, edges):
    v = _v(vertices)
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    d = v[e[:, 1]] - v[e[:, 0]]
    return np.sqrt((d * d).sum(axis=1))


def evaluateConstraintSet(set_, vertices, edges):
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    arr, keep = abi.make_set(set_)
    k = ctx.lib.tpe_constraint_rows(ctx.ptr, arr, len(set_))
    phi = np.zeros(max(k, 1))
    Cm = np.zeros((max(k, 1), 3 * len(v)))
    ctx.check(ctx.lib.tpe_evaluate_constraints(ctx.ptr, _dp(v), arr, len(set_), _dp(phi), _dp(Cm)),
              "evaluateConstraintSet")
    return {"phi": phi[:k], "C": Cm[:k]}


# ---- lineSearch.ts / linsolve.ts / gradient.ts --------------------------------------

def l2CurveNorm(values, vertices, edges) -> float:
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    vals = _v(values)
    out = C.c_double(0)
    ctx.check(ctx.lib.tpe_l2_curve_norm(ctx.ptr, _dp(vals), _dp(v), C.byref(out)), "l2CurveNorm")
    return out.value


def solveSaddleFromA(a, n: int, Cm, rhsTop, rhsBottom=None, factorMode: str = "ldlt"):
    """linsolve.ts:742-803. Raises SingularSystemError where the reference throws."""
    ctx = context()
    A = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(n, n))
    k = 0 if Cm is None or len(Cm) == 0 else len(Cm)
    Cd = np.ascontiguousarray(np.asarray(Cm, dtype=np.float64).reshape(k, 3 * n)) if k else np.zeros((1, 3 * n))
    rt = np.ascontiguousarray(np.asarray(rhsTop, dtype=np.float64))
    rb = None if rhsBottom is None else np.ascontiguousarray(np.asarray(rhsBottom, dtype=np.float64))
    x = np.zeros(3 * n)
    lam = np.zeros(max(k, 1))
    res = C.c_double(0)
    fm = abi.FACTOR_LU if factorMode == "lu" else abi.FACTOR_LDLT
    ctx.check(ctx.lib.tpe_solve_saddle(ctx.ptr, _dp(A), n, _dp(Cd), k, _dp(rt),
                                       None if rb is None else _dp(rb), fm, _dp(x), _dp(lam),
                                       C.byref(res)), "solveSaddleFromA")
    return {"x": x, "lambda": lam[:k], "residual": res.value}


def _opts(o: Optional[Dict[str, Any]] = None, **kw) -> abi.tpe_step_opts:
    """SobolevStepOptions (optimizer.ts:95-184) plus this library's extensions
    as the C struct, starting from the library's defaults (a host-only call)."""
    op = abi.default_opts()
    d = dict(o or {})
    d.update(kw)
    if "mode" in d:
        op.mode = abi.DE_FINITE_DIFF if d["mode"] == "finiteDiff" else abi.DE_ANALYTICAL
    for k in ("alpha", "beta", "epsilon", "h"):
        if d.get(k) is not None:
            setattr(op, k, float(d[k]))
    if d.get("energyBefore") is not None:
        op.has_energy_before = 1
        op.energy_before = float(d["energyBefore"])
    if d.get("projectionMode") == "frozen":
        op.projection_mode = abi.PROJECTION_FROZEN
    if d.get("factorMode") == "lu":
        op.factor_mode = abi.FACTOR_LU
    pen = d.get("penalties")
    if pen:
        op.has_penalties = 1
        op.penalties.total_length = float(pen.get("totalLength", 0.0) or 0.0)
        op.penalties.length_diff = float(pen.get("lengthDiff", 0.0) or 0.0)
        fld = pen.get("field")
        if fld:
            op.penalties.field_weight = float(fld.get("weight", 0.0) or 0.0)
            for c in range(3):
                op.penalties.field_X[c] = float(fld["X"][c])
    for key, attr in (("c1", "c1"), ("shrink", "shrink"), ("tau0", "tau0"), ("tauMin", "tau_min")):
        if d.get(key) is not None:
            setattr(op, attr, float(d[key]))
    proj = d.get("projection") or {}
    if proj.get("tolAbs") is not None:
        op.proj_tol_abs = float(proj["tolAbs"])
    if proj.get("tolRel") is not None:
        op.proj_tol_rel = float(proj["tolRel"])
    if proj.get("maxIter") is not None:
        op.proj_max_iter = int(proj["maxIter"])
    if d.get("precision") == "mixed":
        op.precision = abi.PRECISION_MIXED
    if d.get("refineTol") is not None:
        op.refine_tol = float(d["refineTol"])
    if d.get("refineMaxIter") is not None:
        op.refine_max_iter = int(d["refineMaxIter"])
    if d.get("trials"):
        op.trials = int(d["trials"])
    if d.get("collectField"):
        op.collect_field = 1
    return op


def solveConstrainedGradientSet(vertices, edges, disjointPairs, alpha, beta, epsilon, dE, set_):
    """gradient.ts:42-65."""
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    arr, keep = abi.make_set(set_)
    k = ctx.lib.tpe_constraint_rows(ctx.ptr, arr, len(set_))
    o = _opts(alpha=alpha, beta=beta, epsilon=epsilon)
    d = _v(dE)
    g = np.zeros_like(v)
    lam = np.zeros(max(k, 1))
    res = C.c_double(0)
    ctx.check(ctx.lib.tpe_solve_constrained_gradient(ctx.ptr, _dp(v), _dp(d), arr, len(set_), C.byref(o),
                                                     _dp(g), _dp(lam), C.byref(res)),
              "solveConstrainedGradientSet")
    return {"gTilde": g, "lambda": lam[:k], "residual": res.value}


def projectOntoConstraintSet(vertices, edges, disjointPairs, alpha, beta, epsilon, set_, opts=None,
                             frozenBase=None):
    """lineSearch.ts:196-295. ``frozenBase`` (the step's base vertices) selects the
    frozen operator K(base) of solveConstrainedGradientSetFrozen."""
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    arr, keep = abi.make_set(set_)
    o = _opts(alpha=alpha, beta=beta, epsilon=epsilon, projection=opts or {})
    out = np.zeros_like(v)
    ok, it, pn = C.c_int32(0), C.c_int32(0), C.c_double(0)
    base = None if frozenBase is None else _v(frozenBase)
    ctx.check(ctx.lib.tpe_project(ctx.ptr, _dp(v), arr, len(set_), C.byref(o),
                                  None if base is None else _dp(base), _dp(out), C.byref(ok),
                                  C.byref(it), C.byref(pn)), "projectOntoConstraintSet")
    return {"vertices": out, "ok": bool(ok.value), "iterations": it.value, "phiNorm": pn.value}


def _stats_dict(st: abi.tpe_step_stats) -> Dict[str, Any]:
    return {
        "tau": st.tau,
        "residual": st.residual,
        "gradientL2Norm": st.gradient_l2_norm,
        "projectionIterations": None if st.projection_iterations < 0 else st.projection_iterations,
        **({"reason": abi.REASONS[st.reason]} if st.reason else {}),
        # extension: CG iterations of the mixed-precision solve (0 = FP64, -1 = FP64 fallback)
        "refineIterations": st.refine_iterations,
    }


def lineSearchStepSet(vertices, edges, disjointPairs, alpha, beta, epsilon, dE, gTilde, set_,
                      opts=None):
    """lineSearch.ts:423-562; opts may hold c1/shrink/tau0/tauMin/energyBefore/penalties/
    projection ({tolAbs, tolRel, maxIter}) and projectionMode ('frozen' freezes K at vertices)."""
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    arr, keep = abi.make_set(set_)
    o = _opts(opts or {}, alpha=alpha, beta=beta, epsilon=epsilon)
    out = np.zeros_like(v)
    st = abi.tpe_step_stats()
    ctx.check(ctx.lib.tpe_line_search_step(ctx.ptr, _dp(v), _dp(_v(dE)), _dp(_v(gTilde)), arr, len(set_),
                                           C.byref(o), _dp(out), C.byref(st)), "lineSearchStepSet")
    res = {
        "accepted": bool(st.accepted),
        "tau": st.tau,
        "energyBefore": st.energy_before,
        "energyAfter": st.energy,
        "vertices": out,
        "projectionIterations": None if st.projection_iterations < 0 else st.projection_iterations,
        "projectionPhiNorm": None if math.isnan(st.projection_phi_norm) else st.projection_phi_norm,
    }
    if not math.isnan(st.slope):
        res["slope"] = st.slope
    if not math.isnan(st.gradient_l2_norm):
        res["gradientL2Norm"] = st.gradient_l2_norm
    if st.reason:
        res["reason"] = abi.REASONS[st.reason]
    return res


def sobolevStepSet(vertices, edges, disjointPairs, set_, opts=None):
    """optimizer.ts:231-440: dE -> constrained saddle solve -> convergence test ->
    Armijo line search with projection. Never raises for numeric failures: those
    come back as ``stats.reason``."""
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    arr, keep = abi.make_set(set_)
    o = _opts(opts or {})
    out = np.zeros_like(v)
    st = abi.tpe_step_stats()
    timings = (C.c_double * (2 * abi.PHASE_COUNT))() if (opts or {}).get("collectTimings") else None
    field = np.zeros_like(v) if (opts or {}).get("collectField") else None
    ctx.check(ctx.lib.tpe_sobolev_step(ctx.ptr, _dp(v), arr, len(set_), C.byref(o), _dp(out), C.byref(st),
                                       timings, None if field is None else _dp(field)),
              "sobolevStepSet")
    res = {
        "vertices": out,
        "energy": st.energy,
        "accepted": bool(st.accepted),
        "converged": bool(st.converged),
        "stats": _stats_dict(st),
        "_raw": st,
    }
    if timings is not None:
        res["timings"] = {k: {"ms": timings[2 * i], "calls": int(timings[2 * i + 1])}
                          for i, k in enumerate(abi.PHASE_KEYS) if timings[2 * i + 1] > 0}
    if field is not None:
        res["descentField"] = None if st.reason == 6 else field
    return res


class Batch:
    """Many independent curves (own topology each), stepped together by
    ``tpe_step_batch``: one context per curve, curves run concurrently."""

    def __init__(self, curves, device: int = 0):
        """curves: list of (vertices, edges)."""
        self.lib = abi.load_library()
        st = C.c_int32(0)
        self.ptr = self.lib.tpe_batch_create(device, len(curves), C.byref(st))
        if not self.ptr:
            raise TpeError(f"tpe_batch_create({len(curves)} curves) failed with status {st.value}")
        self.n = len(curves)
        self.V = []
        for i, (v, e) in enumerate(curves):
            e = np.ascontiguousarray(np.asarray(e, dtype=np.int32).reshape(-1, 2))
            V = int(np.asarray(v).reshape(-1, 3).shape[0])
            self._check(i, self.lib.tpe_batch_set_topology(self.ptr, i, e.ctypes.data_as(abi.ip), len(e), V),
                        "tpe_batch_set_topology")
            self.V.append(V)

    def _check(self, i, status, what):
        if status == abi.TPE_OK:
            return
        msg = self.lib.tpe_last_error(self.lib.tpe_batch_context(self.ptr, i))
        raise TpeError(f"{what} (curve {i}) failed with status {status}: {msg.decode() if msg else ''}")

    def close(self):
        if self.ptr:
            self.lib.tpe_batch_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, vertices, sets, opts=None, max_threads: int = 0):
        """One sobolevStepSet per curve: vertices[i] (V_i x 3), sets[i] (blocks),
        opts (one dict for all curves, or a list). Returns the per-curve results
        in the form of sobolevStepSet (without timings / descent field)."""
        n = self.n
        ins = [_v(v) for v in vertices]
        outs = [np.zeros_like(v) for v in ins]
        keep = []
        arrs = (C.POINTER(abi.tpe_constraint) * n)()
        nblocks = (C.c_int32 * n)()
        for i, s_ in enumerate(sets):
            arr, k = abi.make_set(s_)
            keep.append((arr, k))
            arrs[i] = C.cast(arr, C.POINTER(abi.tpe_constraint))
            nblocks[i] = len(s_)
        olist = opts if isinstance(opts, (list, tuple)) else [opts or {}] * n
        oarr = (abi.tpe_step_opts * n)()
        for i, od in enumerate(olist):
            oarr[i] = _opts(od)
        xin = (abi.dp * n)(*[_dp(v) for v in ins])
        xout = (abi.dp * n)(*[_dp(v) for v in outs])
        stats = (abi.tpe_step_stats * n)()
        status = (C.c_int32 * n)()
        self.lib.tpe_step_batch(self.ptr, xin, arrs, nblocks, oarr, xout, stats, status, max_threads)
        res = []
        for i in range(n):
            self._check(i, status[i], "tpe_step_batch")
            st = stats[i]
            res.append({"vertices": outs[i], "energy": st.energy, "accepted": bool(st.accepted),
                        "converged": bool(st.converged), "stats": _stats_dict(st)})
        return res


def sobolevStep(vertices, edges, disjointPairs, x0, opts=None):
    """optimizer.ts:455-469: barycenter-only set."""
    return sobolevStepSet(vertices, edges, disjointPairs, [barycenterBlock(x0)], opts)


def step(vertices, edges, disjointPairs, opts):
    """optimizer.ts:37-71: one raw L2 gradient-descent step.

    grad (the device's analytic gradient when ``opts["mode"] == "analytical"``,
    else its forward-difference gradient with step ``h``), then
    ``vertices - stepSize * grad`` and the device energy of the result. Returns
    ``{"vertices", "energy"}`` plus ``"field"`` (the gradient at the input
    vertices) when ``collectField`` is set. Inputs are not modified.
    """
    def opt(key):
        val = opts.get(key)
        return DEFAULTS[key] if val is None else val

    alpha, beta, epsilon, h = opt("alpha"), opt("beta"), opt("epsilon"), opt("h")
    v = _v(vertices)
    if opts.get("mode") == "analytical":
        grad = gradientAnalytical(v, edges, disjointPairs, alpha, beta, epsilon)
    else:
        grad = gradientFiniteDiff(v, edges, disjointPairs, alpha, beta, epsilon, h)
    nxt = v - float(opts["stepSize"]) * grad
    out = {"vertices": nxt, "energy": calculateEnergy(nxt, edges, disjointPairs, alpha, beta, epsilon)}
    if opts.get("collectField"):
        out["field"] = grad
    return out


# ---- penalties.ts ---------------------------------------------------------------------

def _pen(config) -> abi.tpe_penalties:
    p = abi.tpe_penalties()
    p.total_length = float(config.get("totalLength", 0.0) or 0.0)
    p.length_diff = float(config.get("lengthDiff", 0.0) or 0.0)
    fld = config.get("field")
    if fld:
        p.field_weight = float(fld.get("weight", 0.0) or 0.0)
        for c in range(3):
            p.field_X[c] = float(fld["X"][c])
    return p


def penaltiesActive(config) -> bool:
    if not config:
        return False
    p = _pen(config)
    wf = p.field_weight
    if wf != 0.0 and math.sqrt(sum(x * x for x in p.field_X)) < 1e-14:
        wf = 0.0
    return p.total_length != 0.0 or p.length_diff != 0.0 or wf != 0.0


def penaltyEnergy(vertices, edges, config) -> float:
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    out = C.c_double(0)
    ctx.check(ctx.lib.tpe_penalty_energy(ctx.ptr, _dp(v), C.byref(_pen(config)), C.byref(out)),
              "penaltyEnergy")
    return out.value


def penaltyGradient(vertices, edges, config):
    ctx = context()
    v = _v(vertices)
    ctx.topology(v, edges)
    g = np.zeros_like(v)
    ctx.check(ctx.lib.tpe_penalty_gradient(ctx.ptr, _dp(v), C.byref(_pen(config)), _dp(g)),
              "penaltyGradient")
    return g
