"""Loaders for the committed golden fixtures (tests/golden/, written by make_golden.py)."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

STAGE1 = ["crossing", "junction-y", "helix", "linked-rings", "knot"]
# Constraint-set goldens: (name, projection mode)
SETS = [
    ("crossing-length", "reassemble"),
    ("linked-rings-length", "reassemble"),
    ("crossing-edgelengths", "reassemble"),
    ("junction-y-edgelengths", "reassemble"),
    ("crossing-point", "reassemble"),
    ("linked-rings-point", "reassemble"),
    ("crossing-length-frozen", "frozen"),
    ("linked-rings-length-frozen", "frozen"),
    ("knot-length-frozen", "frozen"),
    ("crossing-edgelengths-frozen", "frozen"),
    ("junction-y-edgelengths-frozen", "frozen"),
    ("crossing-point-frozen", "frozen"),
    ("crossing-bary-pen-length", "reassemble"),
    ("helix-bary-pen-field", "reassemble"),
    ("junction-y-bary-pen-diff", "reassemble"),
    ("crossing-length-pen-combo", "reassemble"),
]


def load(name):
    with open(os.path.join(GOLDEN_DIR, name), encoding="utf-8") as f:
        return json.load(f)


def ref(name):
    d = load(f"ref_{name}.json")
    fx = d["fixture"]
    v = np.asarray(fx["vertices"], dtype=np.float64)
    e = np.asarray(fx["edges"], dtype=np.int32)
    return fx, d["golden"], v, e


def blocks_of(golden):
    """The constraint set a golden was generated with, in its row order."""
    kinds = golden.get("block_kinds", ["barycenter"])
    out = []
    for k in kinds:
        if k == "barycenter":
            out.append({"kind": "barycenter", "target": golden["x0_barycenter_target"]})
        elif k == "totalLength":
            out.append({"kind": "totalLength", "L0": golden["L0_total_length_target"]})
        elif k == "edgeLengths":
            out.append({"kind": "edgeLengths", "ell0": golden["ell0_edge_length_targets"]})
        elif k == "point":
            out.append({"kind": "point", "vertex": golden["pin_vertex_index"],
                        "target": golden["pin_target"]})
    return out


def penalties_of(golden):
    p = golden.get("penalties")
    if not p:
        return None
    return dict(w_length=p["w_length"], w_diff=p["w_diff"], w_field=p["w_field"], X=tuple(p["X"]))


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
