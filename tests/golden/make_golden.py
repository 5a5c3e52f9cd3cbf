"""Regenerates the committed golden fixtures under tests/golden/.

Run where a checkout of the reference repository exists, naming its root in
REFERENCE_ROOT (required; there is no default); the GPU tests never run this
script, they only read the JSON files it wrote:

    REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py

Outputs
  energy_bitexact.json   the reference's test/golden.json cases (energy and
                         gradient pinned bit for bit by test/golden.test.ts)
  ref_<name>.json        one fixture + its oracle/golden/<name>.json, compacted
                         (the redundant 3V x 3V A3 matrix and the step direction
                         are dropped)
  trefoil128*.json       the seeded V=128 trefoil with N(0, 0.01^2) jitter run
                         through the reference's own Python oracles
                         (tpe_stage1_oracle.py; tpe_constraints_oracle.py in
                         length mode, reassemble and frozen), generated here
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("REFERENCE_ROOT", "")
sys.path.insert(0, REPO)

from repulsive_test2_b200 import fixtures  # noqa: E402

# (golden file stem, fixture stem)
REF_GOLDENS = [
    ("crossing", "crossing"),
    ("junction-y", "junction-y"),
    ("helix", "helix"),
    ("linked-rings", "linked-rings"),
    ("knot", "knot"),
    ("crossing-length", "crossing"),
    ("linked-rings-length", "linked-rings"),
    ("crossing-edgelengths", "crossing"),
    ("junction-y-edgelengths", "junction-y"),
    ("crossing-point", "crossing"),
    ("linked-rings-point", "linked-rings"),
    ("crossing-length-frozen", "crossing"),
    ("linked-rings-length-frozen", "linked-rings"),
    ("knot-length-frozen", "knot"),
    ("crossing-edgelengths-frozen", "crossing"),
    ("junction-y-edgelengths-frozen", "junction-y"),
    ("crossing-point-frozen", "crossing"),
    ("crossing-bary-pen-length", "crossing"),
    ("helix-bary-pen-field", "helix"),
    ("junction-y-bary-pen-diff", "junction-y"),
    ("crossing-length-pen-combo", "crossing"),
]

DROP = {"A3"}


def _load(path):
    with open(path, encoding="utf-8") as f:
        return json.load(f)


def _dump(obj, name):
    with open(os.path.join(HERE, name), "w", encoding="utf-8") as f:
        json.dump(obj, f, separators=(",", ":"), sort_keys=True)
        f.write("\n")


def _compact(golden):
    out = {k: v for k, v in golden.items() if k not in DROP}
    if "line_search_step" in out:
        out["line_search_step"] = {
            k: v for k, v in out["line_search_step"].items() if k != "direction"
        }
    return out


def main() -> int:
    if not REF or not os.path.isdir(REF):
        print("set REFERENCE_ROOT to the root of a reference checkout", file=sys.stderr)
        return 2
    _dump(_load(os.path.join(REF, "test", "golden.json")), "energy_bitexact.json")
    for gname, fname in REF_GOLDENS:
        fx = _load(os.path.join(REF, "oracle", "fixtures", f"{fname}.json"))
        gd = _load(os.path.join(REF, "oracle", "golden", f"{gname}.json"))
        _dump({"fixture": fx, "golden": _compact(gd)}, f"ref_{gname}.json")

    # Seeded V=128 trefoil (jitter sigma 0.01, seed 128) through the reference's Python oracles.
    v, e = fixtures.trefoil(128, jitter=0.01, seed=128)
    fx = {"name": "trefoil128", "vertices": v.tolist(), "edges": e.tolist(),
          "alpha": 3, "beta": 6, "epsilon": 1e-10}
    with tempfile.TemporaryDirectory() as tmp:
        fpath = os.path.join(tmp, "trefoil128.json")
        with open(fpath, "w", encoding="utf-8") as f:
            json.dump(fx, f)
        runs = [
            ("trefoil128.json", ["tpe_stage1_oracle.py"]),
            ("trefoil128-length.json", ["tpe_constraints_oracle.py", "length", "reassemble"]),
            ("trefoil128-length-frozen.json", ["tpe_constraints_oracle.py", "length", "frozen"]),
        ]
        for out_name, args in runs:
            gpath = os.path.join(tmp, out_name)
            cmd = [sys.executable, os.path.join(REF, "oracle", args[0]), fpath, gpath] + args[1:]
            subprocess.run(cmd, check=True, timeout=3600, cwd=os.path.join(REF, "oracle"))
            gd = _compact(_load(gpath))
            for big in ("B", "B0"):
                gd.pop(big, None)
            _dump({"fixture": fx, "golden": gd}, out_name)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
