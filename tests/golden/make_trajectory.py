"""Writes the FP64 descent-trajectory fixture of the V=2048 random-walk knot.

The oracle (oracle/tpe_oracle.c, the C restatement of the reference's
sobolevStepSet, src/core/optimizer.ts:231-440, pinned to the reference's golden
vectors by tests/test_oracle_golden.py) runs the trajectory on the CPU:

  curve       random-walk closed knot, V = E = 2048, seed 1 (3-D Gaussian
              steps of sigma 1/sqrt(V), closed by drift removal, total length 10)
  set         [barycenterBlock(x0), totalLengthBlock(L0)] frozen at the
              initial curve
  options     alpha 3, beta 6, eps 1e-10, analytical dE, factorMode 'ldlt',
              projectionMode 'frozen', the reference's line-search defaults
  loop        step i starts at the output of step i-1 with its energy as
              energyBefore (the app's descent loop)

Each step costs about a minute of CPU (the (3V+4)-order Bunch-Kaufman LDL^T),
so the GPU tests read the result from the committed file instead of running
the oracle there:

    python tests/golden/make_trajectory.py [--steps 20] [--V 2048]

Output: tests/golden/traj_rw<V>.npz with
  vertices[steps+1, V, 3]   x_0 .. x_steps
  field[steps, V, 3]        the descent field g~ of every step
  energy[steps+1]           E(x_0) .. E(x_steps)
  tau, accepted, projection_iterations, trials_evaluated, residual,
  gradient_l2_norm, slope, projection_phi_norm          per step
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))

from repulsive_test2_b200 import abi  # noqa: E402
from repulsive_test2_b200 import fixtures as F  # noqa: E402
import oracle_lib as O  # noqa: E402


def blocks_for(v, e):
    return [{"kind": "barycenter", "target": [float(c) for c in O.barycenter_target(v, e)]},
            {"kind": "totalLength", "L0": float(O.total_length(v, e))}]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--V", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args()
    v, e = F.random_walk_knot(args.V, seed=args.seed)
    blocks = blocks_for(v, e)
    xs, fields, energy = [v.copy()], [], [O.energy(v, e)]
    per = {k: [] for k in ("tau", "accepted", "projection_iterations", "trials_evaluated",
                           "residual", "gradient_l2_norm", "slope", "projection_phi_norm")}
    x = v.copy()
    for i in range(args.steps):
        o = O.default_opts(projection_mode=abi.PROJECTION_FROZEN, has_energy_before=1,
                           energy_before=energy[-1])
        t0 = time.perf_counter()
        rc, out, st, field = O.sobolev_step(x, e, blocks, o)
        dt = time.perf_counter() - t0
        assert rc == 0, rc
        for k in per:
            per[k].append(getattr(st, k))
        fields.append(field)
        if st.accepted:
            x = out
        xs.append(x.copy())
        energy.append(st.energy if st.accepted else energy[-1])
        print(f"step {i}: {dt:.1f} s, tau {st.tau}, accepted {st.accepted}, iters "
              f"{st.projection_iterations}, trials {st.trials_evaluated}, E {st.energy:.15g}",
              flush=True)
    out = os.path.join(HERE, f"traj_rw{args.V}.npz")
    np.savez_compressed(out, vertices=np.asarray(xs), field=np.asarray(fields),
                        energy=np.asarray(energy), edges=e,
                        **{k: np.asarray(val) for k, val in per.items()})
    print("wrote", out)


if __name__ == "__main__":
    main()
