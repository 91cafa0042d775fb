"""Training of the learned preconditioner on the plain solver's own pairs from
the two small workloads, for use on a larger grid.

The network is fully convolutional (3x3 kernels on a 4-level U-net, weights
independent of the grid), so weights trained on one grid serve another. This
module trains them on (right-hand side, solution) pairs that the plain FP64
multigrid-PCG solver produces on

* the warm bubble at NX=128, NZ=64, dx = dz = 200 m (its own next steps'
  cal_w right-hand sides, and as many white-noise ones), then on
* the sheared squall line at NX=1024, NZ=128, dx = 250 m on stretched levels
  (dz 100 m -> 500 m, tanh ramp), the same way,

each context starting from the weights the previous one ended with, and
returns the weights (vvm_gpu_learned_weights layout) for any context, e.g.
the stretched-level Poisson workload at NX=2048, NZ=256.

    python -m vvm_b200.learned_training [pairs_each] [adam_steps_each]
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np


def workloads():
    """The two training grids (initial states), small first."""
    from vvm_b200.initial_state import squall_line, stretched_faces, warm_bubble
    return [("warm_bubble_128x64", warm_bubble(128, 64, 200.0, 200.0, 1.0)),
            ("squall_line_1024x128_stretched",
             squall_line(1024, 128, 250.0, 100.0, 2.0, zf=stretched_faces(128, 100.0, 500.0)))]


def train_on_small_workloads(pairs_each: int = 10000, steps_each: int = 2500, batch: int = 4,
                             lr: float = 2e-3, seed: int = 11, device: int = 0):
    """Trains the network on `pairs_each` pairs from each training grid
    (half the model's own steps, half white noise, all solved by the plain
    FP64 multigrid-PCG), `steps_each` Adam steps of `batch` pairs on each.
    Returns (weights, record)."""
    from vvm_b200.gpu import VVM_PREC_FP64, VVM_SOLVER_LEARNED, VVMGpu
    w = None
    rec = {"pairs": 0, "adam_steps": 0, "grids": []}
    for name, st in workloads():
        g = VVMGpu(st.grid, precision=VVM_PREC_FP64, solver=VVM_SOLVER_LEARNED, device=device)
        g.upload(st)
        if w is not None:
            g.learned_weights(w)
        t0 = time.perf_counter()
        l0, l1 = g.learned_train(npairs=pairs_each, steps=steps_each, batch=batch, lr=lr, seed=seed)
        g.synchronize()
        dt = time.perf_counter() - t0
        w = g.learned_weights()
        g.close()
        rec["pairs"] += pairs_each
        rec["adam_steps"] += steps_each
        rec["grids"].append({"grid": name, "pairs": pairs_each, "adam_steps": steps_each, "batch": batch,
                             "loss_first": l0, "loss_last": l1, "seconds": dt})
    return w, rec


if __name__ == "__main__":
    a = [int(x) for x in sys.argv[1:]]
    w, rec = train_on_small_workloads(*(a[:2] if a else ()))
    print(json.dumps(rec), flush=True)
