"""Steps a batch of warm-bubble cases of one grid and times it (grouped launches
against every case as its own branch of the step graph):

    python -m vvm_b200.profile_batch [NX NZ CASES STEPS GROUP PRECISION]

defaults: 256 64 64 10 32 1 (64 cases of 256 x 64, ten timed steps, at most
32 cases a grouped launch, mixed precision; spectral cal_w). GROUP 0 steps
every case as its own branch. The cases differ in their bubbles. Six untimed
steps come first (the first two case by case, then the batch's step graphs);
the timed steps are bracketed by CUDA events on the batch's stream. Prints
one JSON line: ms a step, ns a cell, and the number of grouped launch groups.
"""
from __future__ import annotations

import json
import sys


def main(argv: list[str]) -> None:
    from vvm_b200.gpu import VVM_SOLVER_SPECTRAL, VVMBatch
    from vvm_b200.initial_state import warm_bubble
    a = [int(x) for x in argv]
    nx, nz, n = (a[0] if a else 256), (a[1] if len(a) > 1 else 64), (a[2] if len(a) > 2 else 64)
    steps, group, prec = (a[3] if len(a) > 3 else 10), (a[4] if len(a) > 4 else 32), (a[5] if len(a) > 5 else 1)
    sts = [warm_bubble(nx, nz, 200.0, 200.0, 1.0, amp=1.0 + 2.0 * j / n, radius=2000.0,
                       xc_frac=0.3 + 0.4 * j / n) for j in range(n)]
    b = VVMBatch([s.grid for s in sts], precision=prec, solver=VVM_SOLVER_SPECTRAL)
    b.grouping(group)
    b.upload(sts)
    b.step(6)
    b.synchronize()
    import torch
    stream = torch.cuda.ExternalStream(b.stream, device=torch.device("cuda:0"))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(steps)
    e1.record(stream)
    e1.synchronize()
    b.synchronize()
    ms = e0.elapsed_time(e1) / max(steps, 1)
    print(json.dumps({"NX": nx, "NZ": nz, "cases": n, "group": group, "precision": prec, "ms_per_step": ms,
                      "ns_per_cell": ms * 1e6 / (n * nx * nz), "grouped_launch_groups": b.grouping()}))
    b.close()


if __name__ == "__main__":
    main(sys.argv[1:])
