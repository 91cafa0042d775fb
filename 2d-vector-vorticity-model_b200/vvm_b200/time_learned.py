"""Times the learned preconditioner's network on a warm-bubble grid:

    python -m vvm_b200.time_learned [NX NZ DX REPS]

prints milliseconds per forward pass and per pass of its six tensor-core
convolutions (vvm_gpu_learned_time: REPS passes between one pair of events).
"""
from __future__ import annotations

import sys


def main(argv: list[str]) -> None:
    from vvm_b200.gpu import VVM_SOLVER_LEARNED, VVMGpu
    from vvm_b200.initial_state import warm_bubble
    nx = int(argv[0]) if len(argv) > 0 else 2048
    nz = int(argv[1]) if len(argv) > 1 else 256
    dx = float(argv[2]) if len(argv) > 2 else 100.0
    reps = int(argv[3]) if len(argv) > 3 else 20
    st = warm_bubble(nx, nz, dx, dx, 1.0)
    g = VVMGpu(st.grid, solver=VVM_SOLVER_LEARNED)
    g.upload(st)
    fwd, convs = g.learned_time(reps)
    print(f"NX={nx} NZ={nz}: forward {fwd:.4f} ms, six convolutions {convs:.4f} ms")
    g.close()


if __name__ == "__main__":
    main(sys.argv[1:])
