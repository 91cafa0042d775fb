"""Runs the warm-bubble step for profiling (ncu launch lists and captures):

    python -m vvm_b200.profile_step [NX NZ DX PRECISION SOLVER STEPS]

defaults: 2048 256 100 1 2 3 (mixed precision, spectral cal_w, three steps:
the first two run the host loop, from the third the step runs as a CUDA
graph). Prints the last solve's iterations and residual.
"""
from __future__ import annotations

import sys


def main(argv: list[str]) -> None:
    from vvm_b200.gpu import VVMGpu
    from vvm_b200.initial_state import warm_bubble
    a = [float(x) for x in argv]
    nx, nz, dx = (int(a[0]) if a else 2048), (int(a[1]) if len(a) > 1 else 256), (a[2] if len(a) > 2 else 100.0)
    prec, solver, steps = (int(a[3]) if len(a) > 3 else 1), (int(a[4]) if len(a) > 4 else 2), (int(a[5]) if len(a) > 5 else 3)
    st = warm_bubble(nx, nz, dx, dx, 1.0)
    g = VVMGpu(st.grid, precision=prec, solver=solver)
    g.upload(st)
    g.step(steps)
    g.synchronize()
    print("last solve", g.last_solve())
    g.close()


if __name__ == "__main__":
    main(sys.argv[1:])
