"""Long runs of the mixed-precision step against the FP64 GPU step:

    python -m vvm_b200.precision_runs {config2,config5} [steps]

config5: NX=8192, NZ=256, dx=dz=100 m, dt=1 s, sheared squall line, 1800 steps;
config2: NX=1024, NZ=128, dx=250 m, stretched levels dz 100 m -> 500 m (tanh
ramp, stretched_faces), dt=2 s, sheared squall line, 3600 steps. Each case runs the
mixed step (FP32 fields and stencils, FP64 Poisson residual and reductions)
with the spectral solve and with the FP32-inner / FP64-refined multigrid
PCG, against the FP64 step with multigrid PCG, and prints one JSON line with
the domain means of th, qc, qr, surface rain and kinetic energy and their
relative differences.
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np

CASES = {
    "config5": dict(NX=8192, NZ=256, dx=100.0, dz=100.0, dt=1.0, steps=1800),
    "config2": dict(NX=1024, NZ=128, dx=250.0, dz=100.0, dt=2.0, steps=3600, dz_top=500.0),
}
NAMES = ("th", "qc", "qr", "rain", "ke")


def domain_means(st) -> np.ndarray:
    """[th, qc, qr, surface rain, kinetic energy] over interior cells; kinetic
    energy is 0.5 rhou (u^2 + w^2) at the stored points."""
    f = st.fields
    inner = (slice(1, -1), slice(1, -1))
    rhou = st.prof["rhou"][None, 1:-1]
    ke = 0.5 * rhou * (f["u"][inner] ** 2 + f["w"][inner] ** 2)
    return np.array([f["th"][inner].mean(), f["qc"][inner].mean(), f["qr"][inner].mean(),
                     st.precip[1:-1].mean(), ke.mean()])


VARIANTS = ("fp64_mgpcg", "mixed_spectral", "mixed_mgpcg_refined")


def run(case: str, steps: int | None = None, variants=VARIANTS) -> dict:
    from vvm_b200.gpu import VVM_PREC_FP64, VVM_PREC_MIXED, VVM_SOLVER_MGPCG, VVM_SOLVER_SPECTRAL, VVMGpu
    from vvm_b200.initial_state import squall_line, stretched_faces
    c = CASES[case]
    n = steps or c["steps"]
    zf = stretched_faces(c["NZ"], c["dz"], c["dz_top"]) if "dz_top" in c else None
    st = squall_line(c["NX"], c["NZ"], c["dx"], c["dz"], c["dt"], zf=zf)
    out = {"case": case, "steps": n, "grid": {k: c[k] for k in ("NX", "NZ", "dx", "dz", "dt", "dz_top") if k in c}}
    means = {}
    spec = {"fp64_mgpcg": (VVM_PREC_FP64, VVM_SOLVER_MGPCG),
            "mixed_spectral": (VVM_PREC_MIXED, VVM_SOLVER_SPECTRAL),
            "mixed_mgpcg_refined": (VVM_PREC_MIXED, VVM_SOLVER_MGPCG)}
    for name in variants:
        prec, solver = spec[name]
        g = VVMGpu(st.grid, precision=prec, solver=solver)
        g.upload(st)
        t0 = time.perf_counter()
        g.step(n)
        g.synchronize()
        dt = time.perf_counter() - t0
        out.setdefault("cells", (c["NX"]) * c["NZ"])
        _, rel = g.last_solve()
        means[name] = domain_means(g.download())
        out[name] = {"wall_s": dt, "cell_steps_per_s_wall": c["NX"] * c["NZ"] * n / dt, "last_relres": rel,
                     "means": dict(zip(NAMES, means[name].tolist()))}
        g.close()
    ref = means["fp64_mgpcg"]
    for name in [v for v in variants if v != "fp64_mgpcg"]:
        out[name]["rel_diff_vs_fp64"] = {n: (abs(a - r) / abs(r) if r != 0 else None)
                                         for n, a, r in zip(NAMES, means[name].tolist(), ref.tolist())}
        out[name]["abs_diff_vs_fp64"] = dict(zip(NAMES, np.abs(means[name] - ref).tolist()))
    return out


if __name__ == "__main__":
    print(json.dumps(run(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else None)), flush=True)
