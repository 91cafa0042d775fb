"""Benchmark of the VVM time step on B200 (one JSON line on stdout).

Workload: the warm-bubble VVM step (Kessler warm rain, turbulence, nudging,
anelastic w-equation solved to ||b - A W|| / ||b|| <= 1e-10) on an
NX=2048 x NZ=256 grid, dx = dz = 100 m, dt = 1 s, synthetic seeded initial
state (theta = 300 K + 3 K/km, 80 % RH, +2 K cosine bubble of radius 2 km).
A "step" is one call of the reference's TimeMarching body.

Our arm (default): the headline `value` is the step at the reference's
precision, FP64 throughout, with the cal_w solve by the exact Fourier-mode
solve in FP64, residual-checked against 1e-10, CG only if the check fails
(VVM_SOLVER_SPECTRAL). The plain FP64 multigrid-PCG step is timed the same
way (`plain_fp64`). The mixed-precision step (FP32 fields and stencils, FP64
Kessler arithmetic, residual, refinement and reductions) is reported under
`mixed`, with its accuracy after 600 steps against the FP64 step on the same
grid (domain-mean th and qc within 1e-4 relative is its bar). Every timed step
is bracketed by CUDA events on the stream the library launches on; L2 is
flushed (a 256 MB write) between timed steps, outside the timed windows.
`e2e` repeats the headline through the C ABI with the prognostic fields
copied from pinned host memory before and back after every step.

Reference arm (--impl reference): the reference's own TimeMarching, built from
its sources into oracle/_ref/libvvmref.so (serial: its OpenMP loops race, so
only the serial build computes the reference's numbers, and the Eigen solve
that is 99 % of its step runs on one thread either way), on the same grid and
initial state; each step is one full-grid reference step.

Multi-GPU (torchrun): one independent replica per GPU ("replicas only": one
2D domain does not shard), max time over ranks, value = all ranks' cell-steps
per second. The `ensemble` object measures the batched-ensemble workload, 256
independent cases of uneven grids in one CUDA graph a step, split over the
ranks by cost (strong scaling: the ensemble is fixed).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
for p in (str(REPO / "2d-vector-vorticity-model_b200"), str(REPO)):
    if p not in sys.path:
        sys.path.insert(0, p)

NX, NZ, DX, DT = 2048, 256, 100.0, 1.0
METRIC = "cell-steps/s"
WORKLOAD = "VVM warm-bubble step, Kessler + turbulence, NX=2048 NZ=256 dx=dz=100 m dt=1 s"


def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons every 200 ms."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons)}


# ------------------------------------------------------------- byte model

def class_bytes(cls: str, launches: int, grid, elem: int, cg_iters: float) -> float:
    """Algorithmic (compulsory) bytes of `launches` launches of a kernel class:
    each array a kernel must read or write touched once. cells = nx*nz of one
    field; unknowns = NX*(NZ-1) of the elliptic problem."""
    cells = grid.nx * grid.nz
    unk = grid.NX * (grid.NZ - 1)
    per_launch = {
        "pzeta": 12 * cells * elem,        # zeta u w th qv qc qr + 2 old hist in; zetap + 2 hist out
        "padv": 20 * cells * elem,         # u w + 4 fields + 5 old hist in; 4 fields + 5 hist out
        "apply": 8 * cells * elem,         # 4 fields in place
        "kessler": 12 * cells * elem,      # 4 in, 4 out, 4 rates out
        "rkm": 5 * cells * elem,           # u w thp in; RKM RKH out
        "gs": 12 * cells * elem,           # per STEP, not per launch: 5 fields read
                                           # and written in place + RKM, RKH (the
                                           # tile passes' count varies, 3 typical)
        "cal_u": 3 * cells * elem / 2,     # w zetap in, u out (two launches)
    }
    if cls in per_launch:
        return per_launch[cls] * launches
    if cls == "mg_sweep":
        # one V-cycle: pre-sweeps read f, write x (2 arrays); post-sweeps read
        # f, x, half a coarse array, write y (3.5 arrays); fine levels halve
        nfine, total, n = 0, 0.0, grid.NX
        while n > 32 and n % 2 == 0:
            total += 5.5 * (grid.NZ - 1) * n * elem
            nfine += 1
            n //= 2
        return total / max(2 * nfine, 1) * launches
    if cls == "cg":
        # per iteration: spmv 2, update 6, dot 2, direction 3 arrays of the unknowns
        return 13 * unk * elem * cg_iters
    return float("nan")


# ----------------------------------------------------------------- our arm

GRAPH_WARMUP = 4   # steps until both of a context's step graphs exist


def timed_steps(torch, g, steps, flush):
    import torch as T
    st = T.cuda.current_stream()
    times = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = T.cuda.Event(enable_timing=True), T.cuda.Event(enable_timing=True)
        e0.record(st)
        g.step(1)
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def run_variant(torch, precision, solver, steps, warmup, flush, device):
    from vvm_b200.gpu import VVMGpu
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(NX, NZ, DX, DX, DT)
    g = VVMGpu(st.grid, precision=precision, solver=solver, device=device)
    g.set_stream(torch.cuda.current_stream().cuda_stream)
    g.upload(st)
    # at least GRAPH_WARMUP untimed steps: a step runs as one of two CUDA
    # graphs (one per step parity), each captured on its first use
    g.step(max(warmup, GRAPH_WARMUP))
    g.synchronize()
    n0 = g.launch_count
    times = timed_steps(torch, g, steps, flush)
    launches = g.launch_count - n0
    it, rel = g.last_solve()
    # per-kernel-class device time over two more steps (events around launches)
    g.profile(True)
    g.step(2)
    prof = g.profile_read()
    g.profile(False)
    return g, st, times, launches, prof, it, rel


PER_STEP_CLASSES = ("gs",)   # byte model per step: the launches a step vary


def roofline(prof, grid, elem, hbm, peak_kind, iters_per_step, steps=2):
    """The dominant kernel class over `steps` profiled steps: algorithmic bytes
    over its event-timed device time."""
    cls, (ms, n) = max(prof.items(), key=lambda kv: kv[1][0])
    nbytes = class_bytes(cls, steps if cls in PER_STEP_CLASSES else n, grid, elem, iters_per_step * 2)
    achieved = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else None
    traffic = None
    tf = REPO / "profiles" / "roofline_traffic.txt"
    if tf.exists():
        for ln in tf.read_text().splitlines():
            f = ln.split()
            if len(f) >= 3 and f[0] == cls and f[1] == ("fp32" if elem == 4 else "fp64"):
                traffic = float(f[2])
    per_step = cls in PER_STEP_CLASSES
    return {"kernel": cls, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": (achieved / hbm) if achieved else None, "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": nbytes / max(n, 1), "avg_launch_us": 1e3 * ms / max(n, 1),
            "launches": n, "traffic": traffic,
            "per": "step" if per_step else "launch",
            "algorithmic_bytes_per_step": nbytes / steps if per_step else None,
            "us_per_step": 1e3 * ms / steps}


def cpu_baseline(sample_s=10.0):
    """The CPU baseline on the box's host cores: the C restatement of the step
    built race-free with OpenMP on every host thread and with FFT-based cal_w
    (oracle/_build/libvvmoracle_mt.so), timed over about `sample_s` seconds of
    full-grid steps; beside it, one full-grid step of the reference's own
    serial build (its OpenMP loops share temporaries between threads, so only
    the serial build computes the reference's results)."""
    from oracle.models import PortMTModel, RefModel, port_mt_available, ref_available
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(NX, NZ, DX, DX, DT)
    out = {}
    if port_mt_available():
        m = PortMTModel(st.grid)
        m.load(st)
        m.one_step()                      # warm-up (page-in, thread team)
        t0 = time.perf_counter()
        n = 0
        while n < 3 or time.perf_counter() - t0 < sample_s:
            m.one_step()
            n += 1
        dt = time.perf_counter() - t0
        out = {"value": NX * NZ * n / dt, "unit": METRIC, "cores": m.threads(), "kind": "port",
               "sample": f"{n} full-grid steps of the same workload after one warm-up step, "
                         f"{dt:.1f} s: the C restatement with OpenMP loops (race-free: "
                         f"iteration-local temporaries, per-thread sums, the five Gauss-Seidel "
                         f"sweeps concurrent) and radix-2 FFT cal_w"}
        m.close()
    if ref_available():
        r = RefModel(st.grid)
        r.load(st)
        t0 = time.perf_counter()
        r.one_step()
        dt = time.perf_counter() - t0
        ref = {"value": NX * NZ / dt, "unit": METRIC, "cores": 1, "kind": "reference",
               "sample": f"1 full-grid step of the reference's serial build, {dt:.1f} s"}
        if out:
            out["reference_serial"] = ref
        else:
            out = ref
    return out


def mixed_accuracy(steps=600):
    """Domain means of the mixed-precision step (spectral solve) after
    `steps` steps of the headline workload against the FP64 multigrid-PCG
    step from the same initial state: relative differences of th, qc, qr,
    surface rain and kinetic energy (the bar: th and qc within 1e-4)."""
    from vvm_b200.gpu import VVM_PREC_FP64, VVM_PREC_MIXED, VVM_SOLVER_MGPCG, VVM_SOLVER_SPECTRAL, VVMGpu
    from vvm_b200.initial_state import warm_bubble
    from vvm_b200.precision_runs import NAMES, domain_means
    st = warm_bubble(NX, NZ, DX, DX, DT)
    means = {}
    for name, prec, solver in (("fp64", VVM_PREC_FP64, VVM_SOLVER_MGPCG),
                               ("mixed", VVM_PREC_MIXED, VVM_SOLVER_SPECTRAL)):
        g = VVMGpu(st.grid, precision=prec, solver=solver)
        g.upload(st)
        g.step(steps)
        means[name] = domain_means(g.download())
        g.close()
    rel = {n: (abs(a - r) / abs(r) if r != 0 else None)
           for n, a, r in zip(NAMES, means["mixed"].tolist(), means["fp64"].tolist())}
    return {"steps": steps, "against": "FP64 step, multigrid-PCG, same grid and initial state",
            "rel_diff": rel, "fp64_means": dict(zip(NAMES, means["fp64"].tolist())),
            "bar": "th and qc within 1e-4 relative",
            "meets_bar": bool(rel["th"] is not None and rel["qc"] is not None
                              and rel["th"] <= 1e-4 and rel["qc"] <= 1e-4)}


def our_arm(args, rank, world, device):
    import torch
    torch.cuda.set_device(device)
    # an explicit stream: the library and the timing events must share it
    # (handle 0, the legacy stream, would hand the library its own stream)
    torch.cuda.set_stream(torch.cuda.Stream(device=device))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{device}")  # 256 MB > L2
    from vvm_b200.gpu import (VVM_PREC_FP64, VVM_PREC_MIXED, VVM_SOLVER_MGPCG,
                              VVM_SOLVER_SPECTRAL)
    hbm, peak_kind = peaks()
    results = {}
    variants = (("fp64_spectral", VVM_PREC_FP64, VVM_SOLVER_SPECTRAL),
                ("fp64_mgpcg", VVM_PREC_FP64, VVM_SOLVER_MGPCG),
                ("mixed_spectral", VVM_PREC_MIXED, VVM_SOLVER_SPECTRAL),
                ("mixed_mgpcg", VVM_PREC_MIXED, VVM_SOLVER_MGPCG))
    with ClockSampler(device) as clk:
        for name, prec, solver in variants:
            if dist_on():
                dist_barrier()
            g, st, times, launches, prof, it, rel = run_variant(torch, prec, solver, args.steps,
                                                                 args.warmup, flush, device)
            results[name] = dict(g=g, st=st, times=times, launches=launches, prof=prof, it=it, rel=rel)
            if name != "fp64_spectral":
                g.close()
                results[name]["g"] = None
    clocks = clk.summary()
    head = results["fp64_spectral"]
    cells = NX * NZ
    vms = {name: dist_max(sum(r["times"])) for name, r in results.items()}
    value, total_ms = whole_job_rate(sum(head["times"]), world, cells, args.steps)
    fp64_value, fp64_ms = whole_job_rate(sum(results["fp64_mgpcg"]["times"]), world, cells, args.steps)
    mixed_value, mixed_ms = whole_job_rate(sum(results["mixed_spectral"]["times"]), world, cells, args.steps)

    # e2e through the C ABI with host buffers (pinned) copied in and out each step
    g = head["g"]
    import torch as T
    pinned = {n: T.empty((st_nx(), st_nz()), dtype=T.float64).pin_memory().numpy()
              for n in ("zeta", "th", "qv", "qc", "qr", "u", "w")}
    g.download_prognostic(pinned)
    stream = T.cuda.current_stream()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = T.cuda.Event(enable_timing=True), T.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.upload_prognostic(pinned)
        g.step(1)
        g.download_prognostic(pinned)
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    e2e_ms = dist_max(e2e_ms)
    field_bytes = 7 * st_nx() * st_nz() * 8

    def poisson_ms(prof):
        return sum(prof[c][0] for c in ("poisson_rhs", "cg", "mg_sweep", "mg_restrict", "mg_coarse")) / 2

    def solve_rec(r):
        return {"poisson_ms_per_solve": poisson_ms(r["prof"]), "poisson_iterations_last": r["it"],
                "poisson_relres_last": r["rel"]}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "NX": NX, "NZ": NZ, "dx_m": DX, "dz_m": DX, "dt_s": DT,
                   "precision": "FP64 throughout (fields, stencils, Kessler, solve, reductions)",
                   "solver": "direct Fourier-mode solve (row FFTs + per-mode z tridiagonal) in "
                             "FP64, residual-checked; FP64 CG preconditioned by it if the check "
                             "fails",
                   "poisson_tol": 1e-10, "l2": "flushed (256 MB write) between timed steps",
                   "graph_warmup": f"max(warmup, {GRAPH_WARMUP}) untimed steps, so both step graphs (one per step parity) are captured before timing",
                   "parallelism": f"replicas x{world}"},
        "poisson_ms_per_solve": poisson_ms(head["prof"]),
        "poisson_solves_per_s": 1e3 / poisson_ms(head["prof"]),
        "poisson_iterations_last": head["it"], "poisson_relres_last": head["rel"],
        "plain_fp64": {"solver": "multigrid-PCG", "value": fp64_value,
                       "ms_per_step": fp64_ms / args.steps, **solve_rec(results["fp64_mgpcg"]),
                       "roofline": roofline(results["fp64_mgpcg"]["prof"], head["st"].grid, 8, hbm,
                                            peak_kind, results["fp64_mgpcg"]["it"])},
        "speedup_vs_plain_fp64": value / fp64_value,
        "mixed": {"precision": "FP32 fields/stencils, FP64 Kessler arithmetic, FP64 Poisson "
                               "residual/refinement/reductions",
                  "solver": "spectral", "dtype": "f32+f64", "value": mixed_value,
                  "ms_per_step": mixed_ms / args.steps, **solve_rec(results["mixed_spectral"]),
                  "roofline": roofline(results["mixed_spectral"]["prof"], head["st"].grid, 4, hbm,
                                       peak_kind, results["mixed_spectral"]["it"]),
                  "vs_plain_fp64": mixed_value / fp64_value},
        "variants": {name: {"value": world * cells * args.steps / (vms[name] * 1e-3),
                            "ms_per_step": vms[name] / args.steps, **solve_rec(results[name])}
                     for name in ("mixed_mgpcg",)},
        "roofline": roofline(head["prof"], head["st"].grid, 8, hbm, peak_kind, head["it"]),
        "kernel_ms_per_step": {k: v[0] / 2 for k, v in head["prof"].items()},
        "e2e": {"value": world * cells * args.steps / (e2e_ms * 1e-3), "unit": METRIC,
                "h2d_bytes_per_step": field_bytes, "d2h_bytes_per_step": field_bytes},
        "gpu_launches": head["launches"],
        "clocks": clocks,
    }
    g.close()
    if not args.no_accuracy:
        line["mixed"]["accuracy_600_steps"] = mixed_accuracy()
    if not args.no_learned:
        from vvm_b200.learned_training import train_on_small_workloads
        t0 = time.perf_counter()
        w, trec = train_on_small_workloads(device=device)
        trec["seconds"] = time.perf_counter() - t0
        trec["pairs_from"] = ("the plain FP64 multigrid-PCG solver's own pairs: the warm bubble at 128x64 "
                              "and the squall line at 1024x128 on stretched levels (each half model "
                              "steps, half white noise); the weights then serve both grids below")
        line["learned"] = learned_arm(args, world, device, flush, hbm, peak_kind, fp64_ms / args.steps, w, trec)
        line["poisson_stretched"] = stretched_poisson_arm(world, device, w, trec)
    if not args.no_long_runs:
        from vvm_b200.precision_runs import run as long_run
        line["config5_squall_line"] = long_run("config5", variants=("fp64_mgpcg", "mixed_spectral"))
    if not args.no_ensemble:
        line["ensemble"] = ensemble_arm(args, rank, world, device)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    return line


def net_figures(grid):
    """Algorithmic work of one forward pass of the learned preconditioner's
    network on this grid (levels l = 0..3 of H0 = round_up(NZ-1, 8) by NX
    pixels, halved per level): the 32 -> 32 convolutions are U0 at level 0, D1
    and U1 at level 1, D2 and U2 at level 2, D3 at level 3; each reads its
    input and writes its output once (BF16, 64 B a pixel) and does 2*9*32*32
    FLOPs a pixel."""
    H0, W0 = -(-(grid.NZ - 1) // 8) * 8, grid.NX
    per_level = (1, 2, 2, 1)
    px = sum(n * (H0 >> l) * (W0 >> l) for l, n in enumerate(per_level))
    return {"convs": sum(per_level), "pixels": px, "bytes": 128.0 * px, "flops": 2.0 * 9 * 32 * 32 * px}


def learned_arm(args, world, device, flush, hbm, peak_kind, fp64_ms_per_step, w, trec, steps=3):
    """Learned-preconditioned step (mixed-precision fields, FP64 flexible CG
    to the same residual 1e-10) on the headline grid with the weights `w`
    trained on the small workloads (vvm_b200.learned_training), timed over
    `steps` steps with the network and without it (the ablation). The
    convolutions' roofline comes from repeated forward passes timed between
    one pair of events."""
    import torch
    from vvm_b200.gpu import VVM_PREC_MIXED, VVM_SOLVER_LEARNED, VVMGpu
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(NX, NZ, DX, DX, DT)
    out = {"training": trec}
    for mode, name in ((0, "with_net"), (1, "without_net")):
        g = VVMGpu(st.grid, precision=VVM_PREC_MIXED, solver=VVM_SOLVER_LEARNED, device=device)
        g.set_stream(torch.cuda.current_stream().cuda_stream)
        g.upload(st)
        g.learned_weights(w)
        g.learned_config(mode=mode, cap=4000)
        g.step(GRAPH_WARMUP)   # both step graphs captured before the timed steps
        g.synchronize()
        if dist_on():
            dist_barrier()
        times = timed_steps(torch, g, steps, flush)
        it, fell = g.learned_last()
        _, rel = g.last_solve()
        ms = dist_max(sum(times)) / steps
        rec = {"ms_per_step": ms, "value": world * NX * NZ / (ms * 1e-3), "fcg_iterations_last": it,
               "fell_back": bool(fell), "poisson_relres_last": rel}
        if mode == 0:
            fwd_ms, conv_ms = g.learned_time(reps=20)
            nf = net_figures(st.grid)
            rec["net_forward_ms"] = fwd_ms
            rec["ms_per_fcg_iteration"] = ms / max(it, 1)
            rec["conv_roofline"] = {
                "kernel": "k_conv32_stream (3x3, 32 -> 32, BF16, tcgen05 + TMA); k_conv32_tc below 144 px",
                "bound": "hbm", "achieved": nf["bytes"] / (conv_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": nf["bytes"] / (conv_ms * 1e-3) / 1e9 / hbm, "peak_source": peak_kind,
                "tensor_tflops": nf["flops"] / (conv_ms * 1e-3) / 1e12,
                "algorithmic_bytes_per_forward": nf["bytes"], "flops_per_forward": nf["flops"],
                "ms_per_forward_convs": conv_ms, "convs_per_forward": nf["convs"],
                "note": "20 passes between one event pair, activations L2-resident between launches; "
                        "144 FLOP/B is below the BF16 ridge, so the bound is memory"}
        out[name] = rec
        g.close()
    out["solver"] = ("flexible CG, FP64; preconditioner: z-line solve, tensor-core conv net on the "
                     "remaining residual with a Galerkin step, z-line solve; multigrid-PCG fallback")
    out["vs_plain_fp64_mgpcg"] = fp64_ms_per_step / out["with_net"]["ms_per_step"]
    out["iterations_saved_by_net"] = (out["without_net"]["fcg_iterations_last"]
                                      / max(out["with_net"]["fcg_iterations_last"], 1))
    return out


def stretched_poisson_arm(world, device, w, trec, reps=5):
    """The stretched-level Poisson workload: the cal_w solve on NX=2048, NZ=256 stretched
    levels (dz 100 m -> 500 m, tanh ramp; dx = 250 m), right-hand sides of
    seeded bubble/cold-pool vorticity dipoles. Learned-PCG (the weights `w`
    trained on the small workloads) against FP64 multigrid-PCG and the
    spectral solve, each to ||b - A W|| / ||b|| <= 1e-10 from W = 0, device
    buffers, event-timed on the library's stream; `ms_per_solve` is the mean of
    `reps` solves after two warm-up solves."""
    import torch
    from vvm_b200.gpu import VVM_SOLVER_LEARNED, VVM_SOLVER_MGPCG, VVM_SOLVER_SPECTRAL, VVMGpu
    from vvm_b200.initial_state import poisson_rhs, stretched_poisson_case
    nx, nz = 2048, 256
    st = stretched_poisson_case(nx, nz, seed=7)
    b = poisson_rhs(st)
    dev = torch.device(f"cuda:{device}")
    d_b = torch.from_numpy(b).to(dev)
    d_W = torch.zeros_like(d_b)
    out = {"workload": "cal_w on NX=2048 NZ=256 stretched levels dz 100->500 m (tanh), dx=250 m; "
                       "rhs from 6 seeded vorticity dipoles", "tol": 1e-10, "training": trec}
    stream = torch.cuda.current_stream()
    for name, solver, mode in (("mgpcg_fp64", VVM_SOLVER_MGPCG, None), ("spectral_fp64", VVM_SOLVER_SPECTRAL, None),
                               ("learned_pcg", VVM_SOLVER_LEARNED, 0), ("learned_cycle_without_net", VVM_SOLVER_LEARNED, 1)):
        g = VVMGpu(st.grid, solver=solver, device=device)
        g.set_stream(stream.cuda_stream)
        g.upload(st)
        rec = {}
        if mode is not None:
            g.learned_weights(w)
            g.learned_config(mode=mode, cap=4000)
        for _ in range(2):
            d_W.zero_()
            g.poisson_solve_device(d_b.data_ptr(), d_W.data_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):   # every solve from W = 0 (a warm start would reuse the last answer)
            d_W.zero_()
            it, rel = g.poisson_solve_device(d_b.data_ptr(), d_W.data_ptr())
        e1.record(stream)
        e1.synchronize()
        ms = dist_max(e0.elapsed_time(e1)) / reps
        rec.update({"ms_per_solve": ms, "solves_per_s": world * 1e3 / ms, "iterations": it, "relres": rel})
        if mode is not None:
            rec["fcg_iterations"], rec["fell_back"] = g.learned_last()
        out[name] = rec
        g.close()
    out["learned_vs_mgpcg_time"] = out["mgpcg_fp64"]["ms_per_solve"] / out["learned_pcg"]["ms_per_solve"]
    out["net_iteration_ratio"] = (out["learned_cycle_without_net"]["fcg_iterations"]
                                  / max(out["learned_pcg"]["fcg_iterations"], 1))
    return out


def st_nx():
    return NX + 2


def st_nz():
    return NZ + 2


# ------------------------------------------------------------------ ensemble

ENSEMBLE_CASES, ENSEMBLE_SEED = 256, 3


def ensemble_arm(args, rank, world, device):
    """The batched-ensemble workload: 256 seeded warm-bubble cases of uneven grids
    (vvm_b200.ensemble), mixed precision with the spectral solve, one batch
    graph a step on each rank; the cases are split over the ranks by cost.
    The ensemble is fixed, so more ranks is strong scaling."""
    import torch
    from vvm_b200.ensemble import ensemble_specs, ensemble_state, shard_by_cost
    from vvm_b200.gpu import VVM_PREC_MIXED, VVM_SOLVER_SPECTRAL, VVMBatch
    specs = ensemble_specs(ENSEMBLE_CASES, ENSEMBLE_SEED)
    costs = [sp["NX"] * sp["NZ"] for sp in specs]
    mine = shard_by_cost(costs, world)[rank]
    sts = [ensemble_state(specs[i]) for i in mine]
    b = VVMBatch([st.grid for st in sts], precision=VVM_PREC_MIXED, solver=VVM_SOLVER_SPECTRAL,
                 device=device)
    b.upload(sts)
    b.step(3)
    b.synchronize()
    groups = b.autotune(reps=2)
    b.step(args.warmup)
    b.synchronize()
    stream = torch.cuda.ExternalStream(b.stream, device=torch.device(f"cuda:{device}"))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist_on():
        dist_barrier()
    e0.record(stream)
    b.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    b.synchronize()
    max_ms = dist_max(e0.elapsed_time(e1))
    grouped = b.grouping()
    # the same steps with every case its own branch of the graph (no grouped launches)
    b.grouping(False)
    b.step(2)
    b.synchronize()
    if dist_on():
        dist_barrier()
    e0.record(stream)
    b.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    b.synchronize()
    ungrouped_ms = dist_max(e0.elapsed_time(e1))
    total = sum(costs)
    b.close()
    return {"workload": f"{ENSEMBLE_CASES} warm-bubble cases (seed {ENSEMBLE_SEED}): NX in "
                        "{256,512,1024,2048}, NZ in {64,96,128}, amplitude U(1,3) K, centre "
                        "U(0.2,0.8), radius U(1,3) km, dx=dz=200 m, dt=1 s",
            "metric": METRIC, "value": total * args.steps / (max_ms * 1e-3), "unit": METRIC,
            "ms_per_step": max_ms / args.steps, "cells_per_step": total, "cases": ENSEMBLE_CASES,
            "cases_this_rank": len(mine), "scaling": "strong",
            "sharding": "by cells, longest first to the least-loaded rank; no exchange",
            "precision": "mixed", "solver": "spectral",
            "graph": "one CUDA graph a step; the cases of each grid shape as grouped launches "
                     "(one launch a kernel for the group, blockIdx.z the case)",
            "grouped_groups": grouped, "autotune_groups": groups,
            "ungrouped_ms_per_step": ungrouped_ms / args.steps,
            "l2": "working set larger than L2"}


# ----------------------------------------------------------- reference arm

def reference_arm(args):
    from oracle.models import RefModel, ref_available
    from vvm_b200.initial_state import warm_bubble
    if not ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libvvmref.so is not built "
                "(the reference sources were not present when build() ran)"}
    st = warm_bubble(NX, NZ, DX, DX, DT)
    m = RefModel(st.grid)
    m.load(st)
    for _ in range(min(args.warmup, 1)):
        m.one_step()
    nsteps = max(1, min(args.steps, 4))
    t0 = time.perf_counter()
    for _ in range(nsteps):
        m.one_step()
    dt = time.perf_counter() - t0
    v = NX * NZ * nsteps / dt
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": 0,
            "steps": nsteps, "warmup": min(args.warmup, 1), "ms_per_step": 1e3 * dt / nsteps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "NX": NX, "NZ": NZ, "dx_m": DX, "dz_m": DX, "dt_s": DT,
                       "solver": "Eigen BiCGSTAB + IncompleteLUT (tol 1e-22), serial build"},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": 1, "kind": "reference",
                             "sample": f"{nsteps} full-grid reference step(s) (warm-up "
                                       f"{min(args.warmup, 1)}); the reference's OpenMP loops "
                                       f"race, so the serial build; its Eigen solve (99 % of "
                                       f"the step) is single-threaded either way"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ------------------------------------------------------------ distributed

_DIST = {"on": False}


def dist_on():
    return _DIST["on"]


def dist_barrier():
    import torch.distributed as D
    D.barrier()


def dist_max(x: float) -> float:
    """Max of x over the ranks (the device time of the slowest replica); a
    CUDA tensor under NCCL, a host tensor under gloo."""
    if not _DIST["on"]:
        return x
    import torch
    import torch.distributed as D
    dev = "cuda" if D.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    D.all_reduce(t, op=D.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(local_ms: float, world: int, cells: int, steps: int) -> tuple[float, float]:
    """Whole-job cell-steps/s of `world` replicas, each doing `steps` steps of
    `cells` cells: all ranks' work over the slowest rank's time. Returns
    (rate, max_ms)."""
    max_ms = dist_max(local_ms)
    return world * cells * steps / (max_ms * 1e-3), max_ms


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 256-case batched ensemble")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner step")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the 600-step mixed-vs-FP64 domain means on the headline grid")
    ap.add_argument("--no-long-runs", action="store_true",
                    help="skip the 1800-step 8192x256 squall line (mixed vs FP64 domain means)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(args)), flush=True)
        return
    if args.warmup < 3:
        args.warmup = 3
    if world > 1:
        import datetime
        import torch
        import torch.distributed as D
        torch.cuda.set_device(local)
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                             device_id=torch.device(f"cuda:{local}"))
        _DIST["on"] = True
    line = our_arm(args, rank, world, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as D
        D.barrier()
        D.destroy_process_group()


if __name__ == "__main__":
    main()
