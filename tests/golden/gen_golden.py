"""Generates the golden fixtures of tests/golden/ by running the reference VVM
step itself (oracle/_ref/libvvmref.so, built from the reference's sources by
oracle/build_ref.sh). Run from the repository root:

    python tests/golden/gen_golden.py

Fixtures (all float64, numpy .npz, reference [nx][nz] layout):
  config1_init.npz     warm-bubble initial state (NX=128, NZ=64, dx=dz=200 m,
                       dt=1 s): pins the synthetic initialiser
  config1_step1.npz    prognostic fields after 1 reference step
  config1_step10.npz   ... after 10 steps
  config1_600.npz      per-step domain means over 600 steps (th, qc, qr,
                       surface rain, kinetic energy) and th/qc/qr/w at step 600
  routines_kat.npz     one call of each reference routine on a seeded random
                       34x18 state (inputs and outputs)
  poisson_kat.npz      manufactured solution x = exp(sin(i + k)) of the cal_w
                       matrix (the reference's own POISSONTEST idea,
                       src/PoissonSolver.cpp:815-828): b = A x, the reference's
                       BiCGSTAB solution and its true residual
  halo_kat.npz         BoundaryProcess2D_all (src/Boundary.cpp:36-58) on the
                       34x18 routine state with every ghost cell of the fields
                       it touches overwritten by seeded noise first
  stream_kat.npz       the streamfunction formulation (oracle/_ref/
                       libvvmref_stream.so, STREAMFUNCTION with
                       POISSONPARAM = 0): calpsiuw (src/PoissonSolver.cpp:
                       124-177) on the 34x18 routine state, and 1 and 10 steps
                       of a 64x32 warm bubble (dx = dz = 200 m, dt = 1 s)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO / "2d-vector-vorticity-model_b200"))
sys.path.insert(0, str(REPO))

from oracle.models import RefModel, RefStreamModel  # noqa: E402
from vvm_b200.initial_state import random_state, warm_bubble  # noqa: E402

OUT = Path(__file__).resolve().parent
PROG = ("zeta", "th", "qv", "qc", "qr", "u", "w")


def domain_means(st) -> np.ndarray:
    """[th, qc, qr, surface rain, kinetic energy] over interior cells."""
    f = st.fields
    inner = (slice(1, -1), slice(1, -1))
    rhou = st.prof["rhou"][None, 1:-1]
    ke = 0.5 * rhou * (f["u"][inner] ** 2 + f["w"][inner] ** 2)
    return np.array([f["th"][inner].mean(), f["qc"][inner].mean(), f["qr"][inner].mean(),
                     st.precip[1:-1].mean(), ke.mean()])


def save_state(path, st, names):
    np.savez_compressed(path, **{n: st.fields[n] for n in names},
                        precip=st.precip, ubarTop=st.scalars["ubarTop"], step=st.scalars["step"])


def gen_config1():
    st = warm_bubble()
    np.savez_compressed(OUT / "config1_init.npz", **{f"f_{k}": v for k, v in st.fields.items()},
                        **{f"p_{k}": v for k, v in st.prof.items()}, ubarTop=st.scalars["ubarTop"])
    m = RefModel(st.grid)
    m.load(st)
    means = [domain_means(m.dump())]
    for s in range(1, 601):
        m.one_step()
        d = m.dump()
        means.append(domain_means(d))
        if s in (1, 10):
            save_state(OUT / f"config1_step{s}.npz", d, PROG)
    np.savez_compressed(OUT / "config1_600.npz", means=np.array(means),
                        **{n: d.fields[n] for n in ("th", "qc", "qr", "w")})


ROUTINES = ["pzeta_pt", "pth_pt", "pqv_pt", "pqc_pt", "pqr_pt", "BoundaryProcess2D_all",
            "pubarTop_pt", "cal_w", "cal_u", "autoconversion", "accretion", "evaporation",
            "condensation", "NVP_qvp", "NVP_qcp", "NVP_qrp", "updateMean", "RKM_RKH",
            "Nudge_theta", "Nudge_zeta", "nextTimeStep"]


def kat_input():
    st = random_state(34, 18, seed=7)
    for n in ("zetap", "thp", "qvp", "qcp", "qrp"):
        st.fields[n] = st.fields[n[:-1]] * 1.01
    st.fields["zetap"][:, :2] = 0.0
    st.fields["qcp"][5:9, 3:6] = -2e-5     # negative water for NegativeValueProcess
    return st


def gen_routines():
    st = kat_input()
    out = {f"in_{k}": v for k, v in st.fields.items()}
    out.update({f"inh_{k}": v for k, v in st.hist.items()})
    out.update({f"inp_{k}": v for k, v in st.prof.items()})
    out["in_ubarTop"] = st.scalars["ubarTop"]
    out["in_dubar"] = st.scalars["dubarTop_advect"]
    out["in_step"] = st.scalars["step"]
    base = RefModel(st.grid)
    base.load(st)
    b0 = base.dump()
    for r in ROUTINES:
        m = RefModel(st.grid)
        m.load(st)
        m.call(r)
        d = m.dump()
        # only what the routine changed (everything else equals the input)
        for k, v in d.fields.items():
            if not np.array_equal(v, b0.fields[k], equal_nan=True):
                out[f"{r}__{k}"] = v
        for k, v in d.hist.items():
            if not np.array_equal(v, b0.hist[k], equal_nan=True):
                out[f"{r}__h_{k}"] = v
        for k in ("thb", "qvb", "thvb"):
            if not np.array_equal(d.prof[k], b0.prof[k]):
                out[f"{r}__p_{k}"] = d.prof[k]
        if not np.array_equal(d.precip, b0.precip):
            out[f"{r}__precip"] = d.precip
        out[f"{r}__ubarTopp"] = d.scalars["ubarTopp"]
        out[f"{r}__dubar"] = d.scalars["dubarTop_advect"]
    np.savez_compressed(OUT / "routines_kat.npz", **out)


def gen_poisson():
    st = warm_bubble(64, 32)
    m = RefModel(st.grid)
    m.load(st)
    NX, NK = st.grid.NX, st.grid.NZ - 1
    kk, ii = np.meshgrid(np.arange(NK), np.arange(NX), indexing="ij")
    x_ans = np.exp(np.sin(ii + kk)).ravel()            # src/PoissonSolver.cpp:822-826
    b = m.apply_A(x_ans)
    x, it, err, rc = m.solve_A(b)
    res = np.linalg.norm(b - m.apply_A(x)) / np.linalg.norm(b)
    np.savez_compressed(OUT / "poisson_kat.npz", NX=NX, NZ=st.grid.NZ, x_ans=x_ans, b=b,
                        x_ref=x, iters=it, true_relres=res,
                        rhou=st.prof["rhou"], rhow=st.prof["rhow"])


HALO_FIELDS = ("zetap", "thp", "w", "u", "qvp", "qcp", "qrp")


def ghost_mask(nx, nz):
    m = np.zeros((nx, nz), dtype=bool)
    m[0, :] = m[-1, :] = True
    m[:, 0] = m[:, -1] = True
    return m


def gen_halo():
    st = kat_input()
    rng = np.random.default_rng(11)
    g = ghost_mask(st.grid.nx, st.grid.nz)
    for n in HALO_FIELDS:
        a = st.fields[n]
        a[g] = rng.standard_normal(int(g.sum())) * (np.abs(a).max() + 1.0)
    m = RefModel(st.grid)
    m.load(st)
    m.call("BoundaryProcess2D_all")
    d = m.dump()
    np.savez_compressed(OUT / "halo_kat.npz", **{f"in_{n}": st.fields[n] for n in HALO_FIELDS},
                        **{f"out_{n}": d.fields[n] for n in HALO_FIELDS})


def gen_stream():
    st = kat_input()
    m = RefStreamModel(st.grid)
    m.load(st)
    m.call("calpsiuw")
    out = {"calpsiuw__psi": m.psi().copy(), "calpsiuw__u": m.field("u").copy(),
           "calpsiuw__w": m.field("w").copy()}
    m.close()
    st = warm_bubble(64, 32)
    m = RefStreamModel(st.grid)
    m.load(st)
    for s in range(1, 11):
        m.one_step()
        if s in (1, 10):
            d = m.dump()
            for n in PROG:
                out[f"step{s}__{n}"] = d.fields[n]
            out[f"step{s}__psi"] = m.psi().copy()
    np.savez_compressed(OUT / "stream_kat.npz", **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["poisson", "routines", "config1", "halo", "stream"]
    if "halo" in which:
        gen_halo()
    if "stream" in which:
        gen_stream()
    if "poisson" in which:
        gen_poisson()
    if "routines" in which:
        gen_routines()
    if "config1" in which:
        gen_config1()
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size)
