"""Synthetic, seeded initial states for the VVM step.

Every array uses the reference model's host layout: 2D fields are
``[nx][nz]`` float64 with k (height) the fast index, ghost cells included
(``nx = NX + 2``, ``nz = NZ + 2``; src/Declare.hpp:33,82-83).

The 1D base state is built with the reference's own discrete formulas
(src/Init.cpp:14-135): hydrostatic Exner function from the surface pressure,
anelastic densities at cell centres (``rhou``) and faces (``rhow``), the
``(k-1/2) dz`` level heights and the mixing-length profile ``lambda2``.
Only the input profiles differ from the reference's analytic sounding: the
warm-bubble case uses theta = 300 K + 3 K/km and qv at a fixed relative
humidity of the model's Tetens saturation mixing ratio (src/Init.cpp:88),
solved together with the pressure by fixed-point iteration.

The 2D state follows src/Init.cpp:186-255: theta = base + bubble, qv = base
profile everywhere, qc = qr = 0, zeta diagnosed from (u, w), ubarTop = the
mean of u on the top interior row.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

GRAVITY = 9.80665
CP = 1003.5
CV = 716.5
RD = 287.0
LV = 2.5e6
P0 = 1e5
PSURF = 96500.0


@dataclass
class GridSpec:
    """Interior sizes and spacings of one case (reference vvm_config.txt keys)."""
    NX: int
    NZ: int
    dx: float
    dz: float
    dt: float
    case: int = 1
    moisture_nudge_time: float = 0.0

    @property
    def nx(self) -> int:
        return self.NX + 2

    @property
    def nz(self) -> int:
        return self.NZ + 2


@dataclass
class VVMState:
    """Complete model state in the reference's host layout."""
    grid: GridSpec
    fields: dict = field(default_factory=dict)    # name -> (nx, nz)
    hist: dict = field(default_factory=dict)      # name -> (nx, nz, 2)
    prof: dict = field(default_factory=dict)      # name -> (nz,)
    scalars: dict = field(default_factory=dict)   # ubarTop, ubarTopp, dubarTop_advect, step
    precip: np.ndarray | None = None

    def copy(self) -> "VVMState":
        return VVMState(self.grid,
                        {k: v.copy() for k, v in self.fields.items()},
                        {k: v.copy() for k, v in self.hist.items()},
                        {k: v.copy() for k, v in self.prof.items()},
                        {k: (v.copy() if isinstance(v, np.ndarray) else v)
                         for k, v in self.scalars.items()},
                        None if self.precip is None else self.precip.copy())


FIELDS_2D = ("zeta", "zetap", "th", "thp", "qv", "qvp", "qc", "qcp", "qr", "qrp",
             "u", "w", "RKM", "RKH")
HIST = ("dzeta_advect", "dth_buoyancy", "dth_advect", "dqv_advect", "dqc_advect",
        "dqr_advect", "dqr_VT")
PROFILES = ("rhou", "rhow", "thb", "thvb", "qvb", "pib", "pb", "thb_init", "qvb0",
            "z", "z_zeta", "lambda2")


def _center1d(a: np.ndarray) -> None:
    # src/Boundary.cpp:3-7
    a[0] = a[1]
    a[-1] = a[-2]


def _center2d(a: np.ndarray) -> None:
    # src/Boundary.cpp:9-19: periodic x on interior rows, then zero gradient in z
    a[0, 1:-1] = a[-2, 1:-1]
    a[-1, 1:-1] = a[1, 1:-1]
    a[:, 0] = a[:, 1]
    a[:, -1] = a[:, -2]


def _westdown2d(a: np.ndarray) -> None:
    # src/Boundary.cpp:21-30: periodic x, zero on rows 0, 1 and nz-1
    a[0, 1:-1] = a[-2, 1:-1]
    a[-1, 1:-1] = a[1, 1:-1]
    a[:, 0] = 0.0
    a[:, 1] = 0.0
    a[:, -1] = 0.0


def tetens_qvs(T: np.ndarray, p: np.ndarray) -> np.ndarray:
    """Saturation mixing ratio of the model (src/Init.cpp:88, MicroPhysics.cpp:12)."""
    return (380.0 / p) * np.exp(17.27 * (T - 273.0) / (T - 36.0))


def base_state(g: GridSpec, theta_of_z, rh: float | np.ndarray, qv_of_z=None,
               zf: np.ndarray | None = None) -> dict:
    """1D base state on the reference's staggering (src/Init.cpp:14-135).

    ``theta_of_z(z)`` gives the base potential temperature at cell-centre
    heights ``z = (k - 1/2) dz``. Moisture is either ``rh`` times the Tetens
    saturation value (solved jointly with the hydrostatic pressure) or, when
    ``qv_of_z`` is given, that profile directly.
    """
    nz, dz = g.nz, g.dz
    k = np.arange(nz)
    zc = (k - 0.5) * dz
    if zf is not None:   # stretched levels: faces zf[1..nz-1] (zf[1] = 0), centres midway
        zf = np.asarray(zf, dtype=np.float64)
        zc = np.zeros(nz)
        zc[1:nz - 1] = 0.5 * (zf[1:nz - 1] + zf[2:nz])
        zc[0], zc[nz - 1] = zc[1], zc[nz - 2]
    thb = np.zeros(nz)
    thb[1:nz - 1] = theta_of_z(zc[1:nz - 1])
    _center1d(thb)
    rh_arr = np.broadcast_to(np.asarray(rh, dtype=np.float64), (nz,)) if qv_of_z is None else None

    qvb = np.zeros(nz)
    if qv_of_z is not None:
        qvb[1:nz - 1] = qv_of_z(zc[1:nz - 1])
        _center1d(qvb)

    pisfc = (PSURF / P0) ** (RD / CP)

    def hydrostatic(q):
        thvb = thb * (1.0 + 0.61 * q)                         # src/Init.cpp:38
        _center1d(thvb)
        pib = np.zeros(nz)
        for kk in range(1, nz - 1):                           # src/Init.cpp:46-52
            if kk == 1:
                h1 = 0.5 * dz if zf is None else zc[1] - zf[1]
                pib[kk] = pisfc - GRAVITY * h1 / (CP * thvb[kk])
            else:
                tvbavg = 0.5 * (thvb[kk] + thvb[kk - 1])
                hk = dz if zf is None else zc[kk] - zc[kk - 1]
                pib[kk] = pib[kk - 1] - GRAVITY * hk / (CP * tvbavg)
        _center1d(pib)
        if np.any(pib[1:nz - 1] <= 0.0):
            raise ValueError("base state: the Exner function reaches zero below the model "
                             "top; lower NZ*dz or the lapse rate")
        return thvb, pib

    if qv_of_z is None:
        for _ in range(100):
            thvb, pib = hydrostatic(qvb)
            pb = P0 * pib ** (CP / RD)                        # src/Init.cpp:86
            qnew = np.zeros(nz)
            qnew[1:nz - 1] = rh_arr[1:nz - 1] * tetens_qvs(thb[1:nz - 1] * pib[1:nz - 1],
                                                            pb[1:nz - 1])
            _center1d(qnew)
            done = np.array_equal(qnew, qvb)
            qvb = qnew
            if done:
                break
    thvb, pib = hydrostatic(qvb)

    rhou = np.zeros(nz)
    rhou[1:nz - 1] = P0 * pib[1:nz - 1] ** (CV / RD) / (RD * thvb[1:nz - 1])   # src/Init.cpp:68
    _center1d(rhou)
    rhow = np.zeros(nz)
    for kk in range(2, nz):                                   # src/Init.cpp:74-82
        rhow[kk] = 0.5 * (rhou[kk] + rhou[kk - 1])
    rhow[1] = rhow[2] - (rhow[3] - rhow[2])
    rhow[0] = rhow[1]
    rhou[0] = rhow[0]

    pb = np.zeros(nz)
    pb[1:nz - 1] = P0 * pib[1:nz - 1] ** (CP / RD)
    _center1d(pb)

    thb_init = thb.copy()
    qvb0 = qvb.copy()
    thvb_step1 = thb + 0.61 * qvb                             # src/Init.cpp:119 (additive)

    z = np.zeros(nz)
    z_zeta = np.zeros(nz)
    lambda2 = np.zeros(nz)
    for kk in range(1, nz - 1):                               # src/Init.cpp:125-129
        if zf is None:
            z[kk] = (kk - 0.5) * dz
            z_zeta[kk] = (kk - 1) * dz
            dzk = dz
        else:
            z[kk] = zc[kk]
            z_zeta[kk] = zf[kk]
            dzk = zf[kk + 1] - zf[kk]
        lambda2[kk] = 1.0 / (1.0 / math.pow(0.23 * math.sqrt(g.dx * dzk), 2)
                             + 1.0 / math.pow(0.4 * 0.4 * z[kk], 2))
    z[0], z[-1] = z[1], z[-2]
    z_zeta[0], z_zeta[-1] = z_zeta[1], z_zeta[-2]
    return dict(thb=thb, thvb=thvb_step1, qvb=qvb, pib=pib, pb=pb, rhou=rhou, rhow=rhow,
                thb_init=thb_init, qvb0=qvb0, z=z, z_zeta=z_zeta, lambda2=lambda2)


def _assemble(g: GridSpec, prof: dict, th: np.ndarray, u: np.ndarray,
              w: np.ndarray | None = None, qv: np.ndarray | None = None,
              stretched: bool = False) -> VVMState:
    nx, nz = g.nx, g.nz
    st = VVMState(g)
    f = st.fields
    for name in FIELDS_2D:
        f[name] = np.zeros((nx, nz))
    f["th"][:] = th
    _center2d(f["th"])
    f["qv"][:] = prof["qvb"][None, :] if qv is None else qv
    if qv is not None:
        _center2d(f["qv"])
    f["u"][:] = u
    _center2d(f["u"])
    if w is not None:
        f["w"][:] = w
        _westdown2d(f["w"])
    # zeta from (u, w): src/Init.cpp:231-241
    uu, ww, rhow = f["u"], f["w"], prof["rhow"]
    zeta = f["zeta"]
    pw_px = (ww[1:nx - 1, 1:nz - 1] - ww[0:nx - 2, 1:nz - 1]) * (1.0 / g.dx)
    if stretched:   # centre-to-centre spacing around each face (the first is never used: u[0] = u[1])
        zc = prof["z"]
        dzw = np.empty(nz - 2)
        dzw[0] = 1.0
        dzw[1:] = zc[2:nz - 1] - zc[1:nz - 2]
        pu_pz = (uu[1:nx - 1, 1:nz - 1] - uu[1:nx - 1, 0:nz - 2]) / dzw[None, :]
    else:
        pu_pz = (uu[1:nx - 1, 1:nz - 1] - uu[1:nx - 1, 0:nz - 2]) * (1.0 / g.dz)
    zeta[1:nx - 1, 1:nz - 1] = (pw_px - pu_pz) / rhow[None, 1:nz - 1]
    _westdown2d(zeta)
    # ubarTop: src/Init.cpp:244-248 (sequential sum, as the reference does)
    s = 0.0
    for i in range(1, nx - 1):
        s += uu[i, nz - 2]
    ubar = s / float(nx - 2)
    for name in HIST:
        st.hist[name] = np.zeros((nx, nz, 2))
    st.prof = {k: np.array(v, dtype=np.float64) for k, v in prof.items()}
    st.scalars = dict(ubarTop=ubar, ubarTopp=0.0, dubarTop_advect=np.zeros(2), step=0)
    st.precip = np.zeros(nx)
    return st


def warm_bubble(NX: int = 128, NZ: int = 64, dx: float = 200.0, dz: float = 200.0,
                dt: float = 1.0, amp: float = 2.0, radius: float = 2000.0,
                xc_frac: float = 0.5, zc: float = 2000.0, dthdz: float = 3e-3,
                rh: float = 0.8, case: int = 1, zf: np.ndarray | None = None) -> VVMState:
    """Plain VVM warm bubble: theta = 300 K + dthdz*z, qv at ``rh`` of saturation,
    a cosine bubble of amplitude ``amp`` and radius ``radius`` centred at
    (``xc_frac`` of the domain, ``zc``), u = w = 0. ``zf``: face heights of
    stretched levels (stretched_faces; ``dz`` is then its lowest spacing)."""
    g = GridSpec(NX, NZ, dx, dz, dt, case)
    prof = base_state(g, lambda z: 300.0 + dthdz * z, rh, zf=zf)
    nx, nz = g.nx, g.nz
    i = np.arange(nx)[:, None]
    k = np.arange(nz)[None, :]
    x = (i - 0.5) * dx
    z = (k - 0.5) * dz if zf is None else prof["z"][None, :]
    r = np.sqrt(((x - xc_frac * NX * dx) / radius) ** 2 + ((z - zc) / radius) ** 2)
    bubble = np.where(r <= 1.0, 0.5 * amp * (np.cos(np.pi * r) + 1.0), 0.0)
    th = np.zeros((nx, nz))
    th[1:nx - 1, 1:nz - 1] = prof["thb"][None, 1:nz - 1] + bubble[1:nx - 1, 1:nz - 1]
    return _assemble(g, prof, th, np.zeros((nx, nz)), stretched=zf is not None)


def random_state(NX: int = 32, NZ: int = 16, dx: float = 200.0, dz: float = 200.0,
                 dt: float = 1.0, seed: int = 0, step_parity_hist: bool = True) -> VVMState:
    """A warm-bubble base state with seeded random perturbations in every
    prognostic field, nonzero u/w/RKM and AB2 history: exercises every branch
    of the per-routine kernels (signs of u and w, negative water, Ri ranges)."""
    rng = np.random.default_rng(seed)
    st = warm_bubble(NX, NZ, dx, dz, dt, amp=2.0, radius=0.25 * NX * dx)
    g = st.grid
    nx, nz = g.nx, g.nz
    f = st.fields
    f["th"][1:-1, 1:-1] += rng.normal(0.0, 0.5, (nx - 2, nz - 2))
    f["qv"][1:-1, 1:-1] *= 1.0 + rng.normal(0.0, 0.1, (nx - 2, nz - 2))
    f["qc"][1:-1, 1:-1] = np.maximum(rng.normal(5e-4, 8e-4, (nx - 2, nz - 2)), -1e-5)
    # qr stays >= 0: the fall speed takes qr**0.1346 (src/Advection.cpp:165)
    f["qr"][1:-1, 1:-1] = np.maximum(rng.normal(3e-4, 5e-4, (nx - 2, nz - 2)), 0.0)
    f["u"][1:-1, 1:-1] = rng.normal(0.0, 3.0, (nx - 2, nz - 2))
    f["w"][1:-1, 2:-1] = rng.normal(0.0, 2.0, (nx - 2, nz - 3))
    f["zeta"][1:-1, 2:-1] = rng.normal(0.0, 0.02, (nx - 2, nz - 3))
    f["RKM"][1:-1, 1:-1] = rng.uniform(10.0, 400.0, (nx - 2, nz - 2))
    f["RKH"][1:-1, 1:-1] = rng.uniform(10.0, 400.0, (nx - 2, nz - 2))
    for name in ("th", "qv", "qc", "qr", "u", "RKM", "RKH"):
        _center2d(f[name])
    _westdown2d(f["w"])
    _westdown2d(f["zeta"])
    for name in HIST:
        st.hist[name][1:-1, 1:-1, :] = rng.normal(0.0, 1e-4, (nx - 2, nz - 2, 2))
    st.scalars["ubarTop"] = float(rng.normal(0.0, 1.0))
    st.scalars["dubarTop_advect"] = rng.normal(0.0, 1e-3, 2)
    st.scalars["step"] = 3
    return st


def stretched_faces(NZ: int, dz_bottom: float, dz_top: float) -> np.ndarray:
    """Face heights of NZ levels whose thickness grows from dz_bottom to dz_top
    along a tanh ramp centred at mid-depth: dz_j = dz_bottom + (dz_top -
    dz_bottom) (1 + tanh((j - NZ/2) / (NZ/6))) / 2, j = 0..NZ-1, rescaled so the
    first and last thicknesses are exactly dz_bottom and dz_top. Returned on
    the model's nz = NZ + 2 index: zf[k] for k = 1..NZ+1 (zf[1] = 0; zf[0] =
    zf[1]); the level heights of a stretched case."""
    j = np.arange(NZ, dtype=np.float64)
    t = (1.0 + np.tanh((j - NZ / 2.0) / (NZ / 6.0))) / 2.0
    t = (t - t[0]) / (t[-1] - t[0])
    dzs = dz_bottom + (dz_top - dz_bottom) * t
    zf = np.zeros(NZ + 2)
    zf[2:] = np.cumsum(dzs)
    zf[0] = zf[1]
    return zf


def stratified_theta(z):
    """theta [K]: 300 K + 3 K/km up to 12 km, then growing by e every 22 km,
    close to an isothermal stratosphere at the tropopause temperature (~210 K:
    e-folding c_p T / g), so that the Exner function stays positive to the top
    of deep stretched grids."""
    z = np.asarray(z, dtype=np.float64)
    tp = 300.0 + 3e-3 * 12000.0
    return np.where(z <= 12000.0, 300.0 + 3e-3 * z, tp * np.exp((z - 12000.0) / 22000.0))


def dry_aloft(z, rh_low):
    """Relative humidity rh_low up to 10 km, decaying with a 1.5 km scale
    above (a nearly dry stratosphere: with moist air aloft the coupled
    moisture-hydrostatic solve of base_state runs away to unphysical qv)."""
    z = np.asarray(z, dtype=np.float64)
    return np.where(z <= 10000.0, rh_low, rh_low * np.exp(-(z - 10000.0) / 1500.0))


def stretched_poisson_case(NX: int = 2048, NZ: int = 256, dx: float = 250.0,
                           dz_bottom: float = 100.0, dz_top: float = 500.0,
                           seed: int = 4, blobs: int = 6) -> VVMState:
    """A Poisson-only state on stretched levels (tanh ramp dz_bottom ->
    dz_top): the base state of a stratified atmosphere (stratified_theta,
    80 % relative humidity) and a vorticity field of `blobs` seeded
    bubble/cold-pool dipoles (Gaussian vortex pairs 2-6 km wide, 1-3 km deep,
    centred in the lowest 8 km), the shape of the right-hand sides that warm
    bubbles and squall lines give cal_w. Only rhou, rhow, z, z_zeta and zeta
    matter to the solve. Relative humidity: dry_aloft(z, 0.8)."""
    zf = stretched_faces(NZ, dz_bottom, dz_top)
    g = GridSpec(NX, NZ, dx, dz_bottom, 1.0)
    zc = np.zeros(NZ + 2)
    zc[1:NZ + 1] = 0.5 * (zf[1:NZ + 1] + zf[2:NZ + 2])
    prof = base_state(g, stratified_theta, dry_aloft(zc, 0.8), zf=zf)
    nx, nz = g.nx, g.nz
    rng = np.random.default_rng(seed)
    x = (np.arange(nx)[:, None] - 0.5) * dx
    z = prof["z"][None, :]
    L = NX * dx
    zeta = np.zeros((nx, nz))
    for _ in range(blobs):
        xc, zc = rng.uniform(0.0, L), rng.uniform(1000.0, 8000.0)
        wx, wz = rng.uniform(2000.0, 6000.0), rng.uniform(1000.0, 3000.0)
        amp = rng.uniform(0.5, 2.0) * 1e-2 * rng.choice((-1.0, 1.0))
        dxp = (x - xc + 0.5 * L) % L - 0.5 * L           # periodic distance
        for sgn, off in ((1.0, -0.5 * wx), (-1.0, 0.5 * wx)):
            zeta += sgn * amp * np.exp(-((dxp - off) / (0.5 * wx)) ** 2 - ((z - zc) / wz) ** 2)
    th = np.zeros((nx, nz))
    th[1:nx - 1, 1:nz - 1] = prof["thb"][None, 1:nz - 1]
    st = _assemble(g, prof, th, np.zeros((nx, nz)))
    st.fields["zeta"][1:nx - 1, 1:nz - 1] = zeta[1:nx - 1, 1:nz - 1]
    st.fields["zetap"][:] = st.fields["zeta"]
    _westdown2d(st.fields["zeta"])
    _westdown2d(st.fields["zetap"])
    return st


def poisson_rhs(st: VVMState, field: str = "zeta") -> np.ndarray:
    """The right-hand side cal_w forms from a vorticity field
    (src/PoissonSolver.cpp:444-450): b = rhow_k^2 (zeta[i+1][k] - zeta[i][k]) dx
    for k = 2..nz-2, i = 1..nx-2, in the reference's vector ordering."""
    z, rhow, dx = st.fields[field], st.prof["rhow"], st.grid.dx
    nx, nz = z.shape
    return np.concatenate([rhow[k] * rhow[k] * (z[2:nx, k] - z[1:nx - 1, k]) * dx for k in range(2, nz - 1)])


def squall_line(NX: int = 1024, NZ: int = 128, dx: float = 250.0, dz: float = 250.0, dt: float = 2.0,
                seed: int = 2, pool_amp: float = -3.0, pool_width: float = 10000.0,
                pool_depth: float = 1500.0, u_top: float = 10.0, shear_depth: float = 2500.0,
                zf: np.ndarray | None = None) -> VVMState:
    """Sheared squall line on uniform levels: theta from stratified_theta
    (300 K + 3 K/km to 12 km, a stratosphere above, so deep domains stay warmer
    than the Tetens formula's 36 K singularity), qv at
    90 % relative humidity below 1.5 km falling linearly to 30 % at 10 km and
    dry_aloft above; u
    rising linearly from 0 to u_top over the lowest shear_depth, constant
    above; a cold pool of pool_amp (cosine-tapered, pool_width wide,
    pool_depth deep) at mid-domain; seeded N(0, 0.1 K) noise in the lowest
    1 km. w = 0; zeta follows from the shear. ``zf``: face heights of
    stretched levels (stretched_faces; ``dz`` is then its lowest spacing)."""
    g = GridSpec(NX, NZ, dx, dz, dt, 1)
    nz = g.nz
    zc = (np.arange(nz) - 0.5) * dz
    if zf is not None:
        zc = np.zeros(nz)
        zc[1:nz - 1] = 0.5 * (zf[1:nz - 1] + zf[2:nz])
        zc[0], zc[nz - 1] = zc[1], zc[nz - 2]
    rh = np.clip(np.where(zc <= 1500.0, 0.9, 0.9 - 0.6 * (zc - 1500.0) / 8500.0), 0.3, 0.9)
    rh = np.where(zc <= 10000.0, rh, dry_aloft(zc, 0.3))
    prof = base_state(g, stratified_theta, rh, zf=zf)
    nx = g.nx
    i = np.arange(nx)[:, None]
    x = (i - 0.5) * dx
    z = prof["z"][None, :]
    xc = 0.5 * NX * dx
    rx = np.abs(x - xc) / (0.5 * pool_width)
    rz = z / pool_depth
    pool = np.where((rx <= 1.0) & (rz <= 1.0),
                    pool_amp * np.cos(0.5 * np.pi * rx) ** 2 * np.cos(0.5 * np.pi * rz) ** 2, 0.0)
    rng = np.random.default_rng(seed)
    noise = np.where(z <= 1000.0, rng.normal(0.0, 0.1, (nx, nz)), 0.0)
    th = np.zeros((nx, nz))
    th[1:nx - 1, 1:nz - 1] = (prof["thb"][None, 1:nz - 1] + pool[1:nx - 1, 1:nz - 1]
                              + noise[1:nx - 1, 1:nz - 1])
    u = np.zeros((nx, nz))
    u[1:nx - 1, 1:nz - 1] = (u_top * np.minimum(z / shear_depth, 1.0))[:, 1:nz - 1] * np.ones((nx - 2, 1))
    return _assemble(g, prof, th, u, stretched=zf is not None)


def read_sounding(path) -> np.ndarray:
    """The rows of a sounding file as the reference reads it (Init::LoadFile,
    src/Init.cpp:301-312): a header line and the zero level are skipped, then
    whitespace-separated rows of ZZ, ZT, RHO, THBAR, PBAR, PIBAR, QVBAR, Q1LS,
    Q2LS, RHOZ, read while a whole row parses. Returns [rows][10]."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    words = " ".join(lines[2:]).split()
    vals = []
    for w in words:
        try:
            vals.append(float(w))
        except ValueError:
            break
    n = len(vals) // 10
    return np.array(vals[:10 * n], dtype=np.float64).reshape(n, 10)


def sounding_state(path, NX: int, NZ: int, dx: float, dz: float, dt: float, case: int = 1) -> VVMState:
    """The initial state of the reference's shipped configuration, which reads
    its base state from a sounding file (LOADFILE) and adds the large-scale
    Q1/Q2 forcing and the t = 0 random theta perturbation (TROPICALFORCING):

    * Init::LoadFile (src/Init.cpp:301-370): row r of the file is level
      k = r + 1 (thb, thb_init, qvb, pib, pb; rhou from RHOZ, rhow from RHO;
      Q1LS and Q2LS times 6), ghost levels copied, rhow at the top from rhou
      below it, then the Exner function from the pressure, pib = (pb/1e5)^(Rd/Cp);
    * the rest of Init1d (src/Init.cpp:116-134): thvb = thb + 0.61 qvb (the
      additive form of step 1), qvb0 = qvb, the level heights and lambda2;
    * Init2d (src/Init.cpp:138-182, 231-255): qv = qvb everywhere, qc = qr = 0,
      th = thb + the RandomPerturbation field of step 0 with the declaration's
      default range, +-0.25 K (src/Declare.hpp:870; the reference's own
      generator, made by the GPU library's host entry), u = w = zeta = 0.

    The file must hold at most NZ rows (the reference writes past its arrays
    otherwise); levels without a row keep zero, as the reference's arrays do."""
    from .gpu import random_perturbation_host
    g = GridSpec(NX, NZ, dx, dz, dt, case=case)
    nx, nz = g.nx, g.nz
    rows = read_sounding(path)
    if len(rows) > nz - 2:
        raise ValueError(f"sounding: {len(rows)} rows for {nz - 2} levels")
    thb, thb_init, qvb, pib, pb, rhou, rhow, q1, q2 = (np.zeros(nz) for _ in range(9))
    for r, (ZZ, ZT, RHO, THBAR, PBAR, PIBAR, QVBAR, Q1LS, Q2LS, RHOZ) in enumerate(rows):
        k = r + 1
        thb[k] = THBAR
        thb_init[k] = thb[k]
        qvb[k] = QVBAR
        pib[k] = PIBAR
        pb[k] = PBAR
        rhou[k] = RHOZ
        rhow[k] = RHO
        q1[k] = Q1LS * 6.
        q2[k] = Q2LS * 6.
    for a in (thb, thb_init, qvb, pib, pb, rhou, rhow):
        _center1d(a)
    rhow[nz - 1] = rhou[nz - 2]
    for k in range(nz - 1):
        pib[k] = math.pow(pb[k] / 100000., RD / CP)
    z = np.zeros(nz)
    z_zeta = np.zeros(nz)
    lambda2 = np.zeros(nz)
    for k in range(1, nz - 1):
        z[k] = (k - 0.5) * dz
        z_zeta[k] = (k - 1) * dz
        lambda2[k] = 1. / (1. / math.pow(0.23 * math.sqrt(dx * dz), 2) + 1. / math.pow(0.4 * 0.4 * z[k], 2))
    z[0], z[nz - 1] = z[1], z[nz - 2]
    z_zeta[0], z_zeta[nz - 1] = z_zeta[1], z_zeta[nz - 2]
    prof = dict(thb=thb, thvb=thb + 0.61 * qvb, qvb=qvb, pib=pib, pb=pb, rhou=rhou, rhow=rhow,
                thb_init=thb_init, qvb0=qvb.copy(), z=z, z_zeta=z_zeta, lambda2=lambda2, Q1LS=q1, Q2LS=q2)
    forcing = random_perturbation_host(g, 0, -0.25, 0.25, 1.)
    th = np.zeros((nx, nz))
    th[1:nx - 1, 1:nz - 1] = thb[None, 1:nz - 1] + forcing[1:nx - 1, 1:nz - 1]
    st = _assemble(g, prof, th, np.zeros((nx, nz)), np.zeros((nx, nz)))
    st.fields["qv"][:] = qvb[None, :]
    st.fields["init_th_forcing"] = forcing
    return st
