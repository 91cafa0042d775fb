"""ctypes binding of libvvmgpu.so (include/vvm_gpu.h).

The host side mirrors the reference's own objects: a ``VVMGpu`` owns one
device context built from a ``vvm_gpu_desc`` (Config_VVM, src/Declare.hpp:27),
takes and returns states in the reference model's [nx][nz] layout
(``VVMState``), and exposes one method per reference routine of
vvm::Iteration::TimeMarching (src/Iteration.cpp:262-434) plus the fused
``step``. Failures raise ``VVMGpuError`` with the library's message.

There is no CPU fallback: loading fails loudly when the library or a GPU is
missing.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from .initial_state import HIST, VVMState

PKG = Path(__file__).resolve().parent.parent
LIB_PATH = PKG / "lib" / "libvvmgpu.so"

VVM_PREC_FP64, VVM_PREC_MIXED = 0, 1
VVM_SOLVER_MGPCG, VVM_SOLVER_LEARNED, VVM_SOLVER_SPECTRAL = 0, 1, 2
VVM_FLAG_FIXED_FORCING = 1
VVM_FLAG_STREAMFUNCTION = 2
STATUS = {0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ENOCONV", 4: "ESTATE"}

_dp = ctypes.POINTER(ctypes.c_double)


class VVMGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Desc(ctypes.Structure):
    _fields_ = [("NX", ctypes.c_int), ("NZ", ctypes.c_int),
                ("dx", ctypes.c_double), ("dz", ctypes.c_double), ("dt", ctypes.c_double),
                ("gravity", ctypes.c_double), ("cp", ctypes.c_double), ("cv", ctypes.c_double),
                ("rd", ctypes.c_double), ("lv", ctypes.c_double), ("p0", ctypes.c_double),
                ("psurf", ctypes.c_double), ("poisson_tol", ctypes.c_double),
                ("poisson_maxit", ctypes.c_int), ("case_id", ctypes.c_int),
                ("moisture_nudge_time", ctypes.c_double), ("addforcingtime", ctypes.c_double),
                ("precision", ctypes.c_int), ("solver", ctypes.c_int),
                ("warm_start", ctypes.c_int), ("flags", ctypes.c_int)]


_F2 = ("zeta", "zetap", "th", "thp", "qv", "qvp", "qc", "qcp", "qr", "qrp", "u", "w", "RKM", "RKH")
_H = ("dzeta_advect", "dth_buoyancy", "dth_advect", "dqv_advect", "dqc_advect", "dqr_advect",
      "dqr_VT")
_P = ("rhou", "rhow", "thb", "thvb", "qvb", "pib", "pb", "thb_init", "qvb0", "z", "z_zeta",
      "lambda2")


class HostState(ctypes.Structure):
    _fields_ = ([(n, _dp) for n in _F2] + [(n, _dp) for n in _H] + [(n, _dp) for n in _P] +
                [("Q1LS", _dp), ("Q2LS", _dp), ("init_th_forcing", _dp), ("precip", _dp),
                 ("ubarTop", ctypes.c_double), ("ubarTopp", ctypes.c_double),
                 ("dubarTop_advect", ctypes.c_double * 2), ("step", ctypes.c_int)])


# Kernel classes of vvm_gpu_profile_read (VVM_K_* in include/vvm_gpu.h).
KERNEL_CLASSES = ("pzeta", "padv", "apply", "pubar", "poisson_rhs", "cg", "mg_sweep", "mg_restrict",
                  "mg_coarse", "cal_u", "kessler", "rkm", "gs", "mean", "learned", "conv")

ROUTINES = ("pzeta", "pth", "pqv", "pqc", "pqr", "add_forcing", "halo_all", "pubartop", "cal_w",
            "cal_u", "kessler", "update_mean", "turbulence", "nudge", "next_step", "calpsiuw")

EXPORTS = ("vvm_gpu_desc_default", "vvm_gpu_create", "vvm_gpu_destroy", "vvm_gpu_set_stream",
           "vvm_gpu_synchronize", "vvm_gpu_last_error", "vvm_gpu_upload_state",
           "vvm_gpu_download_state", "vvm_gpu_upload_prognostic", "vvm_gpu_download_prognostic",
           "vvm_gpu_set_step", "vvm_gpu_get_step", "vvm_gpu_step", "vvm_gpu_poisson_solve",
           "vvm_gpu_poisson_solve_device", "vvm_gpu_last_solve", "vvm_gpu_profile",
           "vvm_gpu_profile_read", "vvm_gpu_launch_count", "vvm_gpu_poisson_solve_noalloc",
           "vvm_gpu_set_tuning", "vvm_gpu_get_tuning", "vvm_gpu_batch_create", "vvm_gpu_batch_destroy",
           "vvm_gpu_batch_case", "vvm_gpu_batch_step", "vvm_gpu_batch_synchronize",
           "vvm_gpu_batch_autotune", "vvm_gpu_batch_last_error", "vvm_gpu_batch_stream",
           "vvm_gpu_batch_grouping",
           "vvm_gpu_conv3x3_c32", "vvm_gpu_learned_shape", "vvm_gpu_learned_weights",
           "vvm_gpu_learned_eval", "vvm_gpu_learned_train", "vvm_gpu_learned_config",
           "vvm_gpu_learned_last", "vvm_gpu_learned_time", "vvm_gpu_learned_train_rhs",
           "vvm_gpu_random_perturbation", "vvm_gpu_random_perturbation_host",
           "vvm_gpu_download_psi") + tuple(
               "vvm_gpu_" + r for r in ROUTINES)

_lib = None


def load_library(path: Path | None = None):
    """Loads libvvmgpu.so (no compute; works without a GPU)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is not built; run __graft_entry__.build()")
    L = ctypes.CDLL(str(p))
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.vvm_gpu_desc_default.argtypes = [ctypes.POINTER(Desc), ip, ip, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double]
    L.vvm_gpu_desc_default.restype = None
    L.vvm_gpu_create.argtypes = [ctypes.POINTER(Desc), ip, ctypes.POINTER(vp)]
    L.vvm_gpu_destroy.argtypes = [vp]
    L.vvm_gpu_set_stream.argtypes = [vp, vp]
    L.vvm_gpu_synchronize.argtypes = [vp]
    L.vvm_gpu_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    for n in ("upload_state", "download_state", "upload_prognostic", "download_prognostic"):
        getattr(L, "vvm_gpu_" + n).argtypes = [vp, ctypes.POINTER(HostState)]
    L.vvm_gpu_set_step.argtypes = [vp, ip]
    L.vvm_gpu_get_step.argtypes = [vp, ctypes.POINTER(ip)]
    L.vvm_gpu_step.argtypes = [vp, ip]
    L.vvm_gpu_poisson_solve.argtypes = [vp, _dp, _dp, ctypes.c_double, ctypes.POINTER(ip), _dp]
    L.vvm_gpu_poisson_solve_device.argtypes = [vp, vp, vp, ctypes.c_double,
                                               ctypes.POINTER(ip), _dp]
    L.vvm_gpu_last_solve.argtypes = [vp, ctypes.POINTER(ip), _dp]
    L.vvm_gpu_poisson_solve_noalloc.argtypes = [ip, ip, _dp, _dp, vp, vp, ctypes.c_double, ip, vp,
                                                ctypes.POINTER(ip), _dp]
    L.vvm_gpu_set_tuning.argtypes = [vp, ip, ip]
    L.vvm_gpu_get_tuning.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.vvm_gpu_batch_create.argtypes = [ctypes.POINTER(Desc), ip, ip, ctypes.POINTER(vp)]
    L.vvm_gpu_batch_destroy.argtypes = [vp]
    L.vvm_gpu_batch_case.argtypes = [vp, ip, ctypes.POINTER(vp)]
    L.vvm_gpu_batch_step.argtypes = [vp, ip]
    L.vvm_gpu_batch_synchronize.argtypes = [vp]
    L.vvm_gpu_batch_autotune.argtypes = [vp, ip, ctypes.POINTER(ip)]
    L.vvm_gpu_batch_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    L.vvm_gpu_batch_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.vvm_gpu_batch_grouping.argtypes = [vp, ip, ctypes.POINTER(ip)]
    _fp = ctypes.POINTER(ctypes.c_float)
    L.vvm_gpu_conv3x3_c32.argtypes = [_fp, _fp, _fp, ip, ip, ip, ip]
    L.vvm_gpu_learned_shape.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.vvm_gpu_learned_weights.argtypes = [vp, _fp, _fp, ip]
    L.vvm_gpu_learned_eval.argtypes = [vp, _fp, _fp, _fp, _fp, _dp]
    L.vvm_gpu_learned_train.argtypes = [vp, ip, ip, ip, ctypes.c_double, ip, _dp, _dp]
    L.vvm_gpu_learned_config.argtypes = [vp, ip, ip]
    L.vvm_gpu_learned_last.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.vvm_gpu_learned_time.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.vvm_gpu_learned_train_rhs.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ip, ip, ip, ctypes.c_double, ip,
                                            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    dbl = ctypes.c_double
    L.vvm_gpu_random_perturbation.argtypes = [vp, ip, dbl, dbl, dbl]
    L.vvm_gpu_random_perturbation_host.argtypes = [ip, ip, dbl, ip, dbl, dbl, dbl, _dp]
    L.vvm_gpu_profile.argtypes = [vp, ip]
    L.vvm_gpu_profile_read.argtypes = [vp, ip, _dp, ctypes.POINTER(ctypes.c_longlong)]
    L.vvm_gpu_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.vvm_gpu_download_psi.argtypes = [vp, _dp]
    for r in ROUTINES:
        getattr(L, "vvm_gpu_" + r).argtypes = [vp]
    if path is None:
        _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def poisson_solve_noalloc(NX: int, NZ: int, rhou: np.ndarray, rhow: np.ndarray, d_b: int, d_W: int,
                          tol: float = 1e-10, maxit: int = 10000, stream: int = 0):
    """vvm_gpu_poisson_solve_noalloc: the cal_w solve on caller-owned device
    buffers (raw pointers, NX*(NZ-1) doubles) with no context and no device
    allocation. Returns (iterations, relative residual)."""
    L = load_library()
    rhou = np.ascontiguousarray(rhou, dtype=np.float64)
    rhow = np.ascontiguousarray(rhow, dtype=np.float64)
    if rhou.size < NZ + 2 or rhow.size < NZ + 2:
        raise ValueError("rhou and rhow need NZ+2 values")
    it, rel = ctypes.c_int(), ctypes.c_double()
    rc = L.vvm_gpu_poisson_solve_noalloc(int(NX), int(NZ), _ptr(rhou), _ptr(rhow), ctypes.c_void_p(d_b),
                                         ctypes.c_void_p(d_W), float(tol), int(maxit),
                                         ctypes.c_void_p(stream), ctypes.byref(it), ctypes.byref(rel))
    if rc != 0:
        buf = ctypes.create_string_buffer(512)
        L.vvm_gpu_last_error(None, buf, 512)
        raise VVMGpuError(rc, buf.value.decode())
    return it.value, rel.value


def random_perturbation_host(grid, t: int, min_range: float = -0.001, max_range: float = 0.001,
                             standard_deviation: float = 1.0) -> np.ndarray:
    """Init::RandomPerturbation's field of step t for `grid` ([nx][nz], ghost
    cells filled), made on the host by the library (no GPU needed)."""
    L = load_library()
    out = np.zeros((grid.NX + 2, grid.NZ + 2))
    rc = L.vvm_gpu_random_perturbation_host(int(grid.NX), int(grid.NZ), float(grid.dz), int(t),
                                            float(min_range), float(max_range), float(standard_deviation),
                                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        raise VVMGpuError(rc, "random_perturbation_host: needs min_range <= max_range and standard_deviation > 0")
    return out


class VVMGpu:
    """One GPU context of the VVM step (a `vvm` model living in HBM)."""

    def __init__(self, grid, precision: int = VVM_PREC_FP64, solver: int = VVM_SOLVER_MGPCG,
                 poisson_tol: float = 1e-10, warm_start: bool = True, device: int = 0,
                 addforcingtime: float = 0.0, poisson_maxit: int = 200, fixed_forcing: bool = False,
                 streamfunction: bool = False):
        self.L = load_library()
        self.grid = grid
        self.owned = True
        d = self.make_desc(self.L, grid, precision, solver, poisson_tol, warm_start, addforcingtime,
                           poisson_maxit, fixed_forcing, streamfunction)
        self.desc = d
        h = ctypes.c_void_p()
        rc = self.L.vvm_gpu_create(ctypes.byref(d), int(device), ctypes.byref(h))
        if rc != 0:
            raise VVMGpuError(rc, self._err(None))
        self.h = h
        self._keep = []

    @staticmethod
    def make_desc(L, grid, precision=VVM_PREC_FP64, solver=VVM_SOLVER_MGPCG, poisson_tol=1e-10,
                  warm_start=True, addforcingtime=0.0, poisson_maxit=200, fixed_forcing=False,
                  streamfunction=False):
        """vvm_gpu_desc of a grid (reference defaults, then the options).
        fixed_forcing keeps the uploaded init_th_forcing at every forced step
        instead of regenerating it each step as TimeMarching does;
        streamfunction steps with calpsiuw in place of pubarTop_pt, cal_w and
        cal_u (the reference's STREAMFUNCTION switch)."""
        d = Desc()
        L.vvm_gpu_desc_default(ctypes.byref(d), grid.NX, grid.NZ, float(grid.dx),
                                    float(grid.dz), float(grid.dt))
        d.case_id = int(grid.case)
        d.moisture_nudge_time = float(grid.moisture_nudge_time)
        d.addforcingtime = float(addforcingtime)
        d.precision = int(precision)
        d.solver = int(solver)
        d.poisson_tol = float(poisson_tol)
        d.poisson_maxit = int(poisson_maxit)
        d.warm_start = 1 if warm_start else 0
        d.flags = (VVM_FLAG_FIXED_FORCING if fixed_forcing else 0) | \
            (VVM_FLAG_STREAMFUNCTION if streamfunction else 0)
        return d

    @classmethod
    def _borrow(cls, L, handle, grid, desc):
        """A view of a context another object owns (a batch's case)."""
        self = cls.__new__(cls)
        self.L, self.grid, self.desc, self.h, self.owned, self._keep = L, grid, desc, handle, False, []
        return self

    def _err(self, h):
        buf = ctypes.create_string_buffer(512)
        self.L.vvm_gpu_last_error(h, buf, 512)
        return buf.value.decode()

    def _check(self, rc):
        if rc != 0:
            raise VVMGpuError(rc, self._err(self.h))

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "owned", True):
                self.L.vvm_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state -----------------------------------------------------------
    def _host_state(self, st: VVMState, with_all: bool):
        hs = HostState()
        keep = []

        def put(name, a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            setattr(hs, name, _ptr(a))

        for n in _F2:
            if n in st.fields and (with_all or n in ("zeta", "th", "qv", "qc", "qr", "u", "w")):
                put(n, st.fields[n])
        if with_all:
            for n in _H:
                if n in st.hist:
                    put(n, st.hist[n])
            for n in _P:
                put(n, st.prof[n])
            for n in ("Q1LS", "Q2LS"):
                if n in st.prof:
                    put(n, st.prof[n])
            if "init_th_forcing" in st.fields:
                put("init_th_forcing", st.fields["init_th_forcing"])
            if st.precip is not None:
                put("precip", st.precip)
            hs.ubarTop = float(st.scalars["ubarTop"])
            hs.ubarTopp = float(st.scalars.get("ubarTopp", 0.0))
            hs.dubarTop_advect[0] = float(st.scalars["dubarTop_advect"][0])
            hs.dubarTop_advect[1] = float(st.scalars["dubarTop_advect"][1])
            hs.step = int(st.scalars.get("step", 0))
        return hs, keep

    def upload(self, st: VVMState):
        hs, keep = self._host_state(st, True)
        self._check(self.L.vvm_gpu_upload_state(self.h, ctypes.byref(hs)))
        # inputs the step reads but never changes: download() returns them too,
        # so a downloaded state is complete (a restart file holds it all)
        self._const = {"prof": {n: np.array(st.prof[n]) for n in tuple(_P) + ("Q1LS", "Q2LS") if n in st.prof},
                       "fields": {n: np.array(st.fields[n]) for n in ("init_th_forcing",) if n in st.fields}}

    def download(self) -> VVMState:
        g = self.grid
        st = VVMState(g)
        nx, nz = g.nx, g.nz
        st.fields = {n: np.zeros((nx, nz)) for n in _F2}
        st.hist = {n: np.zeros((nx, nz, 2)) for n in _H}
        st.prof = {n: np.zeros(nz) for n in ("thb", "qvb", "thvb", "rhou", "rhow")}
        st.precip = np.zeros(nx)
        hs = HostState()
        for n, a in st.fields.items():
            setattr(hs, n, _ptr(a))
        for n, a in st.hist.items():
            setattr(hs, n, _ptr(a))
        for n, a in st.prof.items():
            setattr(hs, n, _ptr(a))
        hs.precip = _ptr(st.precip)
        self._check(self.L.vvm_gpu_download_state(self.h, ctypes.byref(hs)))
        st.scalars = dict(ubarTop=hs.ubarTop, ubarTopp=hs.ubarTopp,
                          dubarTop_advect=np.array([hs.dubarTop_advect[0], hs.dubarTop_advect[1]]),
                          step=hs.step)
        const = getattr(self, "_const", None)
        if const:
            for n, a in const["prof"].items():
                st.prof.setdefault(n, a.copy())
            for n, a in const["fields"].items():
                st.fields.setdefault(n, a.copy())
        return st

    def upload_prognostic(self, fields: dict):
        hs = HostState()
        keep = []
        for n in ("zeta", "th", "qv", "qc", "qr", "u", "w"):
            a = np.ascontiguousarray(fields[n], dtype=np.float64)
            keep.append(a)
            setattr(hs, n, _ptr(a))
        self._check(self.L.vvm_gpu_upload_prognostic(self.h, ctypes.byref(hs)))

    def download_prognostic(self, out: dict):
        hs = HostState()
        for n in ("zeta", "th", "qv", "qc", "qr", "u", "w"):
            setattr(hs, n, _ptr(out[n]))
        self._check(self.L.vvm_gpu_download_prognostic(self.h, ctypes.byref(hs)))

    # -- stepping ----------------------------------------------------------
    @property
    def step_count(self) -> int:
        v = ctypes.c_int()
        self._check(self.L.vvm_gpu_get_step(self.h, ctypes.byref(v)))
        return v.value

    @step_count.setter
    def step_count(self, v: int):
        self._check(self.L.vvm_gpu_set_step(self.h, int(v)))

    def call(self, routine: str):
        self._check(getattr(self.L, "vvm_gpu_" + routine)(self.h))

    def step(self, nsteps: int = 1):
        self._check(self.L.vvm_gpu_step(self.h, int(nsteps)))

    def time_marching_routines(self, nsteps: int = 1):
        """The reference's TimeMarching body, one C-ABI call per routine
        (src/Iteration.cpp:246-434), the forcing field of the step made before
        AddForcing while step*dt <= addforcingtime (:276-283)."""
        for _ in range(nsteps):
            step = self.step_count + 1
            self.step_count = step
            for r in ("pzeta", "pth", "pqv", "pqc", "pqr"):
                self.call(r)
            if step * self.desc.dt <= self.desc.addforcingtime and not (self.desc.flags & VVM_FLAG_FIXED_FORCING):
                self.random_perturbation(step)
            poisson = ("calpsiuw",) if self.desc.flags & VVM_FLAG_STREAMFUNCTION else ("pubartop", "cal_w", "cal_u")
            for r in ("add_forcing", "halo_all", *poisson, "halo_all", "kessler",
                      "halo_all", "update_mean", "turbulence", "nudge", "next_step"):
                self.call(r)

    def download_psi(self) -> np.ndarray:
        """The streamfunction of the last calpsiuw, [nx][nz] with ghosts."""
        out = np.empty((self.grid.nx, self.grid.nz))
        self._check(self.L.vvm_gpu_download_psi(self.h, _ptr(out)))
        return out

    def random_perturbation(self, t: int, min_range: float = -0.001, max_range: float = 0.001,
                            standard_deviation: float = 1.0):
        """Init::RandomPerturbation (src/Init.cpp:488-515) into the device's
        init_th_forcing, with the reference's own generator."""
        self._check(self.L.vvm_gpu_random_perturbation(self.h, int(t), float(min_range), float(max_range),
                                                        float(standard_deviation)))

    def set_stream(self, stream_handle: int | None):
        self._check(self.L.vvm_gpu_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)))

    def synchronize(self):
        self._check(self.L.vvm_gpu_synchronize(self.h))

    def profile(self, enable: bool = True):
        """Starts (and resets) or stops the per-kernel-class event timers."""
        self._check(self.L.vvm_gpu_profile(self.h, 1 if enable else 0))

    def profile_read(self) -> dict:
        """{class: (device ms, launches)} accumulated since profile(True)."""
        out = {}
        for k, name in enumerate(KERNEL_CLASSES):
            ms, n = ctypes.c_double(), ctypes.c_longlong()
            self._check(self.L.vvm_gpu_profile_read(self.h, k, ctypes.byref(ms), ctypes.byref(n)))
            out[name] = (ms.value, n.value)
        return out

    @property
    def launch_count(self) -> int:
        n = ctypes.c_longlong()
        self._check(self.L.vvm_gpu_launch_count(self.h, ctypes.byref(n)))
        return n.value

    def set_tuning(self, gs_tile_rows: int = 0, fft_threads: int = 0):
        """Launch-shape knobs (0: automatic): the Gauss-Seidel schedule (tile
        rows 4/8/16/32, or 1 for one cluster a field) and the row-FFT block."""
        self._check(self.L.vvm_gpu_set_tuning(self.h, int(gs_tile_rows), int(fft_threads)))

    def tuning(self) -> tuple[int, int]:
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.vvm_gpu_get_tuning(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    # -- learned preconditioner (VVM_SOLVER_LEARNED) -----------------------
    def learned_shape(self) -> tuple[int, int, int]:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.L.vvm_gpu_learned_shape(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def learned_weights(self, new: np.ndarray | None = None) -> np.ndarray:
        fp = ctypes.POINTER(ctypes.c_float)
        n = self.learned_shape()[2]
        out = np.empty(n, dtype=np.float32)
        src = None if new is None else np.ascontiguousarray(new, dtype=np.float32)
        self._check(self.L.vvm_gpu_learned_weights(self.h, out.ctypes.data_as(fp),
                                                   None if src is None else src.ctypes.data_as(fp), n))
        return out

    def learned_eval(self, x: np.ndarray, t: np.ndarray | None = None):
        """z = net(x); with t also (dL/dweights, L)."""
        fp = ctypes.POINTER(ctypes.c_float)
        H0, W0, n = self.learned_shape()
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(H0, W0)
        z = np.empty((H0, W0), dtype=np.float32)
        grad = np.empty(n, dtype=np.float32) if t is not None else None
        tt = None if t is None else np.ascontiguousarray(t, dtype=np.float32).reshape(H0, W0)
        loss = ctypes.c_double()
        self._check(self.L.vvm_gpu_learned_eval(self.h, x.ctypes.data_as(fp),
                                                None if tt is None else tt.ctypes.data_as(fp),
                                                z.ctypes.data_as(fp),
                                                None if grad is None else grad.ctypes.data_as(fp),
                                                ctypes.byref(loss)))
        return (z, grad, loss.value) if t is not None else z

    def learned_train(self, npairs: int, steps: int, batch: int = 4, lr: float = 1e-3, seed: int = 0):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.L.vvm_gpu_learned_train(self.h, int(npairs), int(steps), int(batch), float(lr),
                                                 int(seed), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def learned_train_rhs(self, b: np.ndarray, steps: int, batch: int = 4, lr: float = 1e-3, seed: int = 0):
        """Trains on the given right-hand sides b [npairs][NX*(NZ-1)] (each
        solved by the plain solver); returns (mean loss of the first, last ten
        Adam steps)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        npairs = b.shape[0]
        l0, l1 = ctypes.c_double(), ctypes.c_double()
        self._check(self.L.vvm_gpu_learned_train_rhs(self.h, b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                     int(npairs), int(steps), int(batch), float(lr), int(seed),
                                                     ctypes.byref(l0), ctypes.byref(l1)))
        return l0.value, l1.value

    def learned_config(self, mode: int = 0, cap: int = 200):
        self._check(self.L.vvm_gpu_learned_config(self.h, int(mode), int(cap)))

    def learned_time(self, reps: int = 20) -> tuple[float, float]:
        """(ms per network forward pass, ms per pass of its six convolutions)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.L.vvm_gpu_learned_time(self.h, int(reps), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def learned_last(self) -> tuple[int, int]:
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.vvm_gpu_learned_last(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def last_solve(self):
        it, rel = ctypes.c_int(), ctypes.c_double()
        self._check(self.L.vvm_gpu_last_solve(self.h, ctypes.byref(it), ctypes.byref(rel)))
        return it.value, rel.value

    def poisson_solve(self, b: np.ndarray, W0: np.ndarray | None = None, tol: float = 1e-10):
        b = np.ascontiguousarray(b, dtype=np.float64)
        W = np.zeros_like(b) if W0 is None else np.ascontiguousarray(W0, dtype=np.float64).copy()
        it, rel = ctypes.c_int(), ctypes.c_double()
        self._check(self.L.vvm_gpu_poisson_solve(self.h, _ptr(b), _ptr(W), float(tol),
                                                 ctypes.byref(it), ctypes.byref(rel)))
        return W, it.value, rel.value

    def poisson_solve_device(self, d_b: int, d_W: int, tol: float = 1e-10):
        it, rel = ctypes.c_int(), ctypes.c_double()
        self._check(self.L.vvm_gpu_poisson_solve_device(self.h, ctypes.c_void_p(d_b),
                                                        ctypes.c_void_p(d_W), float(tol),
                                                        ctypes.byref(it), ctypes.byref(rel)))
        return it.value, rel.value


class VVMBatch:
    """Independent cases of any sizes advancing together, one CUDA graph a
    step for all of them (vvm_gpu_batch_*). `cases[i]` is a VVMGpu view of
    case i (owned by the batch) for upload, download and queries."""

    def __init__(self, grids, precision: int = VVM_PREC_MIXED, solver: int = VVM_SOLVER_SPECTRAL,
                 device: int = 0, **desc_options):
        self.L = load_library()
        grids = list(grids)
        descs = (Desc * len(grids))()
        for i, g in enumerate(grids):
            descs[i] = VVMGpu.make_desc(self.L, g, precision, solver, **desc_options)
        h = ctypes.c_void_p()
        rc = self.L.vvm_gpu_batch_create(descs, len(grids), int(device), ctypes.byref(h))
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.L.vvm_gpu_last_error(None, buf, 512)
            raise VVMGpuError(rc, buf.value.decode())
        self.h = h
        self.cases = []
        for i, g in enumerate(grids):
            c = ctypes.c_void_p()
            self._check(self.L.vvm_gpu_batch_case(self.h, i, ctypes.byref(c)))
            self.cases.append(VVMGpu._borrow(self.L, c, g, descs[i]))

    def _check(self, rc):
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.L.vvm_gpu_batch_last_error(self.h, buf, 512)
            raise VVMGpuError(rc, buf.value.decode())

    def upload(self, states):
        for c, st in zip(self.cases, states):
            c.upload(st)

    def step(self, n: int = 1):
        self._check(self.L.vvm_gpu_batch_step(self.h, int(n)))

    def synchronize(self):
        self._check(self.L.vvm_gpu_batch_synchronize(self.h))

    @property
    def stream(self) -> int:
        """cudaStream_t of the batch graphs (for timing events)."""
        p = ctypes.c_void_p()
        self._check(self.L.vvm_gpu_batch_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def grouping(self, max_cases: int | bool | None = None) -> int:
        """Sets the most cases one grouped launch takes (False or 0: no
        grouped launches; True: the default of 32; None: unchanged); returns
        the number of grouped launch groups in the last captured step graph."""
        if max_cases is True:
            max_cases = 32
        v = -1 if max_cases is None else int(max_cases)
        n = ctypes.c_int()
        self._check(self.L.vvm_gpu_batch_grouping(self.h, v, ctypes.byref(n)))
        return n.value

    def autotune(self, reps: int = 3) -> int:
        n = ctypes.c_int()
        self._check(self.L.vvm_gpu_batch_autotune(self.h, int(reps), ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "h", None):
            for c in self.cases:
                c.h = None
            self.L.vvm_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def conv3x3_c32(x: np.ndarray, w: np.ndarray, adjoint: bool = False, device: int = 0) -> np.ndarray:
    """vvm_gpu_conv3x3_c32: x [H][W][32], w [9][32][32] (tap = 3 (dy+1) + dx+1,
    in, out) -> [H][W][32] on the tensor cores (BF16 operands, FP32
    accumulation, BF16 result)."""
    L = load_library()
    x = np.ascontiguousarray(x, dtype=np.float32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    H, W = x.shape[0], x.shape[1]
    assert x.shape == (H, W, 32) and w.shape == (9, 32, 32)
    y = np.empty_like(x)
    fp = ctypes.POINTER(ctypes.c_float)
    rc = L.vvm_gpu_conv3x3_c32(x.ctypes.data_as(fp), w.ctypes.data_as(fp), y.ctypes.data_as(fp), H, W,
                               1 if adjoint else 0, int(device))
    if rc != 0:
        buf = ctypes.create_string_buffer(512)
        L.vvm_gpu_last_error(None, buf, 512)
        raise VVMGpuError(rc, buf.value.decode())
    return y
