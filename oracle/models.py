"""ctypes views of the two CPU oracles of the VVM step.

* ``RefModel``  -- oracle/_ref/libvvmref.so: the reference's own sources built
  by oracle/build_ref.sh behind oracle/ref_harness.cpp (uniform dx = dz only).
* ``RefTropicalModel`` -- oracle/_ref/libvvmref_tropical.so: the same sources
  built with the reference's sounding file and Q1/Q2 forcing switched on
  (oracle/ref_config_tropical.hpp), for the initial state read from it.
* ``RefStreamModel`` -- oracle/_ref/libvvmref_stream.so: the same sources
  built with the streamfunction formulation (STREAMFUNCTION) switched on
  (oracle/ref_config_stream.hpp), for calpsiuw.
* ``RefDropinModel`` -- oracle/_ref/libvvmref_dropin.so: the reference model
  as a maintainer builds it with GPU_STEP, TimeMarching taken from the
  committed binding 2d-vector-vorticity-model_b200/integration/
  Iteration_GPU.cpp (the B200 step through libvvmgpu.so). Not an oracle: the
  thing the tests check against RefModel.
* ``PortModel`` -- oracle/_build/libvvmoracle.so: the C restatement in
  oracle/vvm_oracle.c (exact elliptic solves).
* ``PortMTModel`` -- oracle/_build/libvvmoracle_mt.so: the same source built
  with OpenMP and FFT-based cal_w, the race-free multi-core CPU baseline.

Test infrastructure only: used by tests/, the fixture generator under
tests/golden/, __graft_entry__.smoke() and bench.py's CPU-baseline leg. Arrays
are numpy views onto the model's own memory in the reference's [nx][nz] layout.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libvvmref.so"
REF_TROPICAL_LIB = HERE / "_ref" / "libvvmref_tropical.so"
REF_STREAM_LIB = HERE / "_ref" / "libvvmref_stream.so"
REF_DROPIN_LIB = HERE / "_ref" / "libvvmref_dropin.so"
PORT_LIB = HERE / "_build" / "libvvmoracle.so"
PORT_MT_LIB = HERE / "_build" / "libvvmoracle_mt.so"

HIST_NAMES = ("dzeta_advect", "dth_buoyancy", "dth_advect", "dqv_advect", "dqc_advect",
              "dqr_advect", "dqr_VT")
PROF_NAMES = ("rhou", "rhow", "thb", "thvb", "qvb", "pib", "pb", "thb_init", "qvb0", "z",
              "z_zeta", "lambda2")
FIELD_NAMES = ("zeta", "zetap", "th", "thp", "qv", "qvp", "qc", "qcp", "qr", "qrp", "u", "w",
               "RKM", "RKH")
PAST = {"zeta": "zetam", "th": "thm", "qv": "qvm", "qc": "qcm", "qr": "qrm"}

_libs: dict = {}


def _load(path: Path, prefix: str):
    key = (str(path), prefix)
    if key in _libs:
        return _libs[key]
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built")
    L = ctypes.CDLL(str(path))
    vp, ip, dp, cp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    f = lambda n: getattr(L, prefix + n)  # noqa: E731
    f("create").restype = vp
    f("destroy").argtypes = [vp]
    f("dims").argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
    for n in ("field", "hist", "prof", "scalar"):
        f(n).restype = ctypes.POINTER(dp)
        f(n).argtypes = [vp, cp]
    f("step_ptr").restype = ctypes.POINTER(ip)
    f("step_ptr").argtypes = [vp]
    f("call").restype = ip
    f("call").argtypes = [vp, cp]
    f("apply_A").argtypes = [vp, ctypes.POINTER(dp), ctypes.POINTER(dp)]
    _libs[key] = L
    return L


def ref_available() -> bool:
    return REF_LIB.exists()


def ref_tropical_available() -> bool:
    return REF_TROPICAL_LIB.exists()


def ref_stream_available() -> bool:
    return REF_STREAM_LIB.exists()


def ref_dropin_available() -> bool:
    return REF_DROPIN_LIB.exists()


def port_available() -> bool:
    return PORT_LIB.exists()


def port_mt_available() -> bool:
    return PORT_MT_LIB.exists()


def _view(ptr, shape):
    n = int(np.prod(shape))
    return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(shape)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class _CModel:
    prefix = ""
    path = None

    def __init__(self, grid):
        self.L = _load(self.path, self.prefix)
        self.grid = grid
        self.h = self._create(grid)
        nx, nz = ctypes.c_int(), ctypes.c_int()
        self._f("dims")(self.h, ctypes.byref(nx), ctypes.byref(nz))
        self.nx, self.nz = nx.value, nz.value
        if (self.nx, self.nz) != (grid.nx, grid.nz):
            raise ValueError(f"model grid {self.nx}x{self.nz} != {grid.nx}x{grid.nz}")

    def _f(self, n):
        return getattr(self.L, self.prefix + n)

    def close(self):
        if getattr(self, "h", None):
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, name):
        p = self._f("field")(self.h, name.encode())
        if not p:
            raise KeyError(name)
        return _view(p, (self.nx, self.nz))

    def hist(self, name):
        p = self._f("hist")(self.h, name.encode())
        if not p:
            raise KeyError(name)
        return _view(p, (self.nx, self.nz, 2))

    def prof(self, name):
        p = self._f("prof")(self.h, name.encode())
        if not p:
            raise KeyError(name)
        n = {"xi": self.nx, "uxi": self.nx, "precip": self.nx}.get(name, self.nz)
        return _view(p, (n,))

    def scalar(self, name, n=1):
        p = self._f("scalar")(self.h, name.encode())
        if not p:
            raise KeyError(name)
        return _view(p, (n,))

    @property
    def step(self) -> int:
        return self._f("step_ptr")(self.h)[0]

    @step.setter
    def step(self, v: int):
        self._f("step_ptr")(self.h)[0] = int(v)

    def load(self, st):
        """Copies a VVMState (vvm_b200.initial_state) into the model."""
        for name in FIELD_NAMES:
            self.field(name)[:] = st.fields[name]
        for now, past in PAST.items():
            self.field(past)[:] = st.fields[now]
        for name, a in st.hist.items():
            self.hist(name)[:] = a
        for name, a in st.prof.items():
            self.prof(name)[:] = a
        self.prof("thbm")[:] = st.prof["thb"]
        self.prof("thvbm")[:] = st.prof["thvb"]
        self.scalar("ubarTop")[0] = st.scalars["ubarTop"]
        self.scalar("ubarTopm")[0] = st.scalars["ubarTop"]
        self.scalar("ubarTopp")[0] = st.scalars.get("ubarTopp", 0.0)
        self.scalar("dubarTop_advect", 2)[:] = st.scalars["dubarTop_advect"]
        self.step = st.scalars.get("step", 0)
        if st.precip is not None:
            self.prof("precip")[:] = st.precip
        self._after_load()

    def _after_load(self):
        pass

    def dump(self):
        """Returns a VVMState copy of the model's current state."""
        from vvm_b200.initial_state import VVMState
        st = VVMState(self.grid)
        st.fields = {n: self.field(n).copy() for n in FIELD_NAMES}
        st.hist = {n: self.hist(n).copy() for n in HIST_NAMES}
        st.prof = {n: self.prof(n).copy() for n in PROF_NAMES}
        st.scalars = dict(ubarTop=float(self.scalar("ubarTop")[0]),
                          ubarTopp=float(self.scalar("ubarTopp")[0]),
                          dubarTop_advect=self.scalar("dubarTop_advect", 2).copy(),
                          step=self.step)
        st.precip = self.prof("precip").copy()
        return st

    def call(self, routine: str):
        if self._f("call")(self.h, routine.encode()) != 0:
            raise KeyError(routine)

    def one_step(self):
        self.call("one_step")

    # w-equation matrix of cal_w (src/PoissonSolver.cpp:760-796); unknown
    # index (k-2)*(nx-2) + (i-1), k = 2..nz-2, i = 1..nx-2.
    def apply_A(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._f("apply_A")(self.h, _dptr(x), _dptr(y))
        return y


class RefModel(_CModel):
    """The reference `vvm` object (src/Declare.hpp:73) built as src/main.cpp does."""
    prefix = "ref_"
    path = REF_LIB

    def __init__(self, grid, tolerance: float = 1e-22, addforcingtime: float = 0.0):
        self._tol, self._aft = tolerance, addforcingtime
        super().__init__(grid)
        self._poisson_ready = False

    def _create(self, g):
        L = self.L
        L.ref_create.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 3 + \
            [ctypes.c_int] + [ctypes.c_double] * 3
        return L.ref_create(g.NX, g.NZ, float(g.dx), float(g.dz), float(g.dt), int(g.case),
                            float(g.moisture_nudge_time), float(self._tol), float(self._aft))

    def _after_load(self):
        if not self._poisson_ready:
            self.L.ref_init_poisson.argtypes = [ctypes.c_void_p]
            self.L.ref_init_poisson(self.h)
            self._poisson_ready = True

    def random_perturbation(self, t: int, min_range: float = -0.001, max_range: float = 0.001,
                            standard_deviation: float = 1.0) -> np.ndarray:
        """vvm::Init::RandomPerturbation (src/Init.cpp:488-515): the reference's
        own field of step t, returned as a copy of init_th_forcing [nx][nz]."""
        self.L.ref_random_perturbation.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 3
        self.L.ref_random_perturbation(self.h, int(t), float(min_range), float(max_range),
                                       float(standard_deviation))
        return np.array(self.field("init_th_forcing"))

    def time_marching(self, nsteps: int):
        """vvm::Iteration::TimeMarching from step 0 (src/Iteration.cpp:208-438)."""
        self.L.ref_time_marching.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self.L.ref_time_marching(self.h, int(nsteps))

    def solve_A(self, b: np.ndarray):
        """BiCGSTAB + IncompleteLUT as cal_w configures it."""
        L = self.L
        L.ref_solve_A.restype = ctypes.c_int
        L.ref_solve_A.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_double)]
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty_like(b)
        it, err = ctypes.c_int(), ctypes.c_double()
        rc = L.ref_solve_A(self.h, _dptr(b), _dptr(x), ctypes.byref(it), ctypes.byref(err))
        return x, it.value, err.value, rc


class RefTropicalModel(RefModel):
    """The reference built with LOADFILE and TROPICALFORCING: Init1d reads its
    1D base state from the reference's input/init.txt (src/Init.cpp:301-370)."""
    path = REF_TROPICAL_LIB

    @classmethod
    def init_path(cls) -> str:
        """The sounding file the build reads (compiled in by build_ref.sh)."""
        L = _load(cls.path, cls.prefix)
        L.ref_init_path.restype = ctypes.c_char_p
        return L.ref_init_path().decode()

    def init(self):
        """vvm::Init::Init1d then Init2d, as src/main.cpp:81-82 runs them."""
        self.L.ref_init.argtypes = [ctypes.c_void_p]
        self.L.ref_init(self.h)
        self._after_load()   # the cal_w matrix, as after load()


class RefStreamModel(RefModel):
    """The reference built with STREAMFUNCTION (POISSONPARAM = 0): its one_step
    calls calpsiuw in place of pubarTop_pt + cal_w + cal_u
    (src/Iteration.cpp:289-295), and apply_A is the psi matrix
    (src/PoissonSolver.cpp:726-756)."""
    path = REF_STREAM_LIB

    def psi(self) -> np.ndarray:
        return self.field("psi")


class RefDropinModel(RefModel):
    """The reference model whose TimeMarching is the GPU_STEP binding: its
    time_marching(n) runs n steps on the GPU through the C ABI, exactly as a
    maintainer's GPU_STEP build would."""
    path = REF_DROPIN_LIB


class PortModel(_CModel):
    """The C restatement (oracle/vvm_oracle.c)."""
    prefix = "orc_"
    path = PORT_LIB

    def __init__(self, grid, addforcingtime: float = 0.0):
        self._aft = addforcingtime
        super().__init__(grid)

    def _create(self, g):
        L = self.L
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 3 + \
            [ctypes.c_int] + [ctypes.c_double] * 2
        return L.orc_create(g.NX, g.NZ, float(g.dx), float(g.dz), float(g.dt), int(g.case),
                            float(g.moisture_nudge_time), float(self._aft))

    def set_streamfunction(self, on: bool = True):
        """one_step calls calpsiuw in place of pubarTop_pt + cal_w + cal_u."""
        self.L.orc_set_streamfunction.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self.L.orc_set_streamfunction(self.h, int(bool(on)))

    def apply_psi(self, x: np.ndarray) -> np.ndarray:
        """y = A_psi x, the streamfunction matrix (src/PoissonSolver.cpp:726-756)."""
        self.L.orc_apply_psi.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double)]
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self.L.orc_apply_psi(self.h, _dptr(x), _dptr(y))
        return y

    def solve_A(self, b: np.ndarray) -> np.ndarray:
        self.L.orc_solve_A.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double)]
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty_like(b)
        self.L.orc_solve_A(self.h, _dptr(b), _dptr(x))
        return x


class PortMTModel(PortModel):
    """The C restatement built with OpenMP (rows split across threads, the
    five Gauss-Seidel sweeps concurrent, per-thread domain sums) and radix-2
    FFTs in cal_w: the race-free multi-core CPU baseline. Its results equal
    the serial restatement's to round-off (sum order and transform)."""
    path = PORT_MT_LIB

    def threads(self) -> int:
        self.L.orc_threads.restype = ctypes.c_int
        return int(self.L.orc_threads())
