"""Shared test setup: import paths, the `gpu` marker, fixture loaders."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
for p in (str(REPO / "2d-vector-vorticity-model_b200"), str(REPO)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return float(d / n) if n > 0 else float(d)


def golden(name: str):
    return np.load(GOLDEN / name)


def kat_state():
    """The input state of routines_kat.npz, rebuilt from the fixture."""
    from vvm_b200.initial_state import GridSpec, VVMState
    z = golden("routines_kat.npz")
    nx, nz = z["in_th"].shape
    st = VVMState(GridSpec(nx - 2, nz - 2, 200.0, 200.0, 1.0))
    st.fields = {k[3:]: z[k].copy() for k in z.files if k.startswith("in_") and z[k].ndim == 2}
    st.hist = {k[4:]: z[k].copy() for k in z.files if k.startswith("inh_")}
    st.prof = {k[4:]: z[k].copy() for k in z.files if k.startswith("inp_")}
    st.scalars = dict(ubarTop=float(z["in_ubarTop"]), ubarTopp=0.0,
                      dubarTop_advect=z["in_dubar"].copy(), step=int(z["in_step"]))
    st.precip = np.zeros(nx)
    return st, z


@pytest.fixture(scope="session")
def port_lib():
    from oracle import models
    if not models.port_available():
        import subprocess
        subprocess.run(["make", "-s", "-C", str(REPO / "oracle")], check=True)
    return models
