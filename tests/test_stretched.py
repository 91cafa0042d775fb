"""The cal_w operator on stretched levels (no counterpart in the reference):
its restatement (oracle/stretched_poisson.py) reduces to the reference's
matrix on uniform levels, and the level builder is what it claims."""
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "2d-vector-vorticity-model_b200"))


def test_uniform_levels_give_the_reference_matrix():
    from oracle.models import PortModel
    from oracle.stretched_poisson import metric, operator
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(32, 16)
    p = st.prof
    a, h = metric(p["z"], p["z_zeta"], st.grid.dx)
    assert np.array_equal(a, np.ones_like(a)) and np.array_equal(h, np.ones_like(h))
    A = operator(p["rhou"], p["rhow"], p["z"], p["z_zeta"], st.grid.dx, st.grid.NX)
    m = PortModel(st.grid)
    m.load(st)
    x = np.random.default_rng(1).standard_normal(A.shape[0])
    y_ref = m.apply_A(x)
    assert np.abs(A @ x - y_ref).max() <= 1e-12 * np.abs(y_ref).max()


def test_stretched_faces_and_base_state():
    from vvm_b200.initial_state import stretched_faces, stretched_poisson_case
    zf = stretched_faces(64, 100.0, 500.0)
    dz = np.diff(zf[1:])
    assert abs(dz[0] - 100.0) < 1e-9 and abs(dz[-1] - 500.0) < 1e-9 and np.all(np.diff(dz) > 0)
    st = stretched_poisson_case(64, 64)
    p = st.prof
    assert np.all(np.diff(p["z"][1:-1]) > 0) and np.all(p["pib"][1:-1] > 0)
    # centres midway between faces
    assert np.allclose(p["z"][1:-2], 0.5 * (p["z_zeta"][1:-2] + p["z_zeta"][2:-1]))
