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


# ---------------------------------------------------------------- the full step

def _stretched_bubble(NX=128, NZ=64):
    from vvm_b200.initial_state import stretched_faces, warm_bubble
    return warm_bubble(NX, NZ, 200.0, 100.0, 1.0, zf=stretched_faces(NZ, 100.0, 500.0))


def test_stretched_step_keeps_discrete_continuity():
    """After stretched steps the velocities from cal_w and cal_u satisfy the
    anelastic continuity equation cell by cell,
    rhou_k (u[i+1] - u[i]) / dx + (rhow_{k+1} w_{k+1} - rhow_k w_k) / dc_k = 0,
    to round-off: the stretched Poisson operator, cal_u's column integral over
    the centre spacings and its top divergence over dc agree with each other."""
    from oracle.models import PortModel
    st = _stretched_bubble()
    m = PortModel(st.grid)
    m.load(st)
    for _ in range(30):
        m.one_step()
    u, w = m.field("u"), m.field("w")
    rhou, rhow, z, zz = (m.prof(n) for n in ("rhou", "rhow", "z", "z_zeta"))
    dc = 2.0 * (z - zz)
    nz = u.shape[1]
    div = np.array([rhou[k] * (u[2:, k] - u[1:-1, k]) / st.grid.dx
                    + (rhow[k + 1] * w[1:-1, k + 1] - rhow[k] * w[1:-1, k]) / dc[k] for k in range(1, nz - 1)])
    scale = np.abs(rhou[None, :] * u / st.grid.dx).max()
    assert scale > 1e-4 and np.abs(div).max() <= 1e-12 * scale


def test_stretched_advection_conserves_mass_weighted_scalar():
    """Flux-form advection divides each flux difference by its cell's
    thickness, so sum_k rhou_k dc_k sum_i (tendency) vanishes (periodic in x,
    no flux through the bottom and the top)."""
    from oracle.models import PortModel
    st = _stretched_bubble()
    m = PortModel(st.grid)
    m.load(st)
    for _ in range(10):
        m.one_step()
    m.step = 5
    m.call("Advection_thermo_th")
    d = m.hist("dth_advect")[:, :, (m.step + 1) % 2]
    rhou, z, zz = m.prof("rhou"), m.prof("z"), m.prof("z_zeta")
    dc = 2.0 * (z - zz)
    tot = np.sum(rhou[1:-1][None, :] * dc[1:-1][None, :] * d[1:-1, 1:-1])
    ref = np.sum(np.abs(rhou[1:-1][None, :] * dc[1:-1][None, :] * d[1:-1, 1:-1]))
    assert ref > 0 and abs(tot) <= 1e-12 * ref


def test_stretched_diffusion_leaves_linear_profile():
    """The vertical part of Hparam on stretched levels: a field linear in z
    (uniform in x) under constant K and constant density has no diffusive
    tendency; the uniform spacing formula would give one where the spacing
    changes."""
    from oracle.models import PortModel
    st = _stretched_bubble(32, 48)
    m = PortModel(st.grid)
    m.load(st)
    m.prof("rhou")[:] = 1.0
    m.prof("rhow")[:] = 1.0
    z = m.prof("z")
    lin = 1.0 + 1e-3 * z
    for n in ("thp", "qvp", "qcp", "qrp", "zetap"):
        m.field(n)[:] = lin[None, :]
    m.field("u")[:] = 0.0
    m.field("w")[:] = 0.0
    m.call("RKM_RKH")     # K = 10 everywhere (no deformation), then the sweeps
    # away from the boundary rows (whose ghosts are copies, not linear; the
    # in-place sweep carries that a few rows up, ~1e-3 a row)
    got = m.field("qcp")[1:-1, 8:-4]
    assert np.abs(got - lin[None, 8:-4]).max() <= 1e-13 * np.abs(lin).max()


def test_nearly_uniform_levels_approach_the_reference_step():
    """Levels perturbed by 1e-7 of their spacing take the stretched formulas;
    one step then stays within ~1e-6 of the reference's uniform step."""
    from oracle.models import PortModel
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(64, 32)
    sp = st.copy()
    nz = st.grid.nz
    j = np.arange(nz)
    sp.prof["z"] = st.prof["z"] * (1.0 + 1e-7 * np.sin(j))
    a = PortModel(st.grid)
    a.load(st)
    a.one_step()
    b = PortModel(sp.grid)
    b.load(sp)
    b.one_step()
    for n in ("zeta", "th", "u", "w"):
        x, y = b.field(n), a.field(n)
        assert np.linalg.norm(x - y) <= 1e-5 * np.linalg.norm(y), n
        if n in ("zeta", "u", "w"):
            assert not np.array_equal(x, y), n   # the stretched path really ran
