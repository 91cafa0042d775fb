"""Poisson solves on stretched levels (the stretched-level Poisson workload's grid type:
dz from 100 m to 500 m on a tanh ramp, dx = 250 m) against the restatement
in oracle/stretched_poisson.py, solved directly by scipy: each solver reaches
the reference's residual ||b - A W|| / ||b|| <= 1e-10 with the stretched A,
and W agrees with the direct solve to 1e-8. The full step on stretched levels
against the C restatement's (oracle/vvm_oracle.c, levels()): relative L2 of
every prognostic field within 1e-9 after 1 and 10 FP64 steps, the mixed step
within 1e-5 (zeta, u, w) and 1e-8 (th) after one; the streamfunction
formulation, which keeps the reference's uniform matrix, refuses such a
state."""
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))


@pytest.fixture(scope="module")
def case():
    from vvm_b200 import build, gpu as G
    from vvm_b200.initial_state import stretched_poisson_case
    from oracle.stretched_poisson import operator, rhs, solve
    build.build()
    st = stretched_poisson_case(256, 96, seed=7)
    p = st.prof
    A = operator(p["rhou"], p["rhow"], p["z"], p["z_zeta"], st.grid.dx, st.grid.NX)
    b = rhs(p["rhow"], st.fields["zeta"], st.grid.dx)
    return G, st, A, b, solve(A, b)


def _true_rel(A, W, b):
    return np.linalg.norm(b - A @ W) / np.linalg.norm(b)


@pytest.mark.parametrize("precision,solver", [(0, 0), (1, 0), (0, 2), (1, 2)])
def test_stretched_solve_matches_direct(case, precision, solver):
    G, st, A, b, Wd = case
    g = G.VVMGpu(st.grid, precision=precision, solver=solver)
    g.upload(st)
    W, it, rel = g.poisson_solve(b)
    assert rel <= 1e-10
    assert _true_rel(A, W, b) <= 1.5e-10
    assert np.linalg.norm(W - Wd) <= 1e-8 * np.linalg.norm(Wd)
    g.close()


def test_learned_on_stretched_levels_beats_the_cycle_without_it(case):
    G, st, A, b, Wd = case
    from vvm_b200.initial_state import stretched_poisson_case
    from oracle.stretched_poisson import rhs
    train = np.stack([rhs(st.prof["rhow"], stretched_poisson_case(256, 96, seed=100 + s).fields["zeta"],
                          st.grid.dx) for s in range(12)])
    its = {}
    for mode in (0, 1):
        g = G.VVMGpu(st.grid, solver=G.VVM_SOLVER_LEARNED)
        g.upload(st)
        if mode == 0:
            l0, l1 = g.learned_train_rhs(train, steps=200, batch=2, lr=2e-3, seed=3)
            assert l1 < l0
        g.learned_config(mode=mode, cap=3000)
        W, it, rel = g.poisson_solve(b)
        fcg, fell = g.learned_last()
        assert not fell and rel <= 1e-10 and _true_rel(A, W, b) <= 1.5e-10
        assert np.linalg.norm(W - Wd) <= 1e-8 * np.linalg.norm(Wd)
        its[mode] = fcg
        g.close()
    assert its[0] < its[1], its


def test_streamfunction_refuses_stretched_levels(case):
    G, st, A, b, Wd = case
    g = G.VVMGpu(st.grid, streamfunction=True)
    g.upload(st)
    with pytest.raises(G.VVMGpuError) as e:
        g.step(1)
    assert e.value.code == 1   # VVM_GPU_EINVAL
    g.close()


def _bubble():
    from vvm_b200.initial_state import stretched_faces, warm_bubble
    return warm_bubble(128, 64, 200.0, 100.0, 1.0, zf=stretched_faces(64, 100.0, 500.0))


def _squall():
    from vvm_b200.initial_state import squall_line, stretched_faces
    return squall_line(256, 64, 250.0, 100.0, 2.0, zf=stretched_faces(64, 100.0, 500.0))


PROG = ("zeta", "th", "qv", "qc", "qr", "u", "w")


@pytest.mark.parametrize("make", [_bubble, _squall])
@pytest.mark.parametrize("solver", [0, 2])
def test_stretched_fp64_step_matches_restatement(case, make, solver):
    from conftest import rel_l2
    from oracle.models import PortModel
    G = case[0]
    st = make()
    g = G.VVMGpu(st.grid, solver=solver)
    g.upload(st)
    m = PortModel(st.grid)
    m.load(st)
    done = 0
    for n in (1, 10):
        g.step(n - done)
        for _ in range(n - done):
            m.one_step()
        done = n
        out = g.download()
        for f in PROG:
            ref = m.field(f)
            if np.linalg.norm(ref) == 0:
                assert np.abs(out.fields[f]).max() == 0, (n, f)
                continue
            e = rel_l2(out.fields[f], ref)
            assert e <= 1e-9, (n, f, e)
    _, rel = g.last_solve()
    assert rel <= 1e-10
    g.close()


def test_stretched_mixed_one_step(case):
    from conftest import rel_l2
    from oracle.models import PortModel
    G = case[0]
    st = _bubble()
    g = G.VVMGpu(st.grid, precision=G.VVM_PREC_MIXED, solver=G.VVM_SOLVER_SPECTRAL)
    g.upload(st)
    g.step(1)
    out = g.download()
    m = PortModel(st.grid)
    m.load(st)
    m.one_step()
    for f, bound in (("zeta", 1e-5), ("u", 1e-5), ("w", 1e-5), ("th", 1e-8), ("qv", 1e-8)):
        assert rel_l2(out.fields[f], m.field(f)) <= bound, f
    g.close()
