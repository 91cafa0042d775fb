"""Poisson solves on stretched levels (the stretched-level Poisson workload's grid type:
dz from 100 m to 500 m on a tanh ramp, dx = 250 m) against the restatement
in oracle/stretched_poisson.py, solved directly by scipy: each solver reaches
the reference's residual ||b - A W|| / ||b|| <= 1e-10 with the stretched A,
and W agrees with the direct solve to 1e-8. The step refuses such a state."""
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


def test_step_refuses_stretched_levels(case):
    G, st, A, b, Wd = case
    g = G.VVMGpu(st.grid)
    g.upload(st)
    with pytest.raises(G.VVMGpuError) as e:
        g.step(1)
    assert e.value.code == 1   # VVM_GPU_EINVAL
    g.close()
