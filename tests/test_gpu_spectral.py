"""The Fourier-mode solver (VVM_SOLVER_SPECTRAL) against the reference and
against the multigrid-PCG path.

The Fourier-mode solve is the exact inverse of the cal_w operator up to
round-off: it is applied directly and its FP64 residual checked, so no CG
iteration normally follows (last_solve reports those iterations). The
reference comparisons use the same relative-L2 tolerances as the multigrid
path (tests/test_gpu_step.py).
"""
import numpy as np
import pytest

from conftest import golden, rel_l2
from tests_helpers import domain_means

PROG = ("zeta", "th", "qv", "qc", "qr", "u", "w")


@pytest.fixture(scope="module")
def gpu():
    from vvm_b200 import build, gpu as G
    build.build()
    return G


def test_spectral_rejects_non_power_of_two_nx():
    """Checked by create() before any device call (runs without a GPU)."""
    from vvm_b200 import build, gpu as G
    from vvm_b200.initial_state import GridSpec
    build.build()
    with pytest.raises(G.VVMGpuError) as e:
        G.VVMGpu(GridSpec(96, 32, 200.0, 200.0, 1.0), solver=G.VVM_SOLVER_SPECTRAL)
    assert e.value.code == 1 and "power of two" in str(e.value)


@pytest.mark.gpu
def test_spectral_poisson_manufactured_solution(gpu):
    from vvm_b200.initial_state import warm_bubble
    from oracle.models import PortModel
    z = golden("poisson_kat.npz")
    st = warm_bubble(int(z["NX"]), int(z["NZ"]))
    g = gpu.VVMGpu(st.grid, warm_start=False, solver=gpu.VVM_SOLVER_SPECTRAL)
    g.upload(st)
    W, it, rel = g.poisson_solve(z["b"], tol=1e-10)
    assert rel <= 1e-13 and it <= 1, (it, rel)   # CG iterations after the direct solve
    m = PortModel(st.grid)
    m.load(st)
    assert rel_l2(m.apply_A(W), z["b"]) <= 1e-13
    assert rel_l2(W, z["x_ans"]) <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("nstep,tol_dyn,tol_th", [(1, 1e-9, 1e-13), (10, 1e-8, 1e-12)])
def test_spectral_fp64_steps_match_reference(gpu, nstep, tol_dyn, tol_th):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble()
    g = gpu.VVMGpu(st.grid, solver=gpu.VVM_SOLVER_SPECTRAL)
    g.upload(st)
    g.step(nstep)
    out = g.download()
    z = golden(f"config1_step{nstep}.npz")
    for f in PROG:
        tol = tol_th if f in ("th", "qv") else tol_dyn
        assert rel_l2(out.fields[f], z[f]) <= tol, (f, rel_l2(out.fields[f], z[f]))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_spectral_graph_path_equals_host_loop_path(gpu, precision):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(128, 64)
    a = gpu.VVMGpu(st.grid, precision=precision, solver=gpu.VVM_SOLVER_SPECTRAL)
    a.upload(st)
    a.step(6)
    b = gpu.VVMGpu(st.grid, precision=precision, solver=gpu.VVM_SOLVER_SPECTRAL)
    b.upload(st)
    b.profile(True)
    b.step(6)
    da, db = a.download(), b.download()
    for f in PROG:
        assert np.array_equal(da.fields[f], db.fields[f]), f
    ia, ra = a.last_solve()
    ib, rb = b.last_solve()
    assert ia == ib and ra == rb and ra <= 1e-10


@pytest.mark.gpu
def test_spectral_and_multigrid_agree_at_2048x256(gpu):
    """Five steps of the benchmark grid with both solvers: the states agree
    to the solvers' tolerance."""
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(2048, 256, 100.0, 100.0)
    out = {}
    for s in (gpu.VVM_SOLVER_MGPCG, gpu.VVM_SOLVER_SPECTRAL):
        g = gpu.VVMGpu(st.grid, solver=s)
        g.upload(st)
        g.step(5)
        out[s] = g.download()
        it, rel = g.last_solve()
        assert rel <= 1e-10
        g.close()
    for f in PROG:
        e = rel_l2(out[gpu.VVM_SOLVER_SPECTRAL].fields[f], out[gpu.VVM_SOLVER_MGPCG].fields[f])
        assert e <= 1e-8, (f, e)


@pytest.mark.gpu
def test_spectral_largest_nx(gpu):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(8192, 32, 100.0, 100.0)
    g = gpu.VVMGpu(st.grid, solver=gpu.VVM_SOLVER_SPECTRAL)
    g.upload(st)
    g.step(2)
    out = g.download()
    assert all(np.isfinite(out.fields[f]).all() for f in PROG)
    it, rel = g.last_solve()
    assert rel <= 1e-12 and it <= 2


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_spectral_600_steps_domain_means(gpu, precision):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble()
    g = gpu.VVMGpu(st.grid, precision=precision, solver=gpu.VVM_SOLVER_SPECTRAL)
    g.upload(st)
    g.step(600)
    out = g.download()
    z = golden("config1_600.npz")
    got = domain_means(out)
    ref = z["means"][-1]
    if precision == 0:
        assert abs(got[0] - ref[0]) / abs(ref[0]) <= 1e-10
        for j in (1, 2, 3, 4):
            assert abs(got[j] - ref[j]) <= 1e-6 * max(abs(ref[j]), 1e-30), (j, got[j], ref[j])
    else:
        assert abs(got[0] - ref[0]) / abs(ref[0]) <= 1e-4
        assert abs(got[4] - ref[4]) / abs(ref[4]) <= 1e-2
