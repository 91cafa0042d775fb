"""The streamfunction formulation on the GPU (vvm_gpu_calpsiuw and
VVM_FLAG_STREAMFUNCTION) against the reference built with STREAMFUNCTION
(fixture tests/golden/stream_kat.npz, POISSONPARAM = 0) and, for grids the
fixture does not cover, the C restatement.

Bounds (relative L2 over whole fields, ghosts included): psi, u, w of one
call 1e-10 (the psi solve stops at ||b - A psi|| / ||b|| <= 1e-10; the
reference's BiCGSTAB at 1e-31 requested); after 1 and 10 FP64 steps th and qv
1e-13, zeta, u, w, psi 1e-9; the mixed step 1e-5 after one step.
"""
import numpy as np
import pytest

from conftest import golden, kat_state, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from vvm_b200 import build, gpu as G
    build.build()
    return G


def test_calpsiuw_matches_reference_fixture(gpu):
    st, _ = kat_state()
    z = golden("stream_kat.npz")
    g = gpu.VVMGpu(st.grid, streamfunction=True)
    g.upload(st)
    g.call("calpsiuw")
    out = g.download()
    psi = g.download_psi()
    it, rel = g.last_solve()
    g.close()
    assert rel <= 1e-10
    assert rel_l2(psi, z["calpsiuw__psi"]) <= 1e-10, rel_l2(psi, z["calpsiuw__psi"])
    for n in ("u", "w"):
        assert rel_l2(out.fields[n], z[f"calpsiuw__{n}"]) <= 1e-10, (n, rel_l2(out.fields[n], z[f"calpsiuw__{n}"]))


@pytest.mark.parametrize("steps", [1, 10])
def test_stream_steps_match_reference_fixture(gpu, steps):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(64, 32)
    z = golden("stream_kat.npz")
    g = gpu.VVMGpu(st.grid, streamfunction=True)
    g.upload(st)
    g.step(steps)
    out = g.download()
    psi = g.download_psi()
    g.close()
    for n in ("zeta", "th", "qv", "u", "w"):
        bound = 1e-13 if n in ("th", "qv") else 1e-9
        e = rel_l2(out.fields[n], z[f"step{steps}__{n}"])
        assert e <= bound, (n, e)
    assert rel_l2(psi, z[f"step{steps}__psi"]) <= 1e-9


def test_stream_routine_sequence_equals_fused_step(gpu):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(64, 32)
    a = gpu.VVMGpu(st.grid, streamfunction=True)
    a.upload(st)
    a.step(3)
    b = gpu.VVMGpu(st.grid, streamfunction=True)
    b.upload(st)
    b.time_marching_routines(3)
    fa, fb = a.download().fields, b.download().fields
    for n in ("zeta", "th", "qv", "u", "w"):
        assert rel_l2(fa[n], fb[n]) <= 1e-13, n
    a.close()
    b.close()


def test_mixed_stream_step(gpu):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(64, 32)
    z = golden("stream_kat.npz")
    g = gpu.VVMGpu(st.grid, precision=gpu.VVM_PREC_MIXED, streamfunction=True)
    g.upload(st)
    g.step(1)
    out = g.download()
    g.close()
    for n, b in (("zeta", 1e-5), ("th", 1e-8), ("u", 1e-5), ("w", 1e-5)):
        assert rel_l2(out.fields[n], z[f"step1__{n}"]) <= b, n


def test_multigrid_psi_solve_on_odd_grid_against_restatement(gpu, port_lib):
    """NX = 48 is not a power of two: the psi system goes to multigrid-PCG.
    Checked against the restatement's exact solve and the psi matrix."""
    from vvm_b200.initial_state import random_state
    st = random_state(48, 20, seed=5)
    st.fields["zetap"] = st.fields["zeta"] * 1.01
    g = gpu.VVMGpu(st.grid, streamfunction=True)
    g.upload(st)
    g.call("calpsiuw")
    psi = g.download_psi()
    out = g.download()
    g.close()
    m = port_lib.PortModel(st.grid)
    m.load(st)
    m.call("calpsiuw")
    assert rel_l2(psi, m.field("psi")) <= 1e-9
    assert rel_l2(out.fields["w"], m.field("w")) <= 1e-9
    x = psi[1:-1, 2:-1].T.reshape(-1)
    b = (st.fields["zetap"][1:-1, 2:-1] * st.grid.dx ** 2).T.reshape(-1)
    assert np.linalg.norm(b - m.apply_psi(x)) / np.linalg.norm(b) <= 1e-10


def test_stream_errors(gpu):
    import ctypes
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(32, 16)
    g = gpu.VVMGpu(st.grid, streamfunction=True)
    g.upload(st)
    with pytest.raises(gpu.VVMGpuError) as e:
        g.download_psi()             # calpsiuw has not run yet
    assert e.value.code == 4         # VVM_GPU_ESTATE
    g.close()
    # a batch refuses the flag (its graph cannot hold the host-read residual)
    L = gpu.load_library()
    d = gpu.VVMGpu.make_desc(L, st.grid, streamfunction=True)
    h = ctypes.c_void_p()
    assert L.vvm_gpu_batch_create(ctypes.byref(d), 1, 0, ctypes.byref(h)) == 1
    buf = ctypes.create_string_buffer(256)
    L.vvm_gpu_last_error(None, buf, 256)
    assert b"streamfunction" in buf.value
