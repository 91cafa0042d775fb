"""The drop-in proof: the reference model built as a maintainer would build it
with GPU_STEP (oracle/build_ref.sh, REF_VARIANT=dropin): every reference
translation unit, except that vvm::Iteration::TimeMarching comes from the
committed binding 2d-vector-vorticity-model_b200/integration/Iteration_GPU.cpp
and runs the step on the GPU through libvvmgpu.so. The same `vvm` object,
configured and loaded the same way, is stepped by the reference's own
TimeMarching (CPU) and by the GPU_STEP one; the final arrays of the model
must agree within the FP64 step bars (th and qv 1e-12, zeta, u, w 1e-8 after
10 steps, relative L2), with the random th forcing on for the first 10 s, as
the reference's main runs it (addforcingtime = 10).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def models():
    from vvm_b200 import build
    build.build()
    from oracle import models as M
    if not (M.ref_dropin_available() and M.ref_available()):
        pytest.skip("the reference builds (oracle/_ref) are not present")
    return M


@pytest.mark.parametrize("addforcingtime", [0.0, 10.0])
def test_gpu_step_binding_equals_reference_time_marching(models, addforcingtime):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(64, 32)
    cpu = models.RefModel(st.grid, addforcingtime=addforcingtime)
    cpu.load(st)
    cpu.time_marching(12)
    gpu = models.RefDropinModel(st.grid, addforcingtime=addforcingtime)
    gpu.load(st)
    gpu.time_marching(12)
    assert gpu.step == cpu.step == 12
    for n, b in (("th", 1e-12), ("qv", 1e-12), ("zeta", 1e-8), ("u", 1e-8), ("w", 1e-8),
                 ("thp", 1e-12), ("zetap", 1e-8)):
        e = rel_l2(gpu.field(n), cpu.field(n))
        assert e <= b, (n, e)
    assert abs(gpu.scalar("ubarTop")[0] - cpu.scalar("ubarTop")[0]) <= 1e-10 * max(1.0, abs(cpu.scalar("ubarTop")[0]))
    if addforcingtime > 0:
        # the forcing really ran: th differs from an unforced run
        ref = models.RefModel(st.grid, addforcingtime=0.0)
        ref.load(st)
        ref.time_marching(12)
        assert not np.array_equal(ref.field("th"), cpu.field("th"))
