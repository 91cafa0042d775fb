"""Batches of independent cases (vvm_gpu_batch_*) and the launch-shape knobs.

A batch runs every case's step as a branch of one CUDA graph, with the same
kernels a single context launches, so each case must come out bit for bit
equal to the same case stepped on its own with the same knobs. The knobs
the autotuner turns: the Gauss-Seidel schedule (tiles of 4 to 32 rows, or one
cluster a field) and the row-FFT block. The tile heights and the FFT block
change no arithmetic, so results stay bit-identical across them; the cluster
schedule associates the recurrence's carries differently, so it agrees with
the tiles to round-off (1e-13 relative). The autotuner must leave every
case's state exactly as it found it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROG = ("zeta", "th", "qv", "qc", "qr", "u", "w")


@pytest.fixture(scope="module")
def gpu():
    from vvm_b200 import build, gpu as G
    build.build()
    return G


def _states(shapes):
    from vvm_b200.initial_state import warm_bubble
    return [warm_bubble(nx, nz, 200.0, 200.0, radius=max(400.0, nx * 200 / 8)) for nx, nz in shapes]


def _alone(G, st, n, precision, solver, tuning=None):
    g = G.VVMGpu(st.grid, precision=precision, solver=solver)
    if tuning is not None:
        g.set_tuning(*tuning)
    g.upload(st)
    g.step(n)
    out = g.download()
    g.close()
    return out


def _same(a, b):
    return all(np.array_equal(a.fields[f], b.fields[f]) for f in PROG)


@pytest.mark.parametrize("precision,solver,shapes", [
    (1, 2, [(64, 32), (128, 48), (256, 32)]),           # mixed, spectral
    (0, 0, [(64, 32), (96, 33), (128, 24)]),            # FP64, multigrid, non-power-of-two NX
])
def test_batch_equals_cases_alone(gpu, precision, solver, shapes):
    sts = _states(shapes)
    b = gpu.VVMBatch([s.grid for s in sts], precision=precision, solver=solver)
    b.upload(sts)
    b.step(3)          # the first steps run case by case, then the batch graph
    b.step(4)
    b.synchronize()
    for st, c in zip(sts, b.cases):
        assert _same(c.download(), _alone(gpu, st, 7, precision, solver))
    b.close()


def test_autotune_restores_state_and_keeps_results(gpu):
    shapes = [(64, 32), (64, 32), (256, 32)]
    sts = _states(shapes)
    b = gpu.VVMBatch([s.grid for s in sts], precision=1, solver=2)
    b.upload(sts)
    b.step(3)
    b.synchronize()
    before = [c.download() for c in b.cases]
    ngroups = b.autotune(reps=2)
    assert ngroups == 2
    after = [c.download() for c in b.cases]
    for x, y in zip(before, after):
        assert _same(x, y)
    for c in b.cases:
        tr, fft = c.tuning()
        assert tr in (1, 4, 8, 16, 32) and fft in (128, 256, 512, 32, 64)
    b.step(4)
    b.synchronize()
    for st, c in zip(sts, b.cases):
        # alone: the first three steps with the default knobs, as the batch
        # ran them before the autotuner, then the tuned ones
        g = gpu.VVMGpu(st.grid, precision=1, solver=2)
        g.upload(st)
        g.step(3)
        g.set_tuning(*c.tuning())
        g.step(4)
        assert _same(c.download(), g.download())
        g.close()
    b.close()


def test_knobs_leave_results_unchanged(gpu):
    st = _states([(512, 32)])[0]
    ref = _alone(gpu, st, 5, 1, 2)
    for tr, fft in ((4, 128), (16, 512), (32, 64)):
        g = gpu.VVMGpu(st.grid, precision=1, solver=2)
        g.set_tuning(tr, fft)
        g.upload(st)
        g.step(5)
        assert g.tuning()[0] == tr
        assert _same(g.download(), ref), (tr, fft)
        g.close()
    g = gpu.VVMGpu(st.grid, precision=1, solver=2)
    with pytest.raises(gpu.VVMGpuError):
        g.set_tuning(12, 0)                  # not a tile height
    g.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_cluster_schedule_agrees_with_tiles(gpu, precision):
    """The two Gauss-Seidel schedules, each exact to round-off, on 5 steps."""
    from conftest import rel_l2
    st = _states([(512, 48)])[0]
    a = _alone(gpu, st, 5, precision, 2)
    b = _alone(gpu, st, 5, precision, 2, (1, 0))
    for f in PROG:
        assert rel_l2(b.fields[f], a.fields[f]) <= (1e-13 if precision == 0 else 1e-6), f


def test_batch_rejects_cases_at_different_steps(gpu):
    sts = _states([(64, 32), (64, 32)])
    b = gpu.VVMBatch([s.grid for s in sts], precision=1, solver=2)
    b.upload(sts)
    b.cases[0].step(1)
    with pytest.raises(gpu.VVMGpuError) as e:
        b.step(1)
    assert e.value.code == 4
    b.close()


def _varied(shapes):
    """Distinct cases of each shape: bubbles of other amplitudes, places and
    sizes (amplitude 0: a resting atmosphere, whose cal_w right-hand side is
    zero)."""
    from vvm_b200.initial_state import warm_bubble
    out = []
    for j, (nx, nz) in enumerate(shapes):
        amp = (0.0, 1.0, 2.5, 6.0)[j % 4]
        out.append(warm_bubble(nx, nz, 200.0, 200.0, amp=amp, radius=max(400.0, nx * 200 / (6 + j % 3)),
                               xc_frac=0.3 + 0.1 * (j % 5)))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_grouped_launches_equal_cases_alone(gpu, precision):
    """Cases of one shape step as grouped launches (one launch a kernel for
    the group, blockIdx.z the case); each case must still equal itself
    stepped alone, bit for bit, and equal the batch with grouping off."""
    shapes = [(64, 32)] * 4 + [(128, 48)] * 3 + [(256, 32)]
    sts = _varied(shapes)
    outs = {}
    # at most 32 cases a launch (both shapes one group each), at most 2 (4 cases
    # in two groups, 3 in a group of 2 and one case alone), none
    for limit, groups in ((32, 2), (2, 3), (0, 0)):
        b = gpu.VVMBatch([s.grid for s in sts], precision=precision, solver=2)
        b.grouping(limit)
        b.upload(sts)
        b.step(3)
        b.step(5)
        b.synchronize()
        assert b.grouping() == groups, limit
        outs[limit] = [c.download() for c in b.cases]
        b.close()
    for j, st in enumerate(sts):
        alone = _alone(gpu, st, 8, precision, 2)
        for limit in outs:
            assert _same(outs[limit][j], alone), (j, limit)


def test_grouped_loop_gates_cases(gpu):
    """A tolerance the direct solve's check does not meet makes CG iterate in
    the moving cases of a group while the resting case (zero right-hand
    side) leaves its loop at once: the grouped loop runs while any case
    needs it, and a case that has left it must not iterate."""
    shapes = [(128, 48)] * 4
    sts = _varied(shapes)
    tol = 1e-14
    b = gpu.VVMBatch([s.grid for s in sts], precision=0, solver=2, poisson_tol=tol)
    b.upload(sts)
    b.step(3)
    b.step(3)
    b.synchronize()
    assert b.grouping() == 1
    iters = [c.last_solve()[0] for c in b.cases]
    assert iters[0] == 0 and max(iters) > 0, iters
    for st, c in zip(sts, b.cases):
        g = gpu.VVMGpu(st.grid, precision=0, solver=2, poisson_tol=tol)
        g.upload(st)
        g.step(6)
        assert _same(c.download(), g.download())
        g.close()
    b.close()
