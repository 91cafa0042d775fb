"""A run stopped, written to a restart file (vvm_b200.restart), read back
into a new context and continued equals the uninterrupted run bit for bit:
the file holds the AB2 history and every other input of the step. FP64 with
the spectral solve (the multigrid PCG's warm start extrapolates from the
last two solutions, which a new context does not have, so its first solves
after a restart agree only to the solver tolerance)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_restart_continues_bit_for_bit(tmp_path):
    from vvm_b200 import build, gpu as G
    from vvm_b200.initial_state import warm_bubble
    from vvm_b200.restart import read_restart, write_restart
    build.build()
    st = warm_bubble(128, 64)
    a = G.VVMGpu(st.grid, precision=G.VVM_PREC_FP64, solver=G.VVM_SOLVER_SPECTRAL)
    a.upload(st)
    a.step(15)
    ref = a.download()
    a.close()
    b = G.VVMGpu(st.grid, precision=G.VVM_PREC_FP64, solver=G.VVM_SOLVER_SPECTRAL)
    b.upload(st)
    b.step(7)
    write_restart(tmp_path / "r.nc", b.download())
    b.close()
    c = G.VVMGpu(st.grid, precision=G.VVM_PREC_FP64, solver=G.VVM_SOLVER_SPECTRAL)
    c.upload(read_restart(tmp_path / "r.nc"))
    c.step(8)
    out = c.download()
    c.close()
    assert out.scalars["step"] == ref.scalars["step"] == 15
    for n in ("zeta", "th", "qv", "qc", "qr", "u", "w", "RKM", "RKH"):
        assert np.array_equal(out.fields[n], ref.fields[n]), n
    for n in ref.hist:
        assert np.array_equal(out.hist[n], ref.hist[n]), n
    assert np.array_equal(out.precip, ref.precip)
