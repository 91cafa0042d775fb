"""The random theta forcing of Init::RandomPerturbation (src/Init.cpp:488-515)
made by the library on the host: the same numbers as the reference's own
routine (the compiled reference under oracle/_ref), bit for bit. No GPU."""
import numpy as np
import pytest

from oracle.models import RefModel, ref_available
from vvm_b200 import gpu as G
from vvm_b200.initial_state import warm_bubble

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("nx,nz,dz", [(64, 32, 100.0), (48, 20, 50.0), (33, 9, 250.0)])
def test_host_field_equals_reference(nx, nz, dz):
    st = warm_bubble(nx, nz, dz, dz)
    m = RefModel(st.grid, addforcingtime=5.0)
    m.load(st)
    for t in (0, 1, 2, 10):
        ours = G.random_perturbation_host(st.grid, t)
        ref = m.random_perturbation(t)
        assert np.array_equal(ours, ref), (nx, nz, dz, t)
        # only the levels below 200 m are forced, within the range
        zc = (np.arange(st.grid.nz) - 0.5) * dz
        assert np.all(ours[1:-1, (zc >= 200)[None, :][0] & (np.arange(st.grid.nz) < st.grid.nz - 1)] == 0)
        assert np.abs(ours).max() <= 1e-3 and np.count_nonzero(ours[1:-1, 1]) == nx


def test_other_ranges_and_steps_equal_reference():
    st = warm_bubble(40, 12, 100.0, 100.0)
    m = RefModel(st.grid, addforcingtime=5.0)
    m.load(st)
    for t, lo, hi, sd in ((3, -0.5, 0.25, 2.0), (12345, -1e-2, 1e-2, 0.5)):
        assert np.array_equal(G.random_perturbation_host(st.grid, t, lo, hi, sd), m.random_perturbation(t, lo, hi, sd))


def test_rejects_ranges_whose_redraw_would_not_end():
    st = warm_bubble(16, 8, 100.0, 100.0)
    with pytest.raises(G.VVMGpuError):
        G.random_perturbation_host(st.grid, 1, 0.01, -0.01, 1.0)
    with pytest.raises(G.VVMGpuError):
        G.random_perturbation_host(st.grid, 1, -0.01, 0.01, 0.0)
