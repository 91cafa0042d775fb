"""Restart files (vvm_b200.restart): the classic-NetCDF writer and reader
round-trip a full state exactly, and scipy's independent NetCDF-3 reader
sees the same variables, dimensions and values."""
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "2d-vector-vorticity-model_b200"))


def _same(a, b):
    return all(np.array_equal(a.fields[n], b.fields[n]) for n in a.fields) and \
        all(np.array_equal(a.hist[n], b.hist[n]) for n in a.hist) and \
        all(np.array_equal(a.prof[n], b.prof[n]) for n in a.prof) and np.array_equal(a.precip, b.precip)


def test_round_trip_is_exact(tmp_path):
    from vvm_b200.initial_state import random_state
    from vvm_b200.restart import read_restart, write_restart
    st = random_state(32, 16, seed=5)
    st.scalars["ubarTopp"] = 0.25
    p = tmp_path / "s.nc"
    write_restart(p, st)
    back = read_restart(p)
    assert _same(st, back)
    assert back.scalars["step"] == st.scalars["step"] and back.scalars["ubarTop"] == st.scalars["ubarTop"]
    assert np.array_equal(back.scalars["dubarTop_advect"], st.scalars["dubarTop_advect"])
    assert (back.grid.NX, back.grid.NZ, back.grid.dx, back.grid.dt) == (32, 16, st.grid.dx, st.grid.dt)


def test_scipy_reads_the_file(tmp_path):
    from scipy.io import netcdf_file
    from vvm_b200.initial_state import random_state
    from vvm_b200.restart import write_restart
    st = random_state(24, 12, seed=2)
    p = tmp_path / "s.nc"
    write_restart(p, st)
    with netcdf_file(str(p), "r", mmap=False) as f:
        assert f.dimensions["x"] == 26 and f.dimensions["z"] == 14 and f.dimensions["ab2"] == 2
        assert f.variables["th"].dimensions == ("x", "z")
        assert np.array_equal(f.variables["th"][:], st.fields["th"])
        assert np.array_equal(f.variables["dth_advect"][:], st.hist["dth_advect"])
        assert int(f.variables["step"].getValue()) == st.scalars["step"]
        assert f.NX == 24
