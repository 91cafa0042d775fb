"""The initial state of the reference's shipped configuration, read from its
sounding file (Init::LoadFile, src/Init.cpp:301-370) with the large-scale
Q1/Q2 forcing and the random theta perturbation on (TROPICALFORCING), and the
steps that follow: against the reference built with those switches
(oracle/_ref/libvvmref_tropical.so, from oracle/ref_config_tropical.hpp).
No GPU."""
import numpy as np
import pytest

from conftest import rel_l2
from oracle.models import FIELD_NAMES, RefTropicalModel, ref_tropical_available
from vvm_b200 import gpu as G
from vvm_b200.initial_state import read_sounding, sounding_state

pytestmark = pytest.mark.skipif(not ref_tropical_available(), reason="oracle/_ref tropical build absent")

PROFILES = ("thb", "thb_init", "qvb", "qvb0", "thvb", "pib", "pb", "rhou", "rhow", "z", "z_zeta",
            "lambda2", "Q1LS", "Q2LS")


def _state(NX=32):
    path = RefTropicalModel.init_path()
    NZ = len(read_sounding(path))
    return sounding_state(path, NX, NZ, 200.0, 200.0, 1.0)


def test_sounding_state_equals_reference_init():
    st = _state()
    m = RefTropicalModel(st.grid, addforcingtime=10.0)
    m.init()
    for name in PROFILES:
        assert np.array_equal(st.prof[name], m.prof(name)), name
    for name in ("th", "qv", "qc", "qr", "u", "w", "zeta", "init_th_forcing"):
        assert np.array_equal(st.fields[name], m.field(name)), name
    assert np.array_equal(st.fields["th"], m.field("thm")) and np.array_equal(st.fields["qv"], m.field("qvm"))
    assert st.scalars["ubarTop"] == m.scalar("ubarTop")[0]


def test_sounding_rows_beyond_the_levels_are_refused():
    path = RefTropicalModel.init_path()
    NZ = len(read_sounding(path))
    with pytest.raises(ValueError):
        sounding_state(path, 16, NZ - 1, 200.0, 200.0, 1.0)


def test_reader_stops_at_the_first_row_that_does_not_parse(tmp_path):
    """`inputFile >> ZZ >> ... >> RHOZ` stops at the first field that is not a
    number; rows after it are not read (src/Init.cpp:312)."""
    f = tmp_path / "snd.txt"
    rows = np.arange(30, dtype=float).reshape(3, 10) + 1.0
    text = "# header\n0 0 0 0 0 0 0 0 0 0\n" + "\n".join(" ".join(repr(float(v)) for v in r) for r in rows)
    f.write_text(text + "\n1 2 3 x 5 6 7 8 9 10\n" + " ".join(["4"] * 10) + "\n")
    got = read_sounding(f)
    assert got.shape == (3, 10) and np.array_equal(got, rows)


def test_restatement_follows_the_reference_steps(port_lib):
    """Five steps, the first three forced (Q1/Q2 every step, the random th
    field of each step while step*dt <= addforcingtime): the C restatement,
    which the GPU parity tests use, fed each step's field by the library's
    host generator, against the reference's own steps."""
    st = _state()
    ref = RefTropicalModel(st.grid, addforcingtime=3.0)
    ref.init()
    port = port_lib.PortModel(st.grid, addforcingtime=3.0)
    port.load(st)
    for _ in range(5):
        ref.one_step()
        port.field("init_th_forcing")[:] = G.random_perturbation_host(st.grid, port.step + 1)
        port.one_step()
        assert np.array_equal(ref.field("init_th_forcing"), port.field("init_th_forcing")) or ref.step > 3
    a, b = ref.dump(), port.dump()
    for f in FIELD_NAMES:
        assert rel_l2(b.fields[f], a.fields[f]) <= 1e-11, (f, rel_l2(b.fields[f], a.fields[f]))
