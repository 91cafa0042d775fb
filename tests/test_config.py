"""The key=value reader mirrors src/ReadConfig.cpp:3-48."""
from vvm_b200.config import config_from_file, vvm_read_config


def test_reader_semantics(tmp_path):
    p = tmp_path / "vvm_config.txt"
    p.write_text("VVM_XRANGE=25600          # Domain for x [m]\n"
                 "  VVM_DX \t= 200\t\n"
                 "# full-line comment\n"
                 "\n"
                 "NOEQUALS\n"
                 "VVM_DZ=200\n"
                 "VVM_DZ=250   # later keys override\n"
                 "VVM_ZRANGE=12800\nVVM_DT=1\nVVM_CASE=2\nVVM_MOISTURE_NUDGE_TIME=0\n")
    c = vvm_read_config(str(p))
    assert c["VVM_XRANGE"] == "25600"
    assert c["VVM_DX"] == "200"
    assert c["VVM_DZ"] == "250"
    assert "NOEQUALS" not in c
    g = config_from_file(str(p))
    assert (g.NX, g.NZ, g.dx, g.dz, g.dt, g.case) == (128, 51, 200.0, 250.0, 1.0, 2)


def test_missing_file_gives_empty_map(tmp_path):
    assert vvm_read_config(str(tmp_path / "nope.txt")) == {}
