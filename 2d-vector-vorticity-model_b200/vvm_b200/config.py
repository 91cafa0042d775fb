"""Runtime configuration, mirroring the reference's reader and constructor.

``vvm_read_config`` follows src/ReadConfig.cpp:3-48: ``key=value`` lines,
everything after ``#`` ignored, surrounding blanks and tabs stripped, later
keys override earlier ones, lines without ``=`` skipped. ``config_from_file``
builds a ``GridSpec`` from the keys src/main.cpp:48-66 reads.
"""
from __future__ import annotations

from .initial_state import GridSpec


def _strip(s: str) -> str:
    return s.strip(" \t")


def vvm_read_config(path: str) -> dict:
    cfg: dict = {}
    try:
        fh = open(path, "r")
    except OSError:
        return cfg  # std::ifstream on a missing file yields an empty map
    with fh:
        for raw in fh:
            line = raw.rstrip("\n")
            pos = line.find("#")
            if pos != -1:
                line = line[:pos]
            line = _strip(line)
            if not line:
                continue
            if "=" not in line:
                continue
            key, value = line.split("=", 1)
            cfg[_strip(key)] = _strip(value)
    return cfg


def config_from_file(path: str) -> GridSpec:
    """GridSpec from VVM_XRANGE/ZRANGE/DX/DZ/DT/CASE/MOISTURE_NUDGE_TIME
    (src/main.cpp:50-58; nx = XRANGE/dx + 2, src/Declare.hpp:33,82)."""
    c = vvm_read_config(path)
    dx = float(c["VVM_DX"])
    dz = float(c["VVM_DZ"])
    NX = int(int(c["VVM_XRANGE"]) / dx)
    NZ = int(int(c["VVM_ZRANGE"]) / dz)
    return GridSpec(NX=NX, NZ=NZ, dx=dx, dz=dz, dt=float(c["VVM_DT"]),
                    case=int(c.get("VVM_CASE", "1")),
                    moisture_nudge_time=float(c.get("VVM_MOISTURE_NUDGE_TIME", "0")))
