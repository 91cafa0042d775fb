"""Restart files: the whole model state, AB2 history included, in the
NetCDF classic format, written and read without libnetcdf.

The reference restarts from two NetCDF snapshots and a text sounding
(src/Init.cpp:371-486, LOADFROMPREVIOUSFILE) and does not keep the
Adams-Bashforth tendency history, so its restart is not exact. This file
holds everything the step reads: with it a run continues bit for bit (FP64
contexts; a mixed-precision context stores th and qv as FP32 perturbations,
so its round trip through FP64 can move them by one FP32 ulp).

Layout: the reference's snapshot names and dimensions (src/Output.cpp:49-99:
dims "x" = nx, "z" = nz; th, zeta, u, w, qv, qc, qr as double [x][z];
ubarTop; precip [x]) plus the rest of the state: the future time level
(zetap, thp, qvp, qcp, qrp), RKM, RKH, the seven AB2 tendencies [x][z][ab2]
(dim "ab2" = 2, the reference's [i][k][2] arrays), the 1D profiles [z], the
scalars ubarTopp, dubarTop_advect [ab2] and step, and the grid as global
attributes.

Format (classic NetCDF, big-endian): magic "CDF" + version (1: 32-bit
offsets; 2: 64-bit offsets, used when the file passes 2 GiB), numrecs,
dimension list, global attribute list, variable list (name, dimension ids,
attributes, type, size, offset), then each variable's data padded to 4 bytes.
No record (unlimited) dimension is used.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

from .initial_state import FIELDS_2D, HIST, PROFILES, GridSpec, VVMState

EXTRA_FIELDS = ("init_th_forcing",)          # the random theta forcing field, when the case has one
EXTRA_PROFILES = ("Q1LS", "Q2LS")             # large-scale forcing profiles, when present
NC_DIMENSION, NC_VARIABLE, NC_ATTRIBUTE = 0x0A, 0x0B, 0x0C
NC_CHAR, NC_INT, NC_DOUBLE = 2, 4, 6
_NP = {NC_INT: ">i4", NC_DOUBLE: ">f8"}
_SIZE = {NC_CHAR: 1, NC_INT: 4, NC_DOUBLE: 8}


def _pad4(n: int) -> int:
    return (n + 3) & ~3


def _name(s: str) -> bytes:
    b = s.encode()
    return struct.pack(">i", len(b)) + b + b"\0" * (_pad4(len(b)) - len(b))


def _attr_value(v) -> tuple[int, bytes, int]:
    if isinstance(v, str):
        b = v.encode()
        return NC_CHAR, b + b"\0" * (_pad4(len(b)) - len(b)), len(b)
    if isinstance(v, (int, np.integer)) and not isinstance(v, bool):
        return NC_INT, struct.pack(">i", int(v)), 1
    a = np.atleast_1d(np.asarray(v, dtype=">f8"))
    return NC_DOUBLE, a.tobytes(), a.size


def _attrs(attrs: dict) -> bytes:
    if not attrs:
        return b"\0" * 8
    out = struct.pack(">ii", NC_ATTRIBUTE, len(attrs))
    for k, v in attrs.items():
        t, b, n = _attr_value(v)
        out += _name(k) + struct.pack(">ii", t, n) + b
    return out


def write_cdf(path, dims: dict, variables: dict, gattrs: dict | None = None) -> None:
    """dims: name -> length; variables: name -> (dim names, array); arrays
    of integer kind are stored as int32, the rest as double."""
    dnames = list(dims)
    items = []
    for name, (vd, arr) in variables.items():
        a = np.asarray(arr)
        t = NC_INT if np.issubdtype(a.dtype, np.integer) else NC_DOUBLE
        shape = tuple(dims[d] for d in vd)
        if a.shape != shape:
            raise ValueError(f"{name}: shape {a.shape} != {shape}")
        items.append((name, vd, np.ascontiguousarray(a, dtype=_NP[t]), t))
    total = sum(_pad4(a.nbytes) for *_, a, _ in items)
    version = 1 if total < 2**31 - 4096 else 2
    off_fmt = ">i" if version == 1 else ">q"

    def header(begins):
        h = b"CDF" + bytes([version]) + struct.pack(">i", 0)
        h += struct.pack(">ii", NC_DIMENSION, len(dnames)) if dnames else b"\0" * 8
        for d in dnames:
            h += _name(d) + struct.pack(">i", dims[d])
        h += _attrs(gattrs or {})
        h += struct.pack(">ii", NC_VARIABLE, len(items)) if items else b"\0" * 8
        for (name, vd, a, t), beg in zip(items, begins):
            h += _name(name) + struct.pack(">i", len(vd))
            h += b"".join(struct.pack(">i", dnames.index(d)) for d in vd)
            h += b"\0" * 8 + struct.pack(">ii", t, min(_pad4(a.nbytes), 2**32 - 4)) + struct.pack(off_fmt, beg)
        return h

    hlen = len(header([0] * len(items)))
    begins, pos = [], hlen
    for *_, a, _ in items:
        begins.append(pos)
        pos += _pad4(a.nbytes)
    with open(path, "wb") as f:
        f.write(header(begins))
        for *_, a, _ in items:
            f.write(a.tobytes())
            f.write(b"\0" * (_pad4(a.nbytes) - a.nbytes))


def read_cdf(path) -> tuple[dict, dict, dict]:
    """(dims, variables name -> array, global attributes) of a classic
    NetCDF file without record variables."""
    buf = Path(path).read_bytes()
    if buf[:3] != b"CDF" or buf[3] not in (1, 2):
        raise ValueError("not a classic NetCDF file")
    version = buf[3]
    pos = 8

    def i4():
        nonlocal pos
        v = struct.unpack_from(">i", buf, pos)[0]
        pos += 4
        return v

    def name():
        nonlocal pos
        n = i4()
        s = buf[pos:pos + n].decode()
        pos += _pad4(n)
        return s

    def attrs():
        nonlocal pos
        tag, n = i4(), i4()
        out = {}
        for _ in range(n if tag == NC_ATTRIBUTE else 0):
            k, t, m = name(), i4(), i4()
            if t == NC_CHAR:
                out[k] = buf[pos:pos + m].decode()
                pos += _pad4(m)
            else:
                a = np.frombuffer(buf, dtype=_NP[t], count=m, offset=pos).astype(np.float64 if t == NC_DOUBLE else np.int64)
                pos += _pad4(m * _SIZE[t])
                out[k] = a[0] if m == 1 else a
        return out

    tag, n = i4(), i4()
    dims = {}
    for _ in range(n if tag == NC_DIMENSION else 0):
        d = name()
        dims[d] = i4()
    dl = list(dims)
    gattrs = attrs()
    tag, n = i4(), i4()
    variables = {}
    for _ in range(n if tag == NC_VARIABLE else 0):
        v = name()
        vd = [dl[i4()] for _ in range(i4())]
        attrs()
        t = i4()
        i4()   # vsize
        if version == 1:
            beg = i4()
        else:
            beg = struct.unpack_from(">q", buf, pos)[0]
            pos += 8
        shape = tuple(dims[d] for d in vd)
        cnt = int(np.prod(shape)) if shape else 1
        a = np.frombuffer(buf, dtype=_NP[t], count=cnt, offset=beg).reshape(shape)
        variables[v] = a.astype(np.float64 if t == NC_DOUBLE else np.int64)
    return dims, variables, gattrs


def write_restart(path, st: VVMState, **attrs) -> None:
    """The whole state of `st` (as downloaded from a context) to `path`."""
    g = st.grid
    dims = {"x": g.nx, "z": g.nz, "ab2": 2}
    v = {n: (("x", "z"), st.fields[n]) for n in FIELDS_2D + EXTRA_FIELDS if n in st.fields}
    v.update({n: (("x", "z", "ab2"), st.hist[n]) for n in HIST})
    v.update({n: (("z",), st.prof[n]) for n in PROFILES + EXTRA_PROFILES if n in st.prof})
    v["precip"] = (("x",), st.precip if st.precip is not None else np.zeros(g.nx))
    v["ubarTop"] = ((), np.float64(st.scalars["ubarTop"]))
    v["ubarTopp"] = ((), np.float64(st.scalars["ubarTopp"]))
    v["dubarTop_advect"] = (("ab2",), np.asarray(st.scalars["dubarTop_advect"], dtype=np.float64))
    v["step"] = ((), np.int32(st.scalars["step"]))
    ga = {"title": "VVM state (restart)", "NX": g.NX, "NZ": g.NZ, "dx": float(g.dx), "dz": float(g.dz),
          "dt": float(g.dt), "case": int(g.case), "moisture_nudge_time": float(g.moisture_nudge_time)}
    ga.update(attrs)
    write_cdf(path, dims, v, ga)


def read_restart(path) -> VVMState:
    dims, v, ga = read_cdf(path)
    g = GridSpec(int(ga["NX"]), int(ga["NZ"]), float(ga["dx"]), float(ga["dz"]), float(ga["dt"]),
                 int(ga["case"]), float(ga["moisture_nudge_time"]))
    st = VVMState(g)
    st.fields = {n: np.array(v[n]) for n in FIELDS_2D + EXTRA_FIELDS if n in v}
    st.hist = {n: np.array(v[n]) for n in HIST}
    st.prof = {n: np.array(v[n]) for n in PROFILES + EXTRA_PROFILES if n in v}
    st.precip = np.array(v["precip"])
    st.scalars = dict(ubarTop=float(v["ubarTop"]), ubarTopp=float(v["ubarTopp"]),
                      dubarTop_advect=np.array(v["dubarTop_advect"]), step=int(v["step"]))
    return st
