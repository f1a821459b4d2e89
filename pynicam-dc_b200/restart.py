"""Restart files in the reference's fio format, read and written from the
device state.

The format is the one nhm/share/mod_fio.py reads and writes for
input/output_io_mode "ADVANCED": a big-endian C stream of

  file header : header(64) note(256), six uint32 (fmode, endian, topo,
                glevel, rlevel, num_of_rgn), num_of_rgn uint32 region ids,
                uint32 number of items
  per item    : varname(16) description(64) unit(16) layername(16) note(256),
                uint64 datasize, uint32 datatype, num_layer, step, uint64
                time_start, time_end, then datasize bytes of data

with each variable's data a (region, k, ij) stream.  That is the device field
layout, so the payloads move between the file and the device with a byte swap
on the device (``nc_restart_pack`` / ``nc_restart_unpack``) and no host
transposition; this module only writes and parses the headers.
"""
from __future__ import annotations

import struct

import numpy as np

HEADER, NOTE, NAME, DESC, UNIT, LAYER = 64, 256, 16, 64, 16, 16
F8 = 1   # datatype code of big-endian float64 (mod_fio.py DTYPE_MAP)


def _field(s: str, n: int) -> bytes:
    raw = s.encode()[:n]
    return raw + b"\x00" * (n - len(raw))


def _text(b: bytes) -> str:
    return b.decode(errors="ignore").strip("\x00").strip()


def file_header(header: str, note: str, fmode: int, endian: int, topo: int, glevel: int, rlevel: int,
                rgnid) -> bytes:
    """the file header up to (not including) the item count"""
    rgnid = [int(r) for r in rgnid]
    return (_field(header, HEADER) + _field(note, NOTE)
            + struct.pack(">6I", fmode, endian, topo, glevel, rlevel, len(rgnid))
            + struct.pack(f">{len(rgnid)}I", *rgnid))


def item_header(varname: str, description: str, unit: str, layername: str, datasize: int, datatype: int,
                num_layer: int, step: int, time_start: int, time_end: int, note: str = "") -> bytes:
    return (_field(varname, NAME) + _field(description, DESC) + _field(unit, UNIT) + _field(layername, LAYER)
            + _field(note, NOTE) + struct.pack(">Q3I", datasize, datatype, num_layer, step)
            + struct.pack(">QQ", time_start, time_end))


def parse(path: str):
    """(meta, items): the file header fields and, per item, its header fields
    and the byte offset of its data"""
    with open(path, "rb") as f:
        meta = dict(header=_text(f.read(HEADER)), note=_text(f.read(NOTE)))
        (meta["fmode"], meta["endian"], meta["topo"], meta["glevel"], meta["rlevel"],
         nrgn) = struct.unpack(">6I", f.read(24))
        meta["rgnid"] = list(struct.unpack(f">{nrgn}I", f.read(4 * nrgn)))
        (ndata,) = struct.unpack(">I", f.read(4))
        items = []
        for _ in range(ndata):
            it = dict(varname=_text(f.read(NAME)), description=_text(f.read(DESC)), unit=_text(f.read(UNIT)),
                      layername=_text(f.read(LAYER)))
            f.read(NOTE)
            it["datasize"], it["datatype"], it["num_layer"], it["step"] = struct.unpack(">Q3I", f.read(20))
            it["time_start"], it["time_end"] = struct.unpack(">QQ", f.read(16))
            it["offset"] = f.tell()
            f.seek(it["datasize"], 1)
            items.append(it)
    return meta, items


def write(core, path: str, items, layername: str, rgnid, glevel: int, rlevel: int, ctime: int = 0):
    """Prgvar.restart_output (nhm/share/mod_prgvar.py:182-216), "ADVANCED",
    prognostic items: ``items`` = [(varname, description, unit, device var)],
    the data of each read from the device state."""
    G, K, L = core.shape[0], core.shape[2], core.shape[3]
    n = G * G * K * L
    buf = np.empty(n, np.uint64)
    with open(path, "wb") as f:
        f.write(file_header("INITIAL/RESTART_data_of_prognostic_variables", "", 0, 2, 0, glevel, rlevel, rgnid))
        f.write(struct.pack(">I", len(items)))
        for name, desc, unit, var in items:
            f.write(item_header(name, desc, unit, layername, 8 * n, F8, K, 1, int(ctime), int(ctime)))
            core.restart_pack(var, buf)
            buf.tofile(f)


def read(core, path: str, names, pole_src, allow_missingq: bool = False):
    """Prgvar.restart_input's prognostic read (nhm/share/mod_prgvar.py:266-306)
    of a fio file into the device state: ``names`` are the variable names of
    the device variables in order (RHOG .. RHOGE, then rhog<tracer>); a
    missing tracer is zero with ``allow_missingq``, anything else missing is
    an error; then COMM_var with the pole-centre sources ``pole_src``."""
    G, K, L = core.shape[0], core.shape[2], core.shape[3]
    n = G * G * K * L
    meta, items = parse(path)
    if meta["rgnid"] and len(meta["rgnid"]) != L:
        raise ValueError(f"{path}: {len(meta['rgnid'])} regions in the file, {L} on the device")
    by_name = {it["varname"]: it for it in items}
    for var, name in enumerate(names):
        it = by_name.get(name)
        if it is None:
            if var >= 6 and allow_missingq:
                core.restart_unpack(var, np.zeros(n, np.uint64))
                continue
            raise KeyError(f"{path}: variable {name!r} not in the restart file")
        if it["datatype"] != F8:
            raise NotImplementedError(f"{path}: {name!r} has datatype {it['datatype']}; the device path reads "
                                      "big-endian float64 payloads")
        if it["datasize"] != 8 * n:
            raise ValueError(f"{path}: {name!r} holds {it['datasize']} bytes, expected {8 * n}")
        core.restart_unpack(var, np.fromfile(path, dtype=np.uint64, count=n, offset=it["offset"]))
    core.restart_finish(pole_src)
    return meta, items
