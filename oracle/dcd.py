"""Reader of the DCD files the output writes (test infrastructure only).

Restates the layout DcdWriter writes (src/IO/DcdWriter.h writeHeaderImpl,
writeStepFromVector3, updateHeader): Fortran records of little-endian int32
markers; an 84-byte header record "CORD", NFILE, NPRIV, NSAVC, NSTEP, five
zeros, DELTA (float32), the unit-cell flag, eight zeros, the CHARMM version;
a title record (count, 80-character lines); the atom count record; per frame
an optional 48-byte unit cell record (six float64) and X, Y, Z records of
float32.
"""
from __future__ import annotations

import struct

import numpy as np


def _record(buf, off):
    (m,) = struct.unpack_from("<i", buf, off)
    body = buf[off + 4: off + 4 + m]
    (m2,) = struct.unpack_from("<i", buf, off + 4 + m)
    if m2 != m:
        raise ValueError(f"record markers differ at {off}: {m} vs {m2}")
    return body, off + 8 + m


def read_dcd(buf: bytes) -> dict:
    hdr, off = _record(buf, 0)
    if len(hdr) != 84 or hdr[:4] != b"CORD":
        raise ValueError("not a DCD header")
    ints = struct.unpack_from("<9i", hdr, 4)
    nfile, npriv, nsavc, nstep = ints[0], ints[1], ints[2], ints[3]
    (delta,) = struct.unpack_from("<f", hdr, 40)
    (unitcell,) = struct.unpack_from("<i", hdr, 44)
    (version,) = struct.unpack_from("<i", hdr, 80)
    titles_rec, off = _record(buf, off)
    (ntitle,) = struct.unpack_from("<i", titles_rec, 0)
    titles = [titles_rec[4 + 80 * k: 4 + 80 * (k + 1)].decode() for k in range(ntitle)]
    natom_rec, off = _record(buf, off)
    (natoms,) = struct.unpack_from("<i", natom_rec, 0)
    frames, cells = [], []
    while off < len(buf):
        if unitcell:
            cell, off = _record(buf, off)
            cells.append(np.frombuffer(cell, "<f8").copy())
        xyz = []
        for _ in range(3):
            rec, off = _record(buf, off)
            xyz.append(np.frombuffer(rec, "<f4").copy())
        frames.append(np.stack(xyz, axis=1))
    return dict(nfile=nfile, npriv=npriv, nsavc=nsavc, nstep=nstep, delta=np.float32(delta),
                unitcell=unitcell, version=version, titles=titles, natoms=natoms,
                frames=np.array(frames), cells=np.array(cells))


def title_spans(buf: bytes):
    """Byte ranges of the two 80-character title lines (file name and date)."""
    start = 4 + 84 + 4 + 4 + 4  # header record, title record marker, title count
    return [(start, start + 80), (start + 80, start + 160)]
