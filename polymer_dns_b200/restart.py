"""Restart files of the channel run, byte-compatible with the reference's.

The reference writes them at the end of every step with ``mod(it, iprnfrq) == 0`` or
``it == nsteps`` (main_dns.f90:775-794) as Fortran unformatted sequential files and reads them
back in ``initial`` when ``irstrt >= 1`` (main_dns.f90:1742-1916):

  restart    record 1: v, fn, fnm1, omy, gn, gnm1 (complex(8) (nyp,nz,nxh) each),
                       u0, h1n, h1nm1, w0, h3n, h3nm1 (real(8) (nyp) each)
             record 2: fxintg, fyintg, fzintg (real(8) (nyp,mz,mx) each)
  c-restart  (scalar + polymer modules, written once it >= src_start)
             record 1: scalar, c11, c12, c13, c21, c22, c23, c31, c32, c33
             record 2: scn, c11n, c12n, c13n, c22n, c23n, c33n
             record 3: scnm1, c11nm1, c12nm1, c13nm1, c22nm1, c23nm1, c33nm1
             record 4: str11n, str12n, str13n, str22n, str23n, str33n
             record 5: str11nm1, str12nm1, str13nm1, str22nm1, str23nm1, str33nm1

Record framing (the reference is built with ``-r8``, so every real is 8 bytes): each record is
one or more subrecords, each framed by a leading and a trailing little-endian int32 holding its
payload length; a payload holds at most 2**31 - 9 bytes.  Longer records are split, with the
sign bit as the continuation flag: a negative leading marker means another subrecord follows,
a negative trailing marker means one precedes.  This is the variable-length record layout of
both Intel Fortran and gfortran with 4-byte markers.

``irstrt = 2`` reads a file written at half the streamwise resolution (nxh/2, mx/2; the other
sizes equal) and embeds it in zeroed full-size arrays (main_dns.f90:1761-1808).

Reading is strict: a record whose length differs from what the grid implies raises ValueError
(the Fortran read of a shorter record fails; of a longer one it would silently take a prefix,
which for a restart file only happens with a grid mismatch).
"""
import os
import struct

import numpy as np

from . import abi

MAX_SUBRECORD = 2**31 - 9

RESTART_RECORDS = (
    ("V", "FN", "FNM1", "OMY", "GN", "GNM1", "U0", "H1N", "H1NM1", "W0", "H3N", "H3NM1"),
    ("FXINTG", "FYINTG", "FZINTG"),
)
C_RESTART_RECORDS = (
    ("SCALAR", "C11", "C12", "C13", "C21", "C22", "C23", "C31", "C32", "C33"),
    ("SCN", "C11N", "C12N", "C13N", "C22N", "C23N", "C33N"),
    ("SCNM1", "C11NM1", "C12NM1", "C13NM1", "C22NM1", "C23NM1", "C33NM1"),
    ("STR11N", "STR12N", "STR13N", "STR22N", "STR23N", "STR33N"),
    ("STR11NM1", "STR12NM1", "STR13NM1", "STR22NM1", "STR23NM1", "STR33NM1"),
)


# ---------------------------------------------------------------------------
# record framing
# ---------------------------------------------------------------------------
def write_record(fh, payload, max_sub=MAX_SUBRECORD):
    """Write one record (bytes-like) with 4-byte markers, split into subrecords past max_sub."""
    mv = memoryview(payload).cast("B")
    n = len(mv)
    off = 0
    first = True
    while True:
        m = min(n - off, max_sub)
        last = off + m == n
        fh.write(struct.pack("<i", m if last else -m))
        fh.write(mv[off:off + m])
        fh.write(struct.pack("<i", m if first else -m))
        off += m
        first = False
        if last:
            return


def read_record(fh):
    """Read one record; returns its payload (bytes).  Raises ValueError on broken framing."""
    parts = []
    first = True
    while True:
        head = fh.read(4)
        if len(head) != 4:
            raise ValueError("end of file inside a record" if parts else "end of file: no record left")
        lead = struct.unpack("<i", head)[0]
        m = abs(lead)
        data = fh.read(m)
        tail = fh.read(4)
        if len(data) != m or len(tail) != 4:
            raise ValueError("truncated subrecord (%d payload bytes expected)" % m)
        trail = struct.unpack("<i", tail)[0]
        if abs(trail) != m or (trail < 0) == first:
            raise ValueError("record markers disagree (%d ... %d)" % (lead, trail))
        parts.append(data)
        first = False
        if lead >= 0:
            return b"".join(parts)


# ---------------------------------------------------------------------------
# field lists <-> records
# ---------------------------------------------------------------------------
def _layout(name, nx, ny, nz):
    fid = abi.FIELD[name]
    _, dt = abi.field_kind(fid)
    return np.dtype(dt).newbyteorder("<"), abi.field_shape(fid, nx, ny, nz)


def _pack(fields, names, nx, ny, nz):
    chunks = []
    for name in names:
        dt, shape = _layout(name, nx, ny, nz)
        a = np.asarray(fields[name])
        if a.shape != shape:
            raise ValueError("%s has shape %s, the grid needs %s" % (name, a.shape, shape))
        chunks.append(np.asarray(a, dtype=dt).ravel(order="F").tobytes())
    return b"".join(chunks)


def _unpack(payload, names, nx, ny, nz):
    sizes = []
    for name in names:
        dt, shape = _layout(name, nx, ny, nz)
        sizes.append((name, dt, shape, dt.itemsize * int(np.prod(shape))))
    want = sum(s[3] for s in sizes)
    if len(payload) != want:
        raise ValueError("record holds %d bytes, %s on this grid need %d" % (len(payload), "/".join(names), want))
    out, off = {}, 0
    for name, dt, shape, nb in sizes:
        out[name] = np.frombuffer(payload, dtype=dt, count=nb // dt.itemsize, offset=off).reshape(shape, order="F")
        out[name] = out[name].astype(dt.newbyteorder("="), copy=True)
        off += nb
    return out


def write_file(path, fields, records, nx, ny, nz, max_sub=MAX_SUBRECORD):
    """Write `records` (tuples of field names) of `fields` to `path`, replacing it."""
    tmp = path + ".tmp"
    with open(tmp, "wb") as fh:
        for names in records:
            write_record(fh, _pack(fields, names, nx, ny, nz), max_sub)
    os.replace(tmp, path)


def read_file(path, records, nx, ny, nz):
    """Read `records` from `path`; returns {field name: array in the reference layout}."""
    out = {}
    with open(path, "rb") as fh:
        for names in records:
            out.update(_unpack(read_record(fh), names, nx, ny, nz))
    return out


def write_restart(path, fields, nx, ny, nz, max_sub=MAX_SUBRECORD):
    """outputs/last-restart (main_dns.f90:777-779)."""
    write_file(path, fields, RESTART_RECORDS, nx, ny, nz, max_sub)


def write_c_restart(path, fields, nx, ny, nz, max_sub=MAX_SUBRECORD):
    """outputs/c-last-restart (main_dns.f90:784-789)."""
    write_file(path, fields, C_RESTART_RECORDS, nx, ny, nz, max_sub)


def read_restart(path, nx, ny, nz, low_res=False):
    """setup/restart (main_dns.f90:1743-1747); low_res: the irstrt = 2 form written at nx/2,
    embedded in zeroed full-size arrays (main_dns.f90:1761-1808)."""
    if not low_res:
        return read_file(path, RESTART_RECORDS, nx, ny, nz)
    if nx % 4:
        raise ValueError("a half-resolution restart needs nx divisible by 4 (nx = %d)" % nx)
    lr = read_file(path, RESTART_RECORDS, nx // 2, ny, nz)
    out = {}
    for names in RESTART_RECORDS:
        for name in names:
            dt, shape = _layout(name, nx, ny, nz)
            full = np.zeros(shape, dtype=dt.newbyteorder("="), order="F")
            src = lr[name]
            full[tuple(slice(0, s) for s in src.shape)] = src
            out[name] = full
    return out


def read_c_restart(path, nx, ny, nz):
    """setup/c-restart (main_dns.f90:1910-1916)."""
    return read_file(path, C_RESTART_RECORDS, nx, ny, nz)


def restart_due(it, iprnfrq, nsteps):
    """The reference's write condition after step `it` (main_dns.f90:776)."""
    return it % iprnfrq == 0 or it == nsteps


def c_restart_due(params, it):
    """c-last-restart is written with the scalar and polymer modules once it >= src_start
    (main_dns.f90:781-783)."""
    return bool(params.scalar_on and params.polymer_on and it >= params.src_start)


# ---------------------------------------------------------------------------
# contexts: `fetch(name)` returns a field, `store(name, array)` places one
# ---------------------------------------------------------------------------
def save(fetch, params, it, path, c_path=None):
    """Write the restart file(s) of the state after step `it`; c-restart only when due."""
    nx, ny, nz = params.nx, params.ny, params.nz
    write_restart(path, {n: fetch(n) for rec in RESTART_RECORDS for n in rec}, nx, ny, nz)
    if c_path is not None and c_restart_due(params, it):
        write_c_restart(c_path, {n: fetch(n) for rec in C_RESTART_RECORDS for n in rec}, nx, ny, nz)


def load(store, params, path, c_path=None):
    """Place the restart file's fields (and c-restart's, with scalar + polymer and crstrt != 0)
    before `initial` runs with irstrt >= 1."""
    if params.irstrt < 1:
        raise ValueError("loading a restart file needs irstrt >= 1 (irstrt = %d)" % params.irstrt)
    nx, ny, nz = params.nx, params.ny, params.nz
    for name, a in read_restart(path, nx, ny, nz, low_res=params.irstrt == 2).items():
        store(name, a)
    if params.scalar_on and params.polymer_on and params.crstrt != 0:
        if c_path is None:
            raise ValueError("crstrt != 0 with scalar + polymer needs the c-restart file")
        for name, a in read_c_restart(c_path, nx, ny, nz).items():
            store(name, a)
