"""Restart files: record framing, byte layout, and continuation through the oracle.

The reference writes outputs/last-restart (and c-last-restart with scalar + polymer) as Fortran
unformatted sequential files (main_dns.f90:775-794) and reads setup/restart back in `initial`
with irstrt >= 1 (main_dns.f90:1742-1916).  A run of 2n steps and a run of n steps, a restart
file, a fresh context with irstrt = 1 and n more steps must end in the same state: the restart
records hold the whole time-stepping state, and `initial` recomputes nothing from them.
"""
import io
import struct

import numpy as np
import pytest

from oracle import pyoracle
from polymer_dns_b200 import abi, restart
from tests import kmm_cases as kc


def _markers(buf):
    """[(leading marker, payload length, trailing marker)] of a record stream."""
    out, off = [], 0
    while off < len(buf):
        lead = struct.unpack_from("<i", buf, off)[0]
        m = abs(lead)
        trail = struct.unpack_from("<i", buf, off + 4 + m)[0]
        out.append((lead, m, trail))
        off += 8 + m
    return out


def test_record_framing_single_and_split():
    payload = bytes(range(20))
    fh = io.BytesIO()
    restart.write_record(fh, payload)
    assert _markers(fh.getvalue()) == [(20, 20, 20)]
    # 20 bytes with at most 8 per subrecord: 8 + 8 + 4, sign bit = continuation flag
    fh = io.BytesIO()
    restart.write_record(fh, payload, max_sub=8)
    raw = fh.getvalue()
    assert _markers(raw) == [(-8, 8, 8), (-8, 8, -8), (4, 4, -4)]
    assert raw[4:12] == payload[:8] and raw[20:28] == payload[8:16] and raw[36:40] == payload[16:]
    fh.seek(0)
    assert restart.read_record(fh) == payload
    # an exact multiple of the subrecord size and an empty record
    for data, max_sub in [(b"abcdefgh" * 2, 8), (b"", 8)]:
        fh = io.BytesIO()
        restart.write_record(fh, data, max_sub=max_sub)
        restart.write_record(fh, b"next")
        fh.seek(0)
        assert restart.read_record(fh) == data
        assert restart.read_record(fh) == b"next"


def test_record_framing_rejects_broken_files():
    fh = io.BytesIO()
    restart.write_record(fh, b"0123456789", max_sub=4)
    raw = fh.getvalue()
    with pytest.raises(ValueError):
        restart.read_record(io.BytesIO(raw[:-2]))          # truncated
    assert _markers(raw) == [(-4, 4, 4), (-4, 4, -4), (2, 2, -2)]
    bad = bytearray(raw)
    struct.pack_into("<i", bad, 20, 4)                      # second subrecord's trailing marker: -4 -> +4
    with pytest.raises(ValueError):
        restart.read_record(io.BytesIO(bytes(bad)))
    with pytest.raises(ValueError):
        restart.read_record(io.BytesIO(b""))


def _patterned_fields(p, names, seed):
    rng = np.random.default_rng(seed)
    out = {}
    for rec in names:
        for n in rec:
            fid = abi.FIELD[n]
            kind, dt = abi.field_kind(fid)
            shape = abi.field_shape(fid, p.nx, p.ny, p.nz)
            a = rng.standard_normal(shape)
            if np.dtype(dt).kind == "c":
                a = a + 1j * rng.standard_normal(shape)
            out[n] = np.asfortranarray(a.astype(dt))
    return out


def test_restart_byte_layout(tmp_path):
    """Two records; record 1 is v|fn|fnm1|omy|gn|gnm1 (complex(8), Fortran order) followed by
    u0|h1n|h1nm1|w0|h3n|h3nm1; record 2 is fxintg|fyintg|fzintg on the 3/2 grid."""
    p = kc.cfg_small(8, 8, 8)
    nyp, nz, nxh, mz, mx = 9, 8, 4, 12, 12
    f = _patterned_fields(p, restart.RESTART_RECORDS, 1)
    path = str(tmp_path / "last-restart")
    restart.write_restart(path, f, p.nx, p.ny, p.nz)
    raw = open(path, "rb").read()
    nspec = nyp * nz * nxh
    r1 = 6 * nspec * 16 + 6 * nyp * 8
    r2 = 3 * nyp * mz * mx * 8
    assert _markers(raw) == [(r1, r1, r1), (r2, r2, r2)]
    assert len(raw) == r1 + r2 + 16
    # v(2,3,2) (1-based) sits at column-major offset 1 + 2*nyp + 1*nyp*nz
    k = 1 + 2 * nyp + 1 * nyp * nz
    re_, im_ = struct.unpack_from("<dd", raw, 4 + 16 * k)
    assert (re_, im_) == (f["V"][1, 2, 1].real, f["V"][1, 2, 1].imag)
    # omy is the fourth spectral field; u0 follows the six spectral fields
    re_, _ = struct.unpack_from("<dd", raw, 4 + 16 * (3 * nspec))
    assert re_ == f["OMY"][0, 0, 0].real
    assert struct.unpack_from("<d", raw, 4 + 6 * nspec * 16 + 8 * 3)[0] == f["U0"][3]
    assert struct.unpack_from("<d", raw, 4 + 6 * nspec * 16 + 8 * (3 * nyp))[0] == f["W0"][0]
    # fyintg(1,1,2) in record 2
    off2 = 4 + r1 + 4 + 4
    assert struct.unpack_from("<d", raw, off2 + 8 * (nyp * mz * mx + nyp * mz))[0] == f["FYINTG"][0, 0, 1]
    back = restart.read_restart(path, p.nx, p.ny, p.nz)
    for n in f:
        assert np.array_equal(back[n], f[n]), n


def test_restart_rejects_grid_mismatch(tmp_path):
    p = kc.cfg_small(8, 8, 8)
    f = _patterned_fields(p, restart.RESTART_RECORDS, 2)
    path = str(tmp_path / "r")
    restart.write_restart(path, f, 8, 8, 8)
    with pytest.raises(ValueError):
        restart.read_restart(path, 16, 8, 8)
    with pytest.raises(ValueError):
        restart.write_restart(path, f, 8, 16, 8)


def test_low_resolution_restart_embeds(tmp_path):
    """irstrt = 2: a file at nx/2 lands in the first nxh/2 (spectral) and mx/2 (physical)
    planes of zeroed arrays (main_dns.f90:1761-1808)."""
    lo = kc.cfg_small(8, 8, 8)
    f = _patterned_fields(lo, restart.RESTART_RECORDS, 3)
    path = str(tmp_path / "lr")
    restart.write_restart(path, f, 8, 8, 8)
    full = restart.read_restart(path, 16, 8, 8, low_res=True)
    assert full["V"].shape == (9, 8, 8)
    assert np.array_equal(full["V"][:, :, :4], f["V"]) and not full["V"][:, :, 4:].any()
    assert full["FXINTG"].shape == (9, 12, 24)
    assert np.array_equal(full["FXINTG"][:, :, :12], f["FXINTG"]) and not full["FXINTG"][:, :, 12:].any()
    assert np.array_equal(full["H3NM1"], f["H3NM1"])


def test_restart_due_matches_reference_condition():
    assert [it for it in range(1, 11) if restart.restart_due(it, 4, 10)] == [4, 8, 10]
    p = kc.cfg_small(8, 8, 8, scalar_on=1, polymer_on=1, src_start=3)
    assert [restart.c_restart_due(p, it) for it in (2, 3)] == [False, True]
    assert not restart.c_restart_due(kc.cfg_small(8, 8, 8, scalar_on=1, src_start=0), 5)


STATE = ("V", "OMY", "FN", "FNM1", "GN", "GNM1", "U0", "W0", "H1N", "H1NM1", "H3N", "H3NM1")


def _oracle_run(p, fields, n, scalar=None):
    o = pyoracle.Oracle(p)
    kc.load_initial(o, p, fields, scalar)
    assert o.initial() == 0
    for _ in range(n):
        assert o.step() == 0
    return o


@pytest.mark.parametrize("grid", [(16, 16, 16), (24, 32, 16)])
def test_oracle_continuation_is_exact(tmp_path, grid):
    """2n steps == n steps + restart file + irstrt = 1 + n steps, bit for bit (fluid only)."""
    n = 3
    p = kc.cfg_small(*grid)
    fields = kc.initial_fields(p)
    whole = _oracle_run(p, fields, 2 * n)
    first = _oracle_run(p, fields, n)
    path = str(tmp_path / "last-restart")
    restart.save(first.get, p, n, path)
    q = kc.cfg_small(*grid, irstrt=1)
    second = pyoracle.Oracle(q)
    restart.load(second.set, q, path)
    assert second.initial() == 0
    assert second.stats().it == 0
    for _ in range(n):
        assert second.step() == 0
    for f in STATE:
        assert np.array_equal(second.get(f), whole.get(f)), f


def test_oracle_continuation_scalar_polymer_c_restart(tmp_path):
    """Scalar + polymer with crstrt = 1: c-restart carries the conformation tensor, the scalar
    and their histories, and the continuation is exact as well."""
    n = 2
    kw = dict(scalar_on=1, polymer_on=1, src_start=0, tpoly=20.0, alpha_poly=0.0, diffpoly=1000.0,
              c11z=1.0, c22z=1.0, c33z=1.0, zlmax=30.0, qbeta=0.9, diff=1.0)
    p = kc.cfg_small(16, 16, 16, **kw)
    fields = kc.initial_fields(p)
    scl = np.asfortranarray(np.random.default_rng(4).standard_normal((17, 16, 16)) * 0.1)
    whole = _oracle_run(p, fields, 2 * n, scl)
    first = _oracle_run(p, fields, n, scl)
    path, cpath = str(tmp_path / "last-restart"), str(tmp_path / "c-last-restart")
    restart.save(first.get, p, n, path, cpath)
    q = kc.cfg_small(16, 16, 16, irstrt=1, crstrt=1, **kw)
    second = pyoracle.Oracle(q)
    restart.load(second.set, q, path, cpath)
    assert second.initial() == 0
    for _ in range(n):
        assert second.step() == 0
    for f in STATE + ("SCALAR", "SCN", "SCNM1", "C11", "C12", "C22", "C33", "C11N", "STR12NM1"):
        assert np.array_equal(second.get(f), whole.get(f)), f


def test_oracle_restart_scalar_reinitialised_without_norm(tmp_path):
    """Scalar without polymer: a restart takes the scalar from setscl again (main_dns.f90:
    1810-1815) and, unlike irstrt = 0, does not normalise it."""
    p = kc.cfg_small(16, 16, 16, scalar_on=1)
    fields = kc.initial_fields(p)
    scl = np.asfortranarray(np.random.default_rng(5).standard_normal((17, 16, 16)))
    first = _oracle_run(p, fields, 1, scl)
    path = str(tmp_path / "r")
    restart.save(first.get, p, 1, path)
    q = kc.cfg_small(16, 16, 16, scalar_on=1, irstrt=1)
    o = pyoracle.Oracle(q)
    restart.load(o.set, q, path)
    o.set("INITSCL", scl)
    assert o.initial() == 0
    ref = pyoracle.Oracle(p)
    ref.set("INITSCL", scl)
    ref.call("xyzfft", "SCALAR", "INITSCL")
    assert np.array_equal(o.get("SCALAR"), ref.get("SCALAR"))
    assert not o.get("CSOURCE").any()
    assert np.array_equal(o.get("V"), first.get("V"))
