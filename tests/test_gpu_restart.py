"""Restart on the GPU: continuation through the reference's restart file, and the file read by
the GPU path against the oracle.

- 2n fused steps == n steps, restart file, a fresh context with irstrt = 1, n steps: bit for
  bit (FP64 and mixed precision; the step recomputes everything from the restart records).
- Scalar + polymer (routine path) with crstrt = 1 and the c-restart file: bit for bit.
- A restart file written by the oracle, continued on the GPU and on the oracle: within the
  whole-run parity bar of the FP64 drop-in (1e-10 relative).
"""
import numpy as np
import pytest

from polymer_dns_b200 import restart
from tests import kmm_cases as kc

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-10
STATE = ("V", "OMY", "FN", "FNM1", "GN", "GNM1", "U0", "W0", "H1N", "H1NM1", "H3N", "H3NM1")


@pytest.fixture(scope="module")
def rt():
    from polymer_dns_b200 import build, runtime
    build.build()
    return runtime


def _gpu_run(rt, p, fields, n, scalar=None):
    g = rt.KmmContext(p)
    kc.load_initial(g, p, fields, scalar)
    assert g.initial() == 0
    for _ in range(n):
        assert g.step() == 0
    return g


@pytest.mark.parametrize("precision", [0, 1])
def test_fused_continuation_is_exact(rt, tmp_path, precision):
    n = 4
    p = kc.cfg_small(32, 32, 32, precision=precision)
    fields = kc.initial_fields(p, amp=0.1, seed=21)
    whole = _gpu_run(rt, p, fields, 2 * n)
    first = _gpu_run(rt, p, fields, n)
    path = str(tmp_path / "last-restart")
    first.save_restart(path)
    q = kc.cfg_small(32, 32, 32, precision=precision, irstrt=1)
    with rt.KmmContext(q) as second:
        second.load_restart(path)
        assert second.initial() == 0
        assert second.stats().it == 0
        for _ in range(n):
            assert second.step() == 0
        for f in STATE:
            assert np.array_equal(second.download(f), whole.download(f)), (precision, f)
    whole.close()
    first.close()


def test_scalar_polymer_c_restart_continuation_is_exact(rt, tmp_path):
    n = 2
    kw = dict(scalar_on=1, polymer_on=1, src_start=0, diff=1.0)
    p = kc.cfg_small(16, 32, 16, **kw)
    fields = kc.initial_fields(p, amp=0.1, seed=22)
    scl = np.asfortranarray(np.random.default_rng(6).standard_normal((33, 16, 16)) * 0.1)
    whole = _gpu_run(rt, p, fields, 2 * n, scl)
    first = _gpu_run(rt, p, fields, n, scl)
    path, cpath = str(tmp_path / "r"), str(tmp_path / "cr")
    first.save_restart(path, cpath)
    q = kc.cfg_small(16, 32, 16, irstrt=1, crstrt=1, **kw)
    with rt.KmmContext(q) as second:
        second.load_restart(path, cpath)
        assert second.initial() == 0
        for _ in range(n):
            assert second.step() == 0
        for f in STATE + ("SCALAR", "SCN", "SCNM1", "C11", "C12", "C33", "C22N", "STR13NM1"):
            assert np.array_equal(second.download(f), whole.download(f)), f
    whole.close()
    first.close()


@pytest.mark.parametrize("grid", [(32, 32, 32), (16, 32, 12)])
def test_oracle_restart_file_continued_on_gpu(rt, tmp_path, grid):
    from oracle import pyoracle
    p = kc.cfg_small(*grid)
    fields = kc.initial_fields(p, amp=0.1, seed=23)
    o = pyoracle.Oracle(p)
    kc.load_initial(o, p, fields)
    assert o.initial() == 0
    for _ in range(3):
        assert o.step() == 0
    path = str(tmp_path / "oracle-restart")
    restart.save(o.get, p, 3, path)
    for _ in range(5):
        assert o.step() == 0
    q = kc.cfg_small(*grid, irstrt=1)
    with rt.KmmContext(q) as g:
        g.load_restart(path)
        assert g.initial() == 0
        for _ in range(5):
            assert g.step() == 0
        for f in STATE:
            e = kc.rel_err(g.download(f), o.get(f))
            assert e <= RUN_TOL, "%s rel err %.3e" % (f, e)
