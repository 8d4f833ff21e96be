"""State held in host arrays (kmm_bind_host / kmm_run_host): every step uploads the bound fields
from their host arrays and downloads them back, with one step's downloads and the next step's
uploads overlapped on two copy streams.  The host arrays must hold exactly what a device-resident
run computes (same kernels, so bit for bit), a change made to a host array between calls must
reach the device, and a stop status must leave the failing step's state in the host arrays."""
import numpy as np
import pytest

from polymer_dns_b200 import abi, inputs
from tests import kmm_cases as kc

pytestmark = pytest.mark.gpu

STATE = ["V", "FN", "FNM1", "OMY", "GN", "GNM1", "U0", "H1N", "H1NM1", "W0", "H3N", "H3NM1",
         "SCALAR", "SCN", "SCNM1", "XPART", "YPART", "ZPART", "UPART", "VPART", "WPART"]


@pytest.fixture(scope="module")
def rt():
    from polymer_dns_b200 import build, runtime
    build.build()
    return runtime


def _ctx(rt, p, fused=1, seed=4):
    g = rt.KmmContext(p)
    g.call("set_option", abi.OPT_FUSED, fused)
    fields = kc.initial_fields(p, amp=0.05, seed=seed)
    sc = np.asfortranarray(0.2 * np.random.default_rng(seed).standard_normal(fields[0].shape))
    kc.load_initial(g, p, fields, sc)
    if p.npart:
        for name, arr in zip(("XPART", "YPART", "ZPART"), inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 9)):
            g.upload(name, arr)
    assert g.initial() == 0
    return g


def _bind_names(g, names):
    """Page-locked host arrays holding the context's current state, bound to their fields."""
    import torch
    host = {}
    for n in names:
        raw = g.download(n).tobytes(order="F")
        buf = torch.empty(len(raw), dtype=torch.uint8, pin_memory=True)
        buf.numpy()[:] = np.frombuffer(raw, dtype=np.uint8)
        g.bind_host(n, buf.data_ptr(), len(raw))
        host[n] = buf
    return host


def _bind(g):
    return _bind_names(g, STATE)


def _same(host, g, names=STATE):
    for n in names:
        assert host[n].numpy().tobytes() == g.download(n).tobytes(order="F"), n


def _params(**kw):
    base = dict(scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=0.5, npart=64, tracer_scheme=1)
    base.update(kw)
    return kc.cfg_small(32, 32, 32, **base)


@pytest.mark.parametrize("fused", [1, 0])
def test_run_host_matches_device_resident_run(rt, fused):
    p = _params()
    g, r = _ctx(rt, p, fused), _ctx(rt, p, fused)
    host = _bind(g)
    assert g.run_host(6) == 0
    for _ in range(6):
        assert r.step() == 0
    _same(host, r)   # the host arrays hold the last step's result
    _same(host, g)   # and so do the device mirrors
    assert g.stats().it == r.stats().it == 6
    assert g.stats().cflmax == r.stats().cflmax


def test_host_changes_reach_the_device(rt):
    """The uploads happen before every step: a host array changed between two calls is what the
    next step reads, as kmm_upload of the same array would make it."""
    p = _params()
    g, r = _ctx(rt, p), _ctx(rt, p)
    host = _bind(g)
    assert g.run_host(2) == 0
    for _ in range(2):
        assert r.step() == 0
    v = np.frombuffer(host["V"].numpy(), dtype=np.complex128).copy()
    v *= 0.5
    host["V"].numpy()[:] = np.frombuffer(v.tobytes(), dtype=np.uint8)
    r.upload("V", r.download("V") * 0.5)
    assert g.run_host(3) == 0
    for _ in range(3):
        assert r.step() == 0
    _same(host, r)


def test_stop_status_leaves_the_failing_step_in_host_arrays(rt):
    """A step that returns KMM_ERR_CFL (here: the host's v scaled up 200 times before the call)
    still downloads its state, then the call returns."""
    p = _params(npart=0)
    g = _ctx(rt, p)
    names = [n for n in STATE if not n.endswith("PART")]
    host = _bind_names(g, names)
    v = np.frombuffer(host["V"].numpy(), dtype=np.complex128) * 200.0
    host["V"].numpy()[:] = np.frombuffer(v.tobytes(), dtype=np.uint8)
    assert g.run_host(5, allow=(abi.ERR_CFL,)) == abi.ERR_CFL
    assert g.stats().it == 1
    assert g.stats().cflmax > 1.0
    _same(host, g, names)


def test_bind_host_arguments(rt):
    p = _params(npart=0)
    g = rt.KmmContext(p)
    import ctypes
    raw = (ctypes.c_char * 64)()
    buf = ctypes.addressof(raw)
    L, h = g.L, g.h
    assert L.kmm_bind_host(h, abi.FIELD["V"], buf, 64) == abi.ERR_ARG          # size mismatch
    assert L.kmm_bind_host(h, abi.FIELD["IMATRIX"], buf, 64) == abi.ERR_ARG    # layout-transformed field
    assert L.kmm_bind_host(h, abi.FIELD["FXINTG"], buf, 64) == abi.ERR_ARG
    assert L.kmm_bind_host(h, 99999, buf, 64) == abi.ERR_ARG
    assert L.kmm_bind_host(h, -1, None, 0) == 0                                # unbind all
    assert L.kmm_run_host(h, -1) == abi.ERR_ARG
    g.close()


def test_run_host_polymer_routine_path(rt):
    """The routine path with FENE-P polymer and the IB cylinder (the c-restart records bound too:
    their n-1 histories are downloaded during the step, from the buffers the step takes over)."""
    from polymer_dns_b200 import configs
    p, init, _ = configs.make("cfg3", 0, grid=32)
    f, extra = configs.build_inputs(p, init, "cfg3")
    ctxs = []
    for _ in range(2):
        c = rt.KmmContext(p)
        configs.load(f, extra, c.upload)
        assert c.initial() == 0
        ctxs.append(c)
    g, r = ctxs
    comp = ["11", "12", "13", "22", "23", "33"]
    names = [n for n in STATE] + ["C11", "C12", "C13", "C21", "C22", "C23", "C31", "C32", "C33"]
    names += ["C%sN" % c for c in comp] + ["C%sNM1" % c for c in comp]
    names += ["STR%sN" % c for c in comp] + ["STR%sNM1" % c for c in comp]
    if not p.npart:
        names = [n for n in names if not n.endswith("PART")]
    host = _bind_names(g, names)
    assert g.run_host(4) == 0
    for _ in range(4):
        assert r.step() == 0
    _same(host, r, names)
    _same(host, g, names)
