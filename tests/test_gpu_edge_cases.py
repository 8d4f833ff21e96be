"""Edge cases of the drop-in against the oracle, through the C ABI:
  - the statuses the reference stops on (CFL > 1, solvers.f90:3510-3514; a particle outside the
    grid's cells, part_track.f90:580-590) and those the drop-in adds (a non-finite state; IB types
    without a kernel; the mixed form at lengths without compiled FP32 transforms; bad arguments):
    the GPU and the oracle return the same status where both have it, and a refused call leaves
    nothing half-done;
  - grids off the compiled lengths (3/2 lengths 60 and 30, ny = 24: the runtime FFT plans and the
    one-thread-per-column solvers) and the smallest grid (8 x 9 x 8), 5 steps at 1e-10;
  - a run without particles next to one with a single particle.
"""
import ctypes
import math

import numpy as np
import pytest

from polymer_dns_b200 import abi, inputs
from tests import kmm_cases as kc

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-10


@pytest.fixture(scope="module")
def rt():
    from polymer_dns_b200 import build, runtime
    build.build()
    return runtime


def _pair(rt, oracle_mod, p, seed=3, amp=0.05, scalar=False):
    g, o = rt.KmmContext(p), oracle_mod.Oracle(p)
    fields = kc.initial_fields(p, amp=amp, seed=seed)
    sc = None
    if scalar:   # a nonzero scalar (a zero one stays at round-off on both sides)
        sc = np.asfortranarray(0.3 * np.random.default_rng(seed).standard_normal(fields[0].shape))
    for c in (g, o):
        kc.load_initial(c, p, fields, sc)
    return g, o


def _cmp(g, o, name, tol=RUN_TOL):
    e = kc.rel_err(g.download(name), o.get(name))
    assert e <= tol, "%s rel err %.3e > %.1e" % (name, e, tol)


@pytest.mark.parametrize("fused", [1, 0])
def test_cfl_stop_matches_oracle(rt, oracle_mod, fused):
    """A time step far above the CFL limit: both sides report KMM_ERR_CFL from the same call
    (initial's vcw3dp already exceeds it at dt = 0.5; at dt = 0.1 the first step does), with
    the same CFL number."""
    for dt in (0.5, 0.1):
        p = kc.cfg_small(32, 32, 32, dt=dt)
        g, o = _pair(rt, oracle_mod, p, amp=0.3)
        g.call("set_option", abi.OPT_FUSED, fused)
        sg = g.call("initial", allow=(abi.ERR_CFL,))
        so = o.initial()
        if sg == 0 and so == 0:
            sg = g.call("step", allow=(abi.ERR_CFL,))
            so = o.step()
        assert sg == so == abi.ERR_CFL, (dt, sg, so)
        assert abs(g.stats().cflmax - o.stats().cflmax) <= 1e-10 * o.stats().cflmax
        g.close()


def test_nonfinite_state_is_reported(rt, oracle_mod):
    """A NaN in the state: the GPU step reports KMM_ERR_NAN (the reference carries on into NaNs;
    its CFL test is false for NaN) and does not raise a CUDA error; the context still steps a
    clean state afterwards."""
    p = kc.cfg_small(32, 32, 32)
    g, o = _pair(rt, oracle_mod, p)
    assert g.initial() == 0
    v = g.download("V")
    v[3, 2, 1] = np.nan
    g.upload("V", v)
    assert g.call("step", allow=(abi.ERR_NAN,)) == abi.ERR_NAN
    assert not math.isfinite(g.stats().cflmax)
    g2, _ = _pair(rt, oracle_mod, p)
    assert g2.initial() == 0
    assert g2.step() == 0


def test_particle_outside_the_cells(rt, oracle_mod):
    """A tracer above the top wall (y > yl / 2): fluid_interp finds no cell and the reference stops
    (part_track.f90:580-590); both sides return KMM_ERR_INTERP."""
    p = kc.cfg_small(32, 32, 32, npart=4)
    g, o = _pair(rt, oracle_mod, p)
    xs = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 1)
    ys = np.array(xs[1])
    ys[2] = 0.5 * p.yl + 0.3
    for c in (g, o):
        setter = c.upload if hasattr(c, "upload") else c.set
        for name, arr in zip(("XPART", "YPART", "ZPART"), (xs[0], ys, xs[2])):
            setter(name, arr)
    sg = g.call("initial", allow=(abi.ERR_INTERP,))
    so = o.initial()
    if sg == 0 and so == 0:
        sg = g.call("step", allow=(abi.ERR_INTERP,))
        so = o.step()
    assert sg == so == abi.ERR_INTERP


def test_unsupported_ib_types_are_refused(rt, oracle_mod):
    """imatrix types 6, 7, 8 (buffer, suction, moving wall) have no kernel: vcw3dp returns
    KMM_ERR_UNSUPPORTED on both sides instead of running without them."""
    p = kc.cfg_small(16, 16, 12)
    g, o = _pair(rt, oracle_mod, p)
    im = inputs.cylinder_imatrix(p.nx, p.ny, p.nz, p.xl, p.yl, math.pi, 0.0, 0.25)
    im = np.array(im)
    im.flat[im.size // 2] = 7
    g.upload("IMATRIX", im)
    o.set("IMATRIX", im)
    assert g.call("initial", allow=(abi.ERR_UNSUPPORTED,)) == abi.ERR_UNSUPPORTED
    assert o.initial() == abi.ERR_UNSUPPORTED


def test_mixed_form_refuses_uncompiled_lengths(rt):
    """precision = 1 at nx = 40 (3/2 length 60, no compiled FP32 transform): KMM_ERR_UNSUPPORTED,
    never a silent FP64 step."""
    p = kc.cfg_small(40, 32, 32, precision=1)
    g = rt.KmmContext(p)
    fields = kc.initial_fields(p, amp=0.05, seed=2)
    kc.load_initial(g, p, fields)
    assert g.initial() == 0
    assert g.call("step", allow=(abi.ERR_UNSUPPORTED,)) == abi.ERR_UNSUPPORTED
    assert g.stats().it == 0 or g.stats().status == abi.ERR_UNSUPPORTED


def test_bad_arguments(rt):
    """Unknown field ids, size mismatches, options out of range and null pointers return KMM_ERR_ARG
    before any device work."""
    p = kc.cfg_small(16, 16, 12)
    g = rt.KmmContext(p)
    L, h = g.L, g.h
    buf = np.zeros(16, np.float64)
    ptr = buf.ctypes.data
    assert L.kmm_upload(h, 99999, ptr, buf.nbytes) == abi.ERR_ARG
    assert L.kmm_upload(h, abi.FIELD["V"], ptr, buf.nbytes) == abi.ERR_ARG        # size mismatch
    assert L.kmm_download(h, abi.FIELD["V"], ptr, buf.nbytes) == abi.ERR_ARG
    assert L.kmm_set_option(h, 12345, 1) == abi.ERR_ARG
    assert L.kmm_set_option(h, abi.OPT_WAIT_LIMIT_MS, 5) == abi.ERR_ARG           # below 100 ms
    assert L.kmm_target_list(h, ctypes.POINTER(ctypes.c_int)(), -1) == -abi.ERR_ARG
    assert L.kmm_cderiv(h, abi.FIELD["V"], abi.FIELD["V"]) == abi.ERR_ARG          # in place
    g.close()


@pytest.mark.parametrize("grid", [(40, 24, 20), (8, 8, 8)])
def test_uncompiled_and_tiny_grids_match_oracle(rt, oracle_mod, grid):
    """3/2 lengths 60 and 30 and ny = 24 (runtime FFT plans, one thread per column), and the
    smallest grid: a scalar and tracers, 5 steps against the oracle at 1e-10."""
    nx, ny, nz = grid
    p = kc.cfg_small(nx, ny, nz, scalar_on=1, diff=1.0, npart=16, dt=0.002)
    g, o = _pair(rt, oracle_mod, p, scalar=True)
    xs = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 7)
    for c in (g, o):
        setter = c.upload if hasattr(c, "upload") else c.set
        for name, arr in zip(("XPART", "YPART", "ZPART"), xs):
            setter(name, arr)
        assert c.initial() == 0
    for _ in range(5):
        assert g.step() == 0
        assert o.step() == 0
    for name in ("V", "OMY", "FN", "GN", "SCALAR", "U0", "XPART", "YPART"):
        _cmp(g, o, name)


@pytest.mark.parametrize("npart", [0, 1])
def test_zero_and_one_particle(rt, oracle_mod, npart):
    p = kc.cfg_small(32, 32, 32, npart=npart, tracer_scheme=1)
    g, o = _pair(rt, oracle_mod, p)
    if npart:
        xs = inputs.uniform_particles(npart, p.xl, p.yl, p.zl, p.ap, 8)
        for name, arr in zip(("XPART", "YPART", "ZPART"), xs):
            g.upload(name, arr)
            o.set(name, arr)
    assert g.initial() == 0 and o.initial() == 0
    for _ in range(5):
        assert g.step() == 0
        assert o.step() == 0
    names = ["V", "OMY", "FN", "GN"] + (["XPART", "YPART", "ZPART"] if npart else [])
    for name in names:
        _cmp(g, o, name)
