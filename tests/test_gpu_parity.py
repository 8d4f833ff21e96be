"""GPU parity: every routine of the C ABI against the CPU oracle on the same seeded inputs.

Tolerances (FP64 drop-in): per-routine results agree to <= 1e-12 relative (the column routines
share the reference's operation order; transforms differ only in FFT rounding); whole runs agree
to <= 1e-10 relative after 10 steps, the bar of the FP64 drop-in.  Relative error = max|a-b| /
max|b| per field.
"""
import math

import numpy as np
import pytest

from polymer_dns_b200 import abi, inputs
from tests import kmm_cases as kc

pytestmark = pytest.mark.gpu

ROUTINE_TOL = 1e-12
RUN_TOL = 1e-10


@pytest.fixture(scope="module")
def rt():
    from polymer_dns_b200 import build, runtime
    build.build()
    return runtime


def _pair(rt, oracle_mod, p):
    return rt.KmmContext(p), oracle_mod.Oracle(p)


def _put(g, o, name, a):
    g.upload(name, a)
    o.set(name, a)


def _cmp(g, o, name, tol=ROUTINE_TOL):
    e = kc.rel_err(g.download(name), o.get(name))
    assert e <= tol, "%s rel err %.3e > %.1e" % (name, e, tol)
    return e


GRIDS = [(16, 16, 12), (32, 32, 32), (24, 24, 16)]


@pytest.mark.parametrize("grid", GRIDS)
def test_cderiv_wallderiv_norm(rt, oracle_mod, grid):
    p = kc.cfg_small(*grid)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(11)
    a = kc.random_spectral(rng, p, hermitian=False)
    _put(g, o, "WRKC", a)
    g.call("cderiv", "WRKC", "WRK1")
    o.call("cderiv", "WRKC", "WRK1")
    assert np.array_equal(g.download("WRK1"), o.get("WRK1"))   # same operation order: bitwise
    for order in (0, 1, 2):
        for wall in (0, 1):
            g.call("wallderiv", "WRKC", order, wall, "WRK1", 2 + order)
            o.call("wallderiv", "WRKC", order, wall, "WRK1", 2 + order)
    _cmp(g, o, "WRK1")
    g.call("norm", "WRKC")
    o.call("norm", "WRKC")
    assert np.array_equal(g.download("WRKC"), o.get("WRKC"))


@pytest.mark.parametrize("ny", [48, 64, 96, 128])
def test_cderiv_half_warp_is_bitwise(rt, oracle_mod, ny):
    """cderiv at ny = 16 K runs a half-warp per column with the chains handed lane to lane; the
    sums keep the serial order, so the result is bitwise the oracle's."""
    p = kc.cfg_small(20, ny, 12)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(17 + ny)
    a = kc.random_spectral(rng, p, hermitian=False)
    _put(g, o, "WRKC", a)
    g.call("cderiv", "WRKC", "WRK1")
    o.call("cderiv", "WRKC", "WRK1")
    assert np.array_equal(g.download("WRK1"), o.get("WRK1"))


@pytest.mark.parametrize("ny,theta", [(16, 0.5), (32, 1.0), (64, 0.5), (128, 0.5), (128, 1.0)])
def test_uzero_block_solve(rt, oracle_mod, ny, theta):
    """The (0,0)-mode solve with its row work spread over a block and its recurrences on single
    threads, against the oracle for both theta branches (theta > 0.99 skips the two cderivs)."""
    p = kc.cfg_small(16, ny, 12, theta=theta)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(5 + ny)
    for name in ("U0", "W0", "H1N", "H1NM1", "H3N", "H3NM1"):
        v = np.zeros(p.ny + 1)
        v[: min(12, p.ny + 1)] = rng.standard_normal(min(12, p.ny + 1))
        _put(g, o, name, v)
    for uflag, name in ((1, "U0"), (3, "W0")):
        g.call("uzero", uflag)
        o.call("uzero", uflag)
        _cmp(g, o, name)


@pytest.mark.parametrize("grid", GRIDS)
def test_tau_solvers(rt, oracle_mod, grid):
    p = kc.cfg_small(*grid)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(12)
    for g_, ib in ((p.re / (p.dt * p.theta), 0), (0.0, 0), (1000.0, 1), (0.0, 1)):
        a = kc.random_spectral(rng, p, hermitian=False)
        bt = rng.standard_normal((p.nz, p.nx // 2)) + 1j * rng.standard_normal((p.nz, p.nx // 2))
        bb = rng.standard_normal((p.nz, p.nx // 2)) + 1j * rng.standard_normal((p.nz, p.nx // 2))
        for name, v in (("WRKC", a), ("BCTOP", bt), ("BCBOT", bb)):
            _put(g, o, name, v)
        g.call("solve", "WRKC", g_, ib)
        o.call("solve", "WRKC", g_, ib)
        _cmp(g, o, "WRKC")
    for at, bt_, ab, bb_ in ((1.0, 0.0, 1.0, 0.0), (0.0, 1.0, 0.0, 1.0), (1.0, 0.3, 0.7, 0.5)):
        a = kc.random_spectral(rng, p, hermitian=False)
        _put(g, o, "WRKC", a)
        gt = rng.standard_normal((p.nz, p.nx // 2)) + 1j * rng.standard_normal((p.nz, p.nx // 2))
        _put(g, o, "BCTOP", gt)
        _put(g, o, "BCBOT", -gt)
        g.call("penta", "WRKC", 2800.0, 0, at, bt_, ab, bb_)
        o.call("penta", "WRKC", 2800.0, 0, at, bt_, ab, bb_)
        _cmp(g, o, "WRKC")


def test_mean_mode_and_spectral_routines(rt, oracle_mod):
    p = kc.cfg_small(16, 24, 16)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(13)
    for name in ("V", "OMY", "FN", "FNM1", "GN", "GNM1", "OMZ", "U", "W"):
        _put(g, o, name, kc.random_spectral(rng, p))
    for name in ("U0", "W0", "H1N", "H1NM1", "H3N", "H3NM1"):
        v = np.zeros(p.ny + 1)
        v[:12] = rng.standard_normal(12)
        _put(g, o, name, v)
    for r in ("phi_from_v",):
        g.call(r); o.call(r)
    _cmp(g, o, "V")
    g.call("phirhs", "V", "FN", "FNM1", 1.0)
    o.call("phirhs", "V", "FN", "FNM1", 1.0)
    _cmp(g, o, "V")
    g.call("uzero", 1); o.call("uzero", 1)
    g.call("uzero", 3); o.call("uzero", 3)
    _cmp(g, o, "U0")
    _cmp(g, o, "W0")
    for r in ("veloc", "vort", "gradv", "nonlin"):
        g.call(r)
        o.call(r)
    for name in ("U", "W", "OMX", "OMZ", "U11", "U12", "U33", "LU", "LW", "FN", "GN"):
        _cmp(g, o, name)
    g.call("filter"); o.call("filter")
    for name in ("FN", "GN", "OMZ"):
        _cmp(g, o, name)


def test_gfcn_and_influence(rt, oracle_mod):
    p = kc.cfg_small(16, 32, 16)
    g, o = _pair(rt, oracle_mod, p)
    g.call("gfcn")
    o.call("gfcn")
    for name in ("GF1", "GF2", "DNV1B", "DNV1T", "DNV2B", "DNV2T", "DENOM"):
        _cmp(g, o, name)
    rng = np.random.default_rng(14)
    _put(g, o, "V", kc.random_spectral(rng, p))
    g.call("influence")
    o.call("influence")
    _cmp(g, o, "V")


@pytest.mark.parametrize("grid", GRIDS)
def test_xyzfft(rt, oracle_mod, grid):
    p = kc.cfg_small(*grid)
    g, o = _pair(rt, oracle_mod, p)
    iu, iv, iw = kc.initial_fields(p)
    _put(g, o, "INITU", iu)
    g.call("xyzfft", "U", "INITU")
    o.call("xyzfft", "U", "INITU")
    _cmp(g, o, "U")


@pytest.mark.parametrize("grid", GRIDS)
def test_vcw3dp_fluid(rt, oracle_mod, grid):
    p = kc.cfg_small(*grid, dt=1e-5)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(15)
    for name in ("U", "V", "W", "OMX", "OMY", "OMZ"):
        _put(g, o, name, kc.random_spectral(rng, p))
    assert g.call("vcw3dp") == 0
    assert o.call("vcw3dp") == 0
    for name in ("GN", "FN", "OMZ"):
        _cmp(g, o, name)
    _cmp(g, o, "UP3D")
    assert abs(g.stats().cflmax - o.stats().cflmax) <= 1e-12 * o.stats().cflmax


@pytest.mark.parametrize("grid", [(16, 24, 16), (32, 48, 32), (16, 64, 16)])
def test_vcw3dp_scalar_polymer_ib(rt, oracle_mod, grid):
    """All 55 input fields through vcw3dp; ny = 48 and 64 take the half-length DCT-I kernels, ny = 24
    the 2 ny-point FFT form."""
    p = kc.cfg_small(*grid, dt=1e-5, scalar_on=1, polymer_on=1, scalar_q=0.3, zlmax=30.0, tpoly=20.0,
                     qbeta=0.9, gain=2.0, ugain=40.0)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(16)
    names = ["U", "V", "W", "OMX", "OMY", "OMZ", "U11", "U12", "U13", "U21", "U22", "U23", "U31", "U32", "U33",
             "SCALAR", "SCLX", "SCLY", "SCLZ"] + ["C%d%d" % (i, j) for i in (1, 2, 3) for j in (1, 2, 3)] \
        + ["DC%d%d%d" % (i, j, k) for i in (1, 2, 3) for j in (1, 2, 3) for k in (1, 2, 3)]
    for name in names:
        a = kc.random_spectral(rng, p) * 0.1
        if name in ("C11", "C22", "C33"):
            a[0, 0, 0] += 1.0
        _put(g, o, name, a)
    im = inputs.cylinder_imatrix(p.nx, p.ny, p.nz, p.xl, p.yl, xc=math.pi, yc=0.0, radius=0.25)
    _put(g, o, "IMATRIX", im)
    fx = rng.standard_normal(im.shape) * 0.01
    _put(g, o, "FXINTG", np.asfortranarray(fx))
    assert g.call("vcw3dp") == 0
    assert o.call("vcw3dp") == 0
    for name in ("GN", "FN", "OMZ", "SCN", "C11N", "C23N", "STR11N", "STR33N", "QP12", "QP33"):
        _cmp(g, o, name)
    for name in ("FXINTG", "FYINTG", "FZINTG"):
        _cmp(g, o, name)


def test_spreading_semantics(rt, oracle_mod):
    """Solid cells inside the spreading planes (i <= kmaxsurf) exercise the 5x5 scatter order."""
    p = kc.cfg_small(16, 16, 12, dt=1e-5, gain=4.0, ugain=2.0)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(17)
    for name in ("U", "V", "W", "OMX", "OMY", "OMZ"):
        _put(g, o, name, kc.random_spectral(rng, p))
    mx, mz = 3 * p.nx // 2, 3 * p.nz // 2
    im = np.zeros((p.ny + 1, mz, mx), np.int32, order="F")
    im[1:6, :, 3:9] = 1                 # planes 2..6 (1-based), x columns 4..9 -> kmaxsurf = 9
    im[2, 0:2, 0] = 3                   # z-edge cells next to the x seam
    im[3, mz - 2:, mx - 1] = 1
    _put(g, o, "IMATRIX", im)
    assert g.call("vcw3dp") == 0
    assert o.call("vcw3dp") == 0
    for name in ("GN", "FN", "OMZ", "FXINTG", "FZINTG"):
        _cmp(g, o, name)


def test_tracers(rt, oracle_mod):
    p = kc.cfg_small(16, 24, 16, npart=2000, ap=1e-3, dt=1e-3)
    g, o = _pair(rt, oracle_mod, p)
    rng = np.random.default_rng(18)
    for name in ("U", "V", "W", "OMX", "OMY", "OMZ"):
        _put(g, o, name, kc.random_spectral(rng, p) * 0.05)
    x, y, z = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 2)
    for n, a in (("XPART", x), ("YPART", y), ("ZPART", z)):
        _put(g, o, n, a)
    for it in (0, 1, 2):
        g.call("set_it", it)
        o.call("set_it", it)
        assert g.call("vcw3dp") == 0
        assert o.call("vcw3dp") == 0
    for n in ("XPART", "YPART", "ZPART", "UPART", "VPART", "WPART"):
        _cmp(g, o, n)


# ----------------------------------------------------------------------------- whole runs
def _run_pair(rt, oracle_mod, p, nsteps, fields, scalar=None, imatrix=None, particles=None):
    g, o = _pair(rt, oracle_mod, p)
    for ctx in (g, o):
        kc.load_initial(ctx, p, fields, scalar)
        if imatrix is not None:
            (ctx.upload if hasattr(ctx, "upload") else ctx.set)("IMATRIX", imatrix)
        if particles is not None:
            for n, a in zip(("XPART", "YPART", "ZPART"), particles):
                (ctx.upload if hasattr(ctx, "upload") else ctx.set)(n, a)
    assert g.initial() == 0
    assert o.initial() == 0
    for _ in range(nsteps):
        assert g.step() == 0
        assert o.step() == 0
    return g, o


@pytest.mark.parametrize("grid", [(32, 32, 32), (24, 32, 16)])
def test_fp64_dropin_10_steps(rt, oracle_mod, grid):
    """The plain drop-in bar: max relative field difference <= 1e-10 after 10 steps."""
    p = kc.cfg_small(*grid)
    g, o = _run_pair(rt, oracle_mod, p, 10, kc.initial_fields(p, amp=0.05, seed=0))
    for name in kc.SPECTRAL_STATE[:6]:
        _cmp(g, o, name, RUN_TOL)
    for name in kc.MEAN_STATE:
        _cmp(g, o, name, RUN_TOL)


def test_dropin_scalar_tracers_10_steps(rt, oracle_mod):
    p = kc.cfg_small(32, 32, 32, scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=1.0, npart=1000, ap=1e-3,
                     tracer_scheme=0)
    fields = kc.initial_fields(p, amp=0.05, seed=1)
    parts = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 2)
    g, o = _run_pair(rt, oracle_mod, p, 10, fields, scalar=np.zeros_like(fields[0]), particles=parts)
    for name in ("V", "OMY", "FN", "GN", "SCALAR", "SCN"):
        _cmp(g, o, name, RUN_TOL)
    for name in ("XPART", "YPART", "ZPART"):
        _cmp(g, o, name, RUN_TOL)


def test_dropin_polymer_ib_10_steps(rt, oracle_mod):
    p = kc.cfg_small(32, 32, 32, scalar_on=1, polymer_on=1, diff=1.0, scalar_bc=1, scalar_q=1.0,
                     zlmax=30.0, tpoly=20.0, qbeta=0.9, diffpoly=1000.0, gain=2.0, ugain=40.0, dt=0.005)
    fields = kc.initial_fields(p, amp=0.05, seed=1)
    im = inputs.cylinder_imatrix(p.nx, p.ny, p.nz, p.xl, p.yl, xc=math.pi, yc=0.0, radius=0.25)
    g, o = _run_pair(rt, oracle_mod, p, 10, fields, scalar=np.zeros_like(fields[0]), imatrix=im)
    for name in ("V", "OMY", "FN", "GN", "SCALAR", "C11", "C12", "C22", "C33", "STR11N", "QP12"):
        _cmp(g, o, name, RUN_TOL)


def test_full_size_properties():
    """128x129x128 (the Re_tau = 180 grid): continuity and the laminar steady state hold on the GPU."""
    from polymer_dns_b200 import runtime
    p = kc.cfg_small(128, 128, 128, dt=0.005, re=2800.0, xl=4 * math.pi, zl=4 * math.pi / 3)
    with runtime.KmmContext(p) as g:
        kc.load_initial(g, p, kc.initial_fields(p, amp=0.0))
        assert g.initial() == 0
        u0 = g.download("U0")
        assert g.run(5) == 0
        assert np.abs(g.download("U0") - u0).max() < 1e-12
        assert np.abs(g.download("V")).max() < 1e-12
    with runtime.KmmContext(p) as g:
        kc.load_initial(g, p, kc.initial_fields(p, profile="loglaw", amp=0.1, kmax=8, seed=1))
        assert g.initial() == 0
        assert g.run(5) == 0
        g.call("veloc")   # the fused step keeps the prognostic state; u, w are derived on demand
        u, w = g.download("U"), g.download("W")
        g.call("cderiv", "V", "WRKC")
        dv = g.download("WRKC")
        kx = np.arange(p.nx // 2) * 2 * math.pi / p.xl
        kz = np.fft.fftfreq(p.nz, 1.0 / p.nz) * 2 * math.pi / p.zl
        div = 1j * kx[None, None, :] * u + dv + 1j * kz[None, :, None] * w
        assert np.abs(div).max() < 1e-11 * np.abs(u).max()
        assert 0 < g.stats().cflmax < 1.0


@pytest.mark.parametrize("grid,scalar", [((32, 32, 32), 0), ((24, 32, 16), 1), ((16, 64, 12), 1), ((16, 96, 12), 0),
                                         ((16, 128, 16), 1), ((16, 32, 64), 1), ((16, 32, 96), 0), ((16, 32, 128), 1)])
def test_fused_step_matches_routine_path(rt, oracle_mod, grid, scalar):
    """kmm_step's fused kernels against the routine-by-routine kernels and the oracle after 5 steps."""
    kw = dict(scalar_on=scalar, diff=1.0, scalar_bc=1, scalar_q=0.5) if scalar else {}
    p = kc.cfg_small(*grid, **kw)
    fields = kc.initial_fields(p, amp=0.05, seed=3)
    sc = np.zeros_like(fields[0]) if scalar else None
    ctxs = []
    for fused in (1, 0):
        g = rt.KmmContext(p)
        g.call("set_option", 1, fused)
        kc.load_initial(g, p, fields, sc)
        assert g.initial() == 0
        ctxs.append(g)
    o = oracle_mod.Oracle(p)
    kc.load_initial(o, p, fields, sc)
    assert o.initial() == 0
    for _ in range(5):
        for g in ctxs:
            assert g.step() == 0
        assert o.step() == 0
    names = ["V", "OMY", "FN", "FNM1", "GN", "GNM1", "U0", "W0", "H1N", "H3N"] + (["SCALAR", "SCN", "SCNM1"] if scalar else [])
    for name in names:
        a, b = ctxs[0].download(name), ctxs[1].download(name)
        assert kc.rel_err(a, b) <= 1e-12, name
        _cmp(ctxs[0], o, name, RUN_TOL)


@pytest.mark.parametrize("grid", [(16, 32, 16), (16, 64, 12), (12, 96, 12), (16, 128, 16)])
def test_blocked_columns_match_warp_columns(rt, grid):
    """The fused step's blocked-layout column kernels (16 lanes per column) against the
    warp-per-column kernels, with scalar, after 5 steps (KMM_OPT_COLUMN_BLOCKED on / off)."""
    p = kc.cfg_small(*grid, scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=0.5)
    fields = kc.initial_fields(p, amp=0.05, seed=4)
    sc = np.zeros_like(fields[0])
    ctxs = []
    for blocked in (1, 0):
        g = rt.KmmContext(p)
        g.call("set_option", 2, blocked)
        kc.load_initial(g, p, fields, sc)
        assert g.initial() == 0
        ctxs.append(g)
    for _ in range(5):
        for g in ctxs:
            assert g.step() == 0
    for name in ["V", "OMY", "FN", "FNM1", "GN", "GNM1", "U0", "W0", "H1N", "H3N", "SCALAR", "SCN", "SCNM1"]:
        a, b = ctxs[0].download(name), ctxs[1].download(name)
        assert kc.rel_err(a, b) <= 1e-12, name


def test_calcswirl_matches_oracle(rt, oracle_mod):
    """kmm_calcswirl (helpers.f90:197-404) against the oracle on the gradients of a random
    divergence-free field, with particles.  The reference's closed form is ill-conditioned in two
    places: near a zero discriminant Q^2 - P^3 the square root turns O(eps) rounding into
    O(sqrt(eps)) imaginary parts, and for Q < 0 with |P|^3 << Q^2 the sum Q + sqrt(Q^2 - P^3)
    cancels.  There each implementation returns its own rounding (up to ~1e-6 of the largest
    swirl; where the eigenvalues are real, a residue near 1e-8 instead of 0).  Bars: of the
    points with a clear complex pair (swirl > 1e-4 of the largest), at least 99.9% agree to 1e-9
    of the largest swirl; every point and every particle agrees to 1e-5 of it."""
    p = kc.cfg_small(24, 32, 16, npart=64)
    g, o = _pair(rt, oracle_mod, p)
    fields = kc.initial_fields(p, amp=0.3, seed=5)
    kc.load_initial(g, p, fields)
    kc.load_initial(o, p, fields)
    assert g.initial() == 0 and o.initial() == 0
    for ctx in (g, o):
        ctx.call("veloc")
        ctx.call("gradv")
    xs = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, seed=6)
    for name, arr in zip(("XPART", "YPART", "ZPART"), xs):
        _put(g, o, name, arr)
    assert g.call("calcswirl") == 0
    assert o.call("calcswirl") == 0
    a, b = g.download("SWIRL3D"), o.get("SWIRL3D")
    scale = np.abs(b).max()
    assert scale > 0
    diff = np.abs(a - b)
    clear = b > 1e-4 * scale
    assert clear.mean() > 0.5
    assert np.mean(diff[clear] > 1e-9 * scale) < 0.001
    assert diff.max() <= 1e-5 * scale
    sa, sb = g.download("SWIRLPART"), o.get("SWIRLPART")
    assert np.abs(sa - sb).max() <= 1e-5 * scale


@pytest.mark.parametrize("grid", [(32, 32, 32), (32, 64, 32), (32, 32, 96)])
def test_mixed_precision_tracks_fp64(rt, grid):
    """The mixed-precision form (precision = 1: FP32 transforms and products, FP64 solves) against
    the FP64 drop-in from the same state after 10 steps, with scalar and tracers.  FP32 rounding of
    the nonlinear terms gives relative field differences of order 1e-7..1e-6; the bar is 1e-5."""
    kw = dict(scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=0.5, npart=128, tracer_scheme=1)
    ctxs = []
    for prec in (0, 1):
        p = kc.cfg_small(*grid, precision=prec, **kw)
        fields = kc.initial_fields(p, amp=0.1, seed=7)
        g = rt.KmmContext(p)
        kc.load_initial(g, p, fields, np.zeros_like(fields[0]))
        parts = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 3)
        for name, arr in zip(("XPART", "YPART", "ZPART"), parts):
            g.upload(name, arr)
        assert g.initial() == 0
        ctxs.append(g)
    for _ in range(10):
        for g in ctxs:
            assert g.step() == 0
    worst = 0.0
    for name in ["V", "OMY", "FN", "GN", "U0", "W0", "SCALAR", "SCN"]:
        e = kc.rel_err(ctxs[1].download(name), ctxs[0].download(name))
        worst = max(worst, e)
        assert e <= 1e-5, "%s rel err %.3e" % (name, e)
    assert worst > 1e-12   # the mixed form really runs in FP32
    for name in ("XPART", "YPART", "ZPART"):
        assert kc.rel_err(ctxs[1].download(name), ctxs[0].download(name)) <= 1e-6


def test_flowstats_matches_oracle(rt, oracle_mod):
    """kmm_flowstats (Parseval sums over the modes) against the oracle's literal restatement of
    writeoutputs (3/2-grid loops, helpers.f90:1227-1438) on a perturbed channel with a scalar."""
    p = kc.cfg_small(24, 32, 16, scalar_on=1, diff=1.0)
    g, o = _pair(rt, oracle_mod, p)
    fields = kc.initial_fields(p, profile="loglaw", amp=0.2, seed=8)
    kc.load_initial(g, p, fields, np.zeros_like(fields[0]))
    kc.load_initial(o, p, fields, np.zeros_like(fields[0]))
    assert g.initial() == 0 and o.initial() == 0
    for _ in range(3):
        assert g.step() == 0 and o.step() == 0
    pg, sg = g.flowstats()
    po, so = o.flowstats()
    for m in range(7):
        e = kc.rel_err(pg[m], po[m])
        assert e <= 1e-10, "profile %d rel err %.3e" % (m, e)
    assert np.allclose(sg, so, rtol=1e-10, atol=1e-14)


def test_ensemble_matches_independent_runs(rt):
    """kmm_ensemble_run (all members enqueued on their own streams before any is waited on) gives
    each member exactly the state of the same run stepped alone: uneven grids, a scalar, tracers,
    one mixed-precision member and one member on the routine path (immersed boundary)."""
    specs = [dict(grid=(32, 32, 32)),
             dict(grid=(16, 32, 12), scalar_on=1, diff=1.0, npart=64),
             dict(grid=(32, 64, 32), precision=1, scalar_on=1, diff=1.0),
             dict(grid=(16, 32, 12), ib=True)]

    def make(spec):
        kw = {k: v for k, v in spec.items() if k not in ("grid", "ib")}
        p = kc.cfg_small(*spec["grid"], **kw)
        fields = kc.initial_fields(p, amp=0.1, seed=9)
        g = rt.KmmContext(p)
        kc.load_initial(g, p, fields, np.zeros_like(fields[0]) if p.scalar_on else None)
        if p.npart:
            for name, arr in zip(("XPART", "YPART", "ZPART"), inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 4)):
                g.upload(name, arr)
        if spec.get("ib"):
            g.upload("IMATRIX", inputs.cylinder_imatrix(p.nx, p.ny, p.nz, p.xl, p.yl, math.pi, 0.0, 0.25))
        assert g.initial() == 0
        return g

    ens = [make(s) for s in specs]
    alone = [make(s) for s in specs]
    st = rt.ensemble_run(ens, 5)
    assert st == [0] * len(specs)
    for g in alone:
        for _ in range(5):
            assert g.step() == 0
    for a, b in zip(ens, alone):
        for name in ["V", "OMY", "FN", "GN", "U0", "W0"]:
            assert np.array_equal(a.download(name), b.download(name)), name


def test_ensemble_graph_matches_independent_runs(rt):
    """Every member on the fused step: kmm_ensemble_step replays the whole ensemble step as one
    parent graph of the members' step graphs (KMM_OPT_ENSEMBLE_GRAPH = 1).  Each member ends in
    exactly the state of the same run stepped alone, and of the ensemble with the option off;
    after a member is destroyed and a new one takes its place, the cached parent graph is not
    reused (the new member is also exact)."""
    specs = [dict(grid=(32, 32, 32)),
             dict(grid=(16, 32, 12), scalar_on=1, diff=1.0, npart=64, tracer_scheme=1),
             dict(grid=(32, 64, 32), precision=1, scalar_on=1, diff=1.0),
             dict(grid=(48, 32, 32), scalar_on=1, diff=1.0, npart=32)]

    def make(spec, graph=1):
        kw = {k: v for k, v in spec.items() if k != "grid"}
        p = kc.cfg_small(*spec["grid"], **kw)
        fields = kc.initial_fields(p, amp=0.1, seed=12)
        g = rt.KmmContext(p)
        g.call("set_option", abi.OPT_ENSEMBLE_GRAPH, graph)
        kc.load_initial(g, p, fields, np.zeros_like(fields[0]) if p.scalar_on else None)
        if p.npart:
            for name, arr in zip(("XPART", "YPART", "ZPART"), inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 4)):
                g.upload(name, arr)
        assert g.initial() == 0
        return g

    names = ["V", "OMY", "FN", "GN", "U0", "W0"]
    ens = [make(s) for s in specs]
    off = [make(s, graph=0) for s in specs]
    alone = [make(s) for s in specs]
    assert rt.ensemble_run(ens, 6) == [0] * len(specs)
    assert rt.ensemble_run(off, 6) == [0] * len(specs)
    for g in alone:
        for _ in range(6):
            assert g.step() == 0
    for a, b, c in zip(ens, off, alone):
        for name in names:
            assert np.array_equal(a.download(name), c.download(name)), name
            assert np.array_equal(b.download(name), c.download(name)), name
    # replace member 1: the parent graph cached for the old member set must not be replayed
    ens[1].close()
    ens[1] = make(specs[1])
    lone = make(specs[1])
    assert rt.ensemble_run(ens, 3) == [0] * len(specs)
    for _ in range(3):
        assert lone.step() == 0
    for name in names:
        assert np.array_equal(ens[1].download(name), lone.download(name)), name
    for g in ens + off + alone + [lone]:
        g.close()


def test_graph_replay_matches_kernel_launches(rt):
    """The fused step replayed from its two captured CUDA graphs (KMM_OPT_GRAPH) against the same
    step launched kernel by kernel: identical fields, particles and CFL after 7 steps (scalar,
    RK3 tracers; FP64 and mixed precision)."""
    for prec in (0, 1):
        p = kc.cfg_small(32, 32, 32, scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=0.5, npart=256,
                         tracer_scheme=1, precision=prec)
        fields = kc.initial_fields(p, amp=0.1, seed=11)
        parts = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 5)
        ctxs = []
        for graph in (1, 0):
            g = rt.KmmContext(p)
            g.call("set_option", 3, graph)
            kc.load_initial(g, p, fields, np.zeros_like(fields[0]))
            for name, arr in zip(("XPART", "YPART", "ZPART"), parts):
                g.upload(name, arr)
            assert g.initial() == 0
            ctxs.append(g)
        for _ in range(7):
            for g in ctxs:
                assert g.step() == 0
        for name in ["V", "OMY", "FN", "FNM1", "GN", "GNM1", "U0", "W0", "SCALAR", "SCN", "SCNM1", "XPART", "UPART"]:
            assert np.array_equal(ctxs[0].download(name), ctxs[1].download(name)), (prec, name)
        assert ctxs[0].stats().cflmax == ctxs[1].stats().cflmax
        assert ctxs[0].launch_count() == ctxs[1].launch_count()


@pytest.mark.parametrize("grid,scalar,prec", [((32, 32, 128), 1, 0), ((16, 64, 96), 0, 0), ((16, 32, 64), 1, 0),
                                              ((32, 32, 32), 0, 0), ((32, 32, 128), 1, 1), ((32, 64, 96), 0, 1),
                                              ((32, 32, 64), 1, 1), ((32, 32, 32), 1, 1)])
def test_tma_z_transform_matches_plain_loads(rt, grid, scalar, prec):
    """The z transforms with TMA tile copies (KMM_OPT_ZTMA = 1, the default) against the same
    transforms with plain loads and stores: same FFTs and operation order, so the states agree to
    rounding after 4 fused steps, at every specialised z length: 1e-13 relative in FP64, 1e-5 in
    the mixed form (FP32 intermediates)."""
    kw = dict(scalar_on=scalar, diff=1.0, scalar_bc=1, scalar_q=0.5) if scalar else {}
    kw["precision"] = prec
    p = kc.cfg_small(*grid, **kw)
    fields = kc.initial_fields(p, amp=0.1, seed=13)
    sc = np.zeros_like(fields[0]) if scalar else None
    ctxs = []
    for ztma in (1, 0):
        g = rt.KmmContext(p)
        g.call("set_option", 4, ztma)
        kc.load_initial(g, p, fields, sc)
        assert g.initial() == 0
        ctxs.append(g)
    for _ in range(4):
        for g in ctxs:
            assert g.step() == 0
    tol = 1e-13 if prec == 0 else 1e-5
    for name in ["V", "OMY", "FN", "GN", "U0", "W0"] + (["SCALAR", "SCN"] if scalar else []):
        e = kc.rel_err(ctxs[0].download(name), ctxs[1].download(name))
        assert e <= tol, (name, e)


def test_particle_scalar_source_matches_oracle(rt, oracle_mod):
    """scl_flag = 2: the particle-Gaussian scalar source (solvers.f90:2079-2118, added to the
    scalar's nonlinear term at 3061-3063) inside and after the src_start..src_stop window, with
    the tracers moving the sources; whole-run bar after 5 steps."""
    p = kc.cfg_small(32, 32, 32, scalar_on=1, diff=1.0, scl_flag=2, npart=200, deltat=0.5, sigmax=0.1,
                     sigmay=0.05, sigmaz=0.1, src_start=0, src_stop=3)
    fields = kc.initial_fields(p, amp=0.1, seed=17)
    parts = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 9)
    sc = np.zeros_like(fields[0])
    g, o = _pair(rt, oracle_mod, p)
    for c in (g, o):
        kc.load_initial(c, p, fields, sc)
        setter = c.upload if hasattr(c, "upload") else c.set
        for name, arr in zip(("XPART", "YPART", "ZPART"), parts):
            setter(name, arr)
        assert c.initial() == 0
    for _ in range(5):
        assert g.step() == 0
        assert o.step() == 0
    for name in ["SCALAR", "SCN", "SCNM1", "V", "XPART", "ZPART"]:
        _cmp(g, o, name, RUN_TOL)
    assert np.abs(g.download("SCALAR")).max() > 1e-3   # the source did act


@pytest.mark.parametrize("variant", ["polymer_ib", "inertial", "routine_plain"])
def test_mixed_precision_routine_path_tracks_fp64(rt, variant):
    """The mixed form on the routine path (polymer + IB, inertial particles, or a plain run with the
    fused step switched off): FP32 y / z / x transforms and plane intermediates, pointwise terms
    from the FP32 values, FP64 solves and state, against the FP64 drop-in from the same state after
    10 steps; the bar is 1e-5 relative, as for the fused mixed form."""
    kw = dict(scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=0.5)
    im = None
    if variant == "polymer_ib":
        kw.update(polymer_on=1, zlmax=30.0, tpoly=20.0, qbeta=0.9, diffpoly=1000.0, gain=2.0, ugain=40.0,
                  dt=0.005)
    elif variant == "inertial":
        kw.update(particle_flag=1, npart=200, ap=0.002, ratio=2.0, gravity=0.1, cd_switch=2, c_mu=1.0)
    names = ["V", "OMY", "FN", "GN", "U0", "W0", "SCALAR", "SCN"]
    if variant == "polymer_ib":
        names += ["C11", "C12", "C22", "C33", "STR11N"]
    ctxs = []
    for prec in (0, 1):
        p = kc.cfg_small(32, 32, 32, precision=prec, **kw)
        fields = kc.initial_fields(p, amp=0.1, seed=19)
        g = rt.KmmContext(p)
        if variant == "routine_plain":
            g.call("set_option", 1, 0)
        kc.load_initial(g, p, fields, np.zeros_like(fields[0]))
        if variant == "polymer_ib":
            g.upload("IMATRIX", inputs.cylinder_imatrix(p.nx, p.ny, p.nz, p.xl, p.yl, math.pi, 0.0, 0.25))
        if variant == "inertial":
            for name, arr in zip(("XPART", "YPART", "ZPART"), inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl,
                                                                                      p.ap, 5)):
                g.upload(name, arr)
        assert g.initial() == 0
        ctxs.append(g)
    for _ in range(10):
        for g in ctxs:
            assert g.step() == 0
    worst = 0.0
    for name in names:
        e = kc.rel_err(ctxs[1].download(name), ctxs[0].download(name))
        worst = max(worst, e)
        assert e <= 1e-5, "%s rel err %.3e" % (name, e)
    assert worst > 1e-12   # the mixed form really runs in FP32
    if variant == "inertial":
        for name in ("XPART", "YPART", "VPART"):
            assert kc.rel_err(ctxs[1].download(name), ctxs[0].download(name)) <= 1e-5


@pytest.mark.parametrize("n", [64, 96, 128])
def test_polymer_ib_step_at_compiled_grids(rt, n):
    """The polymer + IB + scalar routine step (55 input fields of the x stage) at the compiled
    grids n x (n+1) x n, n = 64, 96, 128 (x-stage lengths 96, 144, 192; every kernel's shared
    memory near its largest), in both precisions: every launch succeeds and the mixed form tracks
    the FP64 drop-in within 1e-5 after 2 steps."""
    kw = dict(scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=0.5, polymer_on=1, zlmax=30.0, tpoly=20.0, qbeta=0.9,
              diffpoly=1000.0, gain=2.0, ugain=40.0, dt=0.005)
    ctxs = []
    for prec in (0, 1):
        p = kc.cfg_small(n, n, n, precision=prec, **kw)
        fields = kc.initial_fields(p, amp=0.1, seed=23)
        g = rt.KmmContext(p)
        kc.load_initial(g, p, fields, np.zeros_like(fields[0]))
        g.upload("IMATRIX", inputs.cylinder_imatrix(p.nx, p.ny, p.nz, p.xl, p.yl, math.pi, 0.0, 0.25))
        assert g.initial() == 0
        ctxs.append(g)
    for _ in range(2):
        for g in ctxs:
            assert g.step() == 0
    for name in ("V", "OMY", "U0", "SCALAR", "C11", "C12", "C22"):
        e = kc.rel_err(ctxs[1].download(name), ctxs[0].download(name))
        assert e <= 1e-5, "%s rel err %.3e" % (name, e)
    for g in ctxs:
        g.close()
