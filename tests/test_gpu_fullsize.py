"""GPU parity at the benchmarked sizes, through the C ABI, against the CPU oracle.

The workloads are built exactly as bench.py builds them (polymer_dns_b200.configs):
  - cfg2: 128 x 129 x 128, scalar with Dirichlet walls and a uniform source, 100,000 RK3 tracers,
    on the fused step with the TMA z transforms and the captured CUDA graphs (the library
    defaults), 10 steps;
  - cfg3: cfg2 + FENE-P polymer + the Goldstein force on the cylinder (spread in every plane), on
    the routine path, 10 steps;
  - cfg1: the constant-flow-rate channel at 32 x 33 x 32 on both step paths, 10 steps.
The bar of the FP64 drop-in: max relative field difference <= 1e-10 (max|gpu - oracle| / max|oracle|
per field), and the tracers' interpolation cells (part_track.f90:560-577) identical to the bit, so
every cell holds the same particles on both sides.
"""
import numpy as np
import pytest

from polymer_dns_b200 import abi, configs
from tests import kmm_cases as kc

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-10


@pytest.fixture(scope="module")
def rt():
    from polymer_dns_b200 import build, runtime
    build.build()
    return runtime


def _setup(rt, oracle_mod, name, **over):
    p, init, _ = configs.make(name, **over)
    f, extra = configs.build_inputs(p, init, name)
    g = rt.KmmContext(p)
    o = oracle_mod.Oracle(p)
    configs.load(f, extra, g.upload)
    configs.load(f, extra, o.set)
    assert g.initial() == 0
    assert o.initial() == 0
    return p, g, o


def _cmp(g, o, name, tol=RUN_TOL):
    e = kc.rel_err(g.download(name), o.get(name))
    assert e <= tol, "%s rel err %.3e > %.1e" % (name, e, tol)
    return e


def _cells_identical(g, o, p):
    cg, co = g.tracer_cells(), o.tracer_cells()
    assert cg.shape == (3, p.npart)
    assert np.array_equal(cg, co), "interpolation cells differ for %d particles" % int(np.any(cg != co, axis=0).sum())
    mx, mz = 3 * p.nx // 2, 3 * p.nz // 2
    flat = (cg[2] - 1) * (mz * mx) + (cg[1] - 1) * mx + (cg[0] - 1)
    counts = np.bincount(flat, minlength=(p.ny + 1) * mz * mx)
    assert counts.sum() == p.npart          # every particle in exactly one cell
    flat_o = (co[2] - 1) * (mz * mx) + (co[1] - 1) * mx + (co[0] - 1)
    assert np.array_equal(counts, np.bincount(flat_o, minlength=counts.size))


def test_cfg2_as_benchmarked_matches_oracle(rt, oracle_mod):
    """The headline workload on the fused / TMA / graph path: 10 steps, state and tracers."""
    p, g, o = _setup(rt, oracle_mod, "cfg2")
    assert (p.nx, p.ny, p.nz, p.npart, p.tracer_scheme) == (128, 128, 128, 100000, 1)
    _cells_identical(g, o, p)
    launches0 = g.launch_count()
    for _ in range(10):
        assert g.step() == 0
        assert o.step() == 0
    assert g.launch_count() > launches0
    for name in ("V", "OMY", "FN", "FNM1", "GN", "GNM1", "SCALAR", "SCN", "U0", "W0", "H1N", "H3N"):
        _cmp(g, o, name)
    for name in ("XPART", "YPART", "ZPART", "UPART", "VPART", "WPART"):
        _cmp(g, o, name)
    _cells_identical(g, o, p)
    assert abs(g.stats().cflmax - o.stats().cflmax) <= 1e-10 * o.stats().cflmax
    g.close()
    o.close()


def test_cfg3_routine_path_matches_oracle(rt, oracle_mod):
    """Polymer + Goldstein IB cylinder + scalar + tracers at 128 x 129 x 128 on the routine path:
    10 steps, with the IB force acting (spread in every plane)."""
    p, g, o = _setup(rt, oracle_mod, "cfg3")
    assert p.polymer_on == 1 and p.ib_spread_all == 1 and abs(p.gain - 2.0) < 1e-12 and p.ugain == 40.0
    for _ in range(10):
        assert g.step() == 0
        assert o.step() == 0
    for name in ("V", "OMY", "FN", "GN", "SCALAR", "U0", "C11", "C12", "C13", "C22", "C23", "C33", "STR11N",
                 "STR23N", "QP12", "QP33"):
        _cmp(g, o, name)
    for name in ("FXINTG", "FYINTG", "FZINTG"):
        _cmp(g, o, name)
    assert np.abs(o.get("FXINTG")).max() > 0.0
    for name in ("XPART", "YPART", "ZPART", "UPART"):
        _cmp(g, o, name)
    _cells_identical(g, o, p)
    g.close()
    o.close()


def test_ib_spread_all_drives_the_cylinder(rt, oracle_mod):
    """With the reference's spreading test the cylinder's planes (above kmaxsurf) get no force;
    ib_spread_all = 1 spreads it.  The two runs differ, and each matches the oracle."""
    states = {}
    for spread in (0, 1):
        p, g, o = _setup(rt, oracle_mod, "cfg3", grid=32, npart=500, ib_spread_all=spread)
        for _ in range(10):
            assert g.step() == 0
            assert o.step() == 0
        for name in ("V", "OMY", "FN", "GN", "C11", "FXINTG"):
            _cmp(g, o, name)
        states[spread] = g.download("V")
        g.close()
        o.close()
    assert kc.rel_err(states[1], states[0]) > 1e-6


@pytest.mark.parametrize("fused", [1, 0])
def test_constant_flow_rate_matches_oracle(rt, oracle_mod, fused):
    """cfg1 (constant flow rate, U_b = 1) on the fused and the routine step: 10 steps against the
    oracle; the trapezoid bulk velocity stays at the target and the pressure-gradient correction
    agrees."""
    p, init, _ = configs.make("cfg1")
    f, extra = configs.build_inputs(p, init, "cfg1")
    g = rt.KmmContext(p)
    g.call("set_option", abi.OPT_FUSED, fused)
    o = oracle_mod.Oracle(p)
    configs.load(f, extra, g.upload)
    configs.load(f, extra, o.set)
    assert g.initial() == 0 and o.initial() == 0
    for _ in range(10):
        assert g.step() == 0
        assert o.step() == 0
    for name in ("V", "OMY", "FN", "GN", "U0", "W0", "H1N"):
        _cmp(g, o, name)
    _, sg = g.flowstats()
    assert abs(sg[0] - p.flow_rate) <= 1e-12
    dg, do = g.stats().dpdx, o.stats().dpdx
    assert abs(dg - do) <= 1e-9 * abs(do)
    g.close()
    o.close()


def test_bounded_wait_runs_out_and_context_survives(rt, oracle_mod):
    """A bounded mbarrier wait that nothing satisfies gives up after its limit, the kernel returns
    KMM_ERR_TIMEOUT, and the same context then steps normally (and matches the oracle)."""
    p = kc.cfg_small(32, 32, 32)
    g = rt.KmmContext(p)
    o = oracle_mod.Oracle(p)
    fields = kc.initial_fields(p, amp=0.05, seed=2)
    kc.load_initial(g, p, fields)
    kc.load_initial(o, p, fields)
    assert g.initial() == 0 and o.initial() == 0
    import time
    t0 = time.perf_counter()
    assert g.wait_selftest(20.0) == abi.ERR_TIMEOUT
    assert time.perf_counter() - t0 >= 0.015
    assert g.wait_selftest(1.0) == abi.ERR_TIMEOUT
    g.call("set_option", abi.OPT_WAIT_LIMIT_MS, 500)
    with pytest.raises(rt.KmmError):
        g.call("set_option", abi.OPT_WAIT_LIMIT_MS, 10)     # below the floor: rejected
    for _ in range(3):
        assert g.step() == 0
        assert o.step() == 0
    g.call("set_option", abi.OPT_WAIT_LIMIT_MS, 2000)
    for name in ("V", "OMY", "FN", "GN"):
        _cmp(g, o, name)
    g.close()


def test_two_pass_x_stage_matches_shared_memory_form(rt):
    """The x stage through an HBM buffer of the physical inputs (used where a row of every input
    field does not fit in shared memory) evaluates the same pointwise terms as the shared-memory
    form; its c2r is the runtime block FFT instead of the compiled warp FFT, so the states agree
    to FFT rounding (1e-12 relative) after 3 polymer + IB + scalar steps."""
    p, init, _ = configs.make("cfg3", grid=32, npart=300)
    f, extra = configs.build_inputs(p, init, "cfg3")
    ctxs = []
    for big in (1, 0):
        g = rt.KmmContext(p)
        g.call("set_option", abi.OPT_XBIG, big)
        configs.load(f, extra, g.upload)
        assert g.initial() == 0
        ctxs.append(g)
    for _ in range(3):
        for g in ctxs:
            assert g.step() == 0
    for name in ("V", "OMY", "FN", "GN", "SCALAR", "C11", "C23", "QP12", "FXINTG", "XPART"):
        e = kc.rel_err(ctxs[0].download(name), ctxs[1].download(name))
        assert e <= 1e-12, "%s rel err %.3e" % (name, e)
    for g in ctxs:
        g.close()


@pytest.mark.parametrize("grid", [(384, 32, 16), (16, 256, 12), (16, 32, 384)])
def test_cfg5_lengths_match_oracle(rt, oracle_mod, grid):
    """The transform lengths of the 384 x 257 x 384 workload on small grids the oracle runs in
    seconds: mx = 576 (the two-pass x stage with 55 polymer inputs), ny = 256 (2 ny = 512 DCTs,
    the one-thread-per-column solves) and mz = 576 (the one-buffer z transforms with in-place warp
    FFTs), polymer + scalar + IB cylinder + tracers, 3 steps."""
    nx, ny, nz = grid
    p, init, _ = configs.make("cfg5", nx=nx, ny=ny, nz=nz, npart=2000, dt=0.002)
    f, extra = configs.build_inputs(p, init, "cfg5")
    g = rt.KmmContext(p)
    o = oracle_mod.Oracle(p)
    configs.load(f, extra, g.upload)
    configs.load(f, extra, o.set)
    assert g.initial() == 0 and o.initial() == 0
    for _ in range(3):
        assert g.step() == 0
        assert o.step() == 0
    for name in ("V", "OMY", "FN", "GN", "SCALAR", "C11", "C12", "C33", "QP12", "FXINTG", "XPART", "YPART"):
        _cmp(g, o, name)
    _cells_identical(g, o, p)
    g.close()
    o.close()


@pytest.mark.parametrize("grid", [(384, 32, 384), (32, 256, 32)])
def test_cfg5_lengths_mixed_matches_fp64(rt, grid):
    """The mixed form at the transform lengths of the 384 x 257 x 384 workload: FP32 576-point x
    (two-pass x stage) and z transforms, and the FP32 half-length DCT-I at ny = 256, against the FP64
    drop-in from the same inputs after 3 polymer + scalar + IB + tracer steps, 1e-5 relative in the
    state (the FP64 form itself meets the oracle at these lengths, test_cfg5_lengths_match_oracle)."""
    nx, ny, nz = grid
    ctxs = []
    for prec in (0, 1):
        p, init, _ = configs.make("cfg5", precision=prec, nx=nx, ny=ny, nz=nz, npart=2000, dt=0.002)
        f, extra = configs.build_inputs(p, init, "cfg5")
        g = rt.KmmContext(p)
        configs.load(f, extra, g.upload)
        assert g.initial() == 0
        ctxs.append(g)
    for _ in range(3):
        for g in ctxs:
            assert g.step() == 0
    for name in ("V", "OMY", "U0", "SCALAR", "C11", "C12", "C33", "FXINTG", "XPART", "YPART"):
        e = kc.rel_err(ctxs[1].download(name), ctxs[0].download(name))
        assert e <= 1e-5, "%s rel err %.3e" % (name, e)
    for g in ctxs:
        g.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_derived_inputs_match_materialised(rt, prec):
    """vcw3dp inside the routine step forming the x and z derivatives of its inputs in the z inverse
    (KMM_OPT_DERIVED_INPUTS = 1, the default: 23 y transforms with polymer and scalar) against the
    reference's sequence of materialised derivative fields (gradv, gradscl, derivscji; 55 y
    transforms): i kx, i kz commute with the y transform, so the states agree to transform rounding
    after 5 polymer + IB + scalar steps (1e-12 relative FP64; 1e-5 for the mixed form's state and
    1e-4 for its nonlinear terms, where the derivative is now taken of the FP32 plane)."""
    p, init, _ = configs.make("cfg3", precision=prec, grid=64, npart=300)
    f, extra = configs.build_inputs(p, init, "cfg3")
    ctxs = []
    for dv in (1, 0):
        g = rt.KmmContext(p)
        g.call("set_option", abi.OPT_DERIVED_INPUTS, dv)
        configs.load(f, extra, g.upload)
        assert g.initial() == 0
        ctxs.append(g)
    for _ in range(5):
        for g in ctxs:
            assert g.step() == 0
    # the state to 1e-12 (FP64) / 1e-5 (mixed); the nonlinear terms of the mixed form, formed from
    # FP32 planes either way, to 1e-4
    state = ("V", "OMY", "U0", "SCALAR", "C11", "C12", "C23", "FXINTG", "XPART")
    terms = ("FN", "GN", "SCN", "QP13", "STR22N")
    for names, tol in ((state, 1e-12 if prec == 0 else 1e-5), (terms, 1e-12 if prec == 0 else 1e-4)):
        for name in names:
            e = kc.rel_err(ctxs[0].download(name), ctxs[1].download(name))
            assert e <= tol, "%s rel err %.3e" % (name, e)
    for g in ctxs:
        g.close()
