"""Pins the CPU oracle with mathematical known answers (the reference ships no tests or golden data).

Covers: FFTW transform conventions (against numpy / scipy), exact Chebyshev derivatives of
polynomials, manufactured solutions of the Dirichlet and Robin tau solvers and of the mean-mode
solver, an independent numpy restatement of vcw3dp, the steady laminar Poiseuille flow, viscous
decay of a Squire mode, continuity, and exact tracer advection / trilinear interpolation.
"""
import math

import numpy as np
import pytest
import scipy.fft as sfft
from numpy.polynomial import chebyshev as C

from polymer_dns_b200 import abi, inputs
from tests import kmm_cases as kc


# ---------------------------------------------------------------- transforms
@pytest.mark.parametrize("n", [9, 17, 33, 65, 97, 129])
def test_dct1_matches_scipy_and_definition(oracle_mod, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    got = oracle_mod.dct1(x)
    np.testing.assert_allclose(got, sfft.dct(x, type=1), rtol=0, atol=1e-12 * np.abs(x).sum())
    # DCT-I applied twice is 2(n-1) times the identity
    np.testing.assert_allclose(oracle_mod.dct1(got) / (2 * (n - 1)), x, atol=1e-13)


@pytest.mark.parametrize("n", [12, 48, 96, 144, 192, 256, 576])
def test_fft_conventions(oracle_mod, n):
    rng = np.random.default_rng(n)
    z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(oracle_mod.fft(z, -1), np.fft.fft(z), atol=1e-12 * n)
    np.testing.assert_allclose(oracle_mod.fft(z, +1), np.fft.ifft(z) * n, atol=1e-12 * n)
    r = rng.standard_normal(n)
    np.testing.assert_allclose(oracle_mod.rfft(r), np.fft.rfft(r), atol=1e-12 * n)
    X = np.fft.rfft(r)
    X[0] += 3j          # c2r ignores the imaginary parts of the DC and Nyquist entries (FFTW)
    X[-1] -= 2j
    np.testing.assert_allclose(oracle_mod.irfft(X, n), r * n, atol=1e-11 * n)


# ---------------------------------------------------------------- derivatives
def _set_columns(o, name, coeffs):
    p = o.params
    a = np.zeros((p.ny + 1, p.nz, p.nx // 2), complex, order="F")
    a[:, :, :] = coeffs[:, None, None]
    o.set(name, a)


def test_cderiv_exact_on_polynomials(oracle_mod):
    p = kc.cfg_small(8, 16, 8)
    o = oracle_mod.Oracle(p)
    rng = np.random.default_rng(1)
    coef = rng.standard_normal(p.ny + 1) + 1j * rng.standard_normal(p.ny + 1)
    _set_columns(o, "WRKC", coef)
    o.call("cderiv", "WRKC", "WRK1")
    dyde = 2.0 / p.yl
    want = np.zeros(p.ny + 1, complex)
    d = C.chebder(coef) * dyde
    want[: len(d)] = d
    got = o.get("WRK1")
    np.testing.assert_allclose(got[:, 3, 2], want, atol=1e-11 * np.abs(want).max())


def test_wall_functionals(oracle_mod):
    p = kc.cfg_small(8, 16, 8)
    o = oracle_mod.Oracle(p)
    rng = np.random.default_rng(2)
    coef = rng.standard_normal(p.ny + 1)
    _set_columns(o, "WRKC", coef.astype(complex))
    dyde = 2.0 / p.yl
    for order in (0, 1, 2):
        for wall, y in ((0, -1.0), (1, 1.0)):
            o.call("wallderiv", "WRKC", order, wall, "WRK1", 3)
            got = o.get("WRK1")[2, 0, 0].real
            c = coef.copy()
            for _ in range(order):
                c = C.chebder(c) * dyde
            want = C.chebval(y, c)
            if order == 2 and wall == 0:
                # c2derbw (derivatives.f90:417-440) reuses c1derbw's sign pattern (-1)^(n+1) and so
                # returns -u''(-1); it is unused on the time-step path and kept as written
                want = -want
            assert abs(got - want) <= 1e-10 * max(1.0, abs(want)), (order, wall, got, want)


# ---------------------------------------------------------------- tau solvers
def _manufactured(p, rng):
    nyp, nz, nxh = p.ny + 1, p.nz, p.nx // 2
    dyde = 2.0 / p.yl
    alpha, beta = 2 * math.pi / p.xl, 2 * math.pi / p.zl
    wavx = np.arange(nxh) * alpha
    wavz = np.array([j * beta if j < nz // 2 else (j - nz) * beta for j in range(nz)])
    u = np.zeros((nyp, nz, nxh), complex)
    for k in range(nxh):
        for j in range(nz):
            c = (rng.standard_normal(nyp) + 1j * rng.standard_normal(nyp)) * np.exp(-0.3 * np.arange(nyp))
            u[:, j, k] = c
    return u, wavx, wavz, dyde


def _apply_op(u, wavx, wavz, dyde, g):
    f = np.zeros_like(u)
    for k in range(u.shape[2]):
        for j in range(u.shape[1]):
            c = u[:, j, k]
            d2 = np.zeros_like(c)
            dd = C.chebder(c, 2) * dyde ** 2
            d2[: len(dd)] = dd
            f[:, j, k] = d2 - (wavz[j] ** 2 + wavx[k] ** 2 + g) * c
    return f


@pytest.mark.parametrize("g", [0.0, 280000.0])
def test_solve_dirichlet_manufactured(oracle_mod, g):
    p = kc.cfg_small(8, 16, 8)
    o = oracle_mod.Oracle(p)
    rng = np.random.default_rng(3)
    u, wavx, wavz, dyde = _manufactured(p, rng)
    f = _apply_op(u, wavx, wavz, dyde, g)
    o.set("WRKC", f)
    bct = np.array([[C.chebval(1.0, u[:, j, k]) for k in range(u.shape[2])] for j in range(u.shape[1])])
    bcb = np.array([[C.chebval(-1.0, u[:, j, k]) for k in range(u.shape[2])] for j in range(u.shape[1])])
    o.set("BCTOP", bct)
    o.set("BCBOT", bcb)
    o.call("solve", "WRKC", g, 0)
    got = o.get("WRKC")
    assert kc.rel_err(got, u) < 1e-11


@pytest.mark.parametrize("at,bt,ab,bb", [(1.0, 0.0, 1.0, 0.0), (0.0, 1.0, 0.0, 1.0), (1.0, 0.3, 0.7, 0.5)])
def test_penta_robin_manufactured(oracle_mod, at, bt, ab, bb):
    p = kc.cfg_small(8, 16, 8)
    o = oracle_mod.Oracle(p)
    rng = np.random.default_rng(4)
    u, wavx, wavz, dyde = _manufactured(p, rng)
    g = 1000.0
    f = _apply_op(u, wavx, wavz, dyde, g)
    o.set("WRKC", f)
    nz, nxh = u.shape[1], u.shape[2]
    gt = np.zeros((nz, nxh), complex)
    gb = np.zeros((nz, nxh), complex)
    for k in range(nxh):
        for j in range(nz):
            c = u[:, j, k]
            d = C.chebder(c) * dyde
            gt[j, k] = at * C.chebval(1.0, c) + bt * C.chebval(1.0, d)
            # bottom row of mixedbc: (ab + dyde bb n^2)(-1)^n  ->  ab u(-1) - bb u'(-1) (outward normal)
            gb[j, k] = ab * C.chebval(-1.0, c) - bb * C.chebval(-1.0, d)
    o.set("BCTOP", gt)
    o.set("BCBOT", gb)
    o.call("penta", "WRKC", g, 0, at, bt, ab, bb)
    assert kc.rel_err(o.get("WRKC"), u) < 1e-10


def test_uzero_is_crank_nicolson_step(oracle_mod):
    """One CN/AB2 step of the mean mode: residual of the discrete equation vanishes."""
    p = kc.cfg_small(8, 32, 8)
    o = oracle_mod.Oracle(p)
    nyp = p.ny + 1
    dyde, re, dt, th = 2.0 / p.yl, p.re, p.dt, p.theta
    rng = np.random.default_rng(5)
    u0 = np.zeros(nyp)
    u0[:10] = rng.standard_normal(10)
    h = np.zeros(nyp)
    h[:8] = rng.standard_normal(8)
    hl = np.zeros(nyp)
    hl[:8] = rng.standard_normal(8)
    o.set("U0", u0)
    o.set("H1N", h)
    o.set("H1NM1", hl)
    o.call("uzero", 1)
    un = o.get("U0")
    d2 = lambda c: np.pad(C.chebder(c, 2) * dyde ** 2, (0, 2))
    lhs = d2(un) - re / (th * dt) * un
    rhs = -re * u0 / (dt * th) - re * (3 * h - hl) / (2 * th) - (1 - th) / th * d2(u0)
    assert np.abs(lhs - rhs)[: nyp - 2].max() < 1e-8 * np.abs(rhs).max()
    assert abs(C.chebval(1.0, un)) < 1e-12 and abs(C.chebval(-1.0, un)) < 1e-12   # no-slip u0


# ---------------------------------------------------------------- vcw3dp, independent numpy restatement
def _numpy_vcw3dp(p, fields, dpdx):
    """u x omega on the 3/2 grid with numpy / scipy transforms (FFTW conventions, solvers.f90:2241-3416)."""
    nyp, nz, nxh = p.ny + 1, p.nz, p.nx // 2
    ny, mx, mz, nzh = p.ny, 3 * p.nx // 2, 3 * p.nz // 2, p.nz // 2
    cw = np.ones(nyp)
    cw[0] = cw[-1] = 2.0
    jj = np.array([j if j < nzh else (mz - nz) + j for j in range(nz)])

    def to_phys(a):
        b = a * (cw / 2.0)[:, None, None]
        b = sfft.dct(b.real, type=1, axis=0) + 1j * sfft.dct(b.imag, type=1, axis=0)
        s = np.zeros((nyp, mz, mx // 2 + 1), complex)
        s[:, jj, :nxh] = b
        s = np.fft.ifft(s, axis=1) * mz
        s[:, :, 0] = s[:, :, 0].real
        return np.fft.irfft(s, n=mx, axis=2) * mx

    U = {k: to_phys(v) for k, v in fields.items()}
    h1 = U["V"] * U["OMZ"] - U["W"] * U["OMY"] - dpdx
    h2 = -U["U"] * U["OMZ"] + U["W"] * U["OMX"]
    h3 = U["U"] * U["OMY"] - U["V"] * U["OMX"]

    def to_spec(h):
        s = np.fft.rfft(h, axis=2)[:, :, :nxh]
        s = np.fft.fft(s, axis=1)[:, jj, :] / (mx * mz)
        s = (sfft.dct(s.real, type=1, axis=0) + 1j * sfft.dct(s.imag, type=1, axis=0)) / ny
        s[0] /= 2
        s[-1] /= 2
        return s

    return to_spec(h1), to_spec(h2), to_spec(h3), U


def test_vcw3dp_matches_numpy_restatement(oracle_mod):
    p = kc.cfg_small(16, 16, 12, dt=1e-5)
    o = oracle_mod.Oracle(p)
    rng = np.random.default_rng(6)
    f = {n: kc.random_spectral(rng, p) for n in ["U", "V", "W", "OMX", "OMY", "OMZ"]}
    for n, a in f.items():
        o.set(n, a)
    assert o.call("vcw3dp") == 0
    g1, g2, g3, U = _numpy_vcw3dp(p, f, o.dpdx())
    assert kc.rel_err(o.get("GN"), g1) < 1e-12
    assert kc.rel_err(o.get("FN"), g2) < 1e-12
    assert kc.rel_err(o.get("OMZ"), g3) < 1e-12
    # 3/2-grid velocity saved for the tracers, (nyp,mz,mx) layout
    assert kc.rel_err(o.get("UP3D"), U["U"]) < 1e-12
    # CFL of the reference: max (|u|/dx + |v|/dy_i + |w|/dz) dt
    y = inputs.grid_y(p.ny)
    seg = np.abs(np.diff(y))
    seg = np.concatenate([[seg[-1]], seg])
    mx, mz = 3 * p.nx // 2, 3 * p.nz // 2
    cfl = ((np.abs(U["U"]) / (p.xl / mx) + np.abs(U["V"]) / seg[:, None, None] + np.abs(U["W"]) / (p.zl / mz)) * p.dt).max()
    assert abs(o.stats().cflmax - cfl) < 1e-12 * cfl


# ---------------------------------------------------------------- whole steps
def test_laminar_poiseuille_is_steady(oracle_mod):
    p = kc.cfg_small(16, 32, 16)
    o = oracle_mod.Oracle(p)
    kc.load_initial(o, p, kc.initial_fields(p, amp=0.0))
    assert o.initial() == 0
    u0 = o.get("U0")
    assert o.run(20) == 0
    np.testing.assert_allclose(o.get("U0"), u0, atol=1e-13)
    assert np.abs(o.get("V")).max() < 1e-13 and np.abs(o.get("OMY")).max() < 1e-13


def test_squire_mode_viscous_decay(oracle_mod):
    """omega_y = -k^2 psi with psi ~ sin(pi(y+1)) cos(kx x + kz z): pure viscous decay, no mean flow."""
    p = kc.cfg_small(16, 32, 16, flow_select=2, uinf=0.0, re=100.0, dt=0.002)
    o = oracle_mod.Oracle(p)
    nyp = p.ny + 1
    y = inputs.grid_y(p.ny)
    x = np.arange(p.nx) * p.xl / p.nx
    z = np.arange(p.nz) * p.zl / p.nz
    a, b = 2 * math.pi / p.xl, 2 * math.pi / p.zl
    Y, Z, X = np.meshgrid(y, z, x, indexing="ij")
    amp = 1e-6
    sy = np.sin(math.pi * (Y + 1))
    ph = a * X + b * Z
    iu = amp * sy * (-b) * np.sin(ph)          # u = dpsi/dz
    iw = -amp * sy * (-a) * np.sin(ph)         # w = -dpsi/dx
    kc.load_initial(o, p, (np.asfortranarray(iu), np.zeros_like(iu, order="F"), np.asfortranarray(iw)))
    assert o.initial() == 0
    w0 = np.abs(o.get("OMY")[:, 1, 1]).max()
    nsteps = 100
    assert o.run(nsteps) == 0
    w1 = np.abs(o.get("OMY")[:, 1, 1]).max()
    rate = (a * a + b * b + math.pi ** 2) / p.re
    assert abs(w1 / w0 - math.exp(-rate * nsteps * p.dt)) < 2e-6


def test_continuity_preserved(oracle_mod):
    p = kc.cfg_small(16, 24, 16)
    o = oracle_mod.Oracle(p)
    kc.load_initial(o, p, kc.initial_fields(p))
    assert o.initial() == 0
    assert o.run(10) == 0
    u, w = o.get("U"), o.get("W")
    o.call("cderiv", "V", "WRKC")
    dv = o.get("WRKC")
    kx = np.arange(p.nx // 2) * 2 * math.pi / p.xl
    kz = np.fft.fftfreq(p.nz, 1.0 / p.nz) * 2 * math.pi / p.zl
    div = 1j * kx[None, None, :] * u + dv + 1j * kz[None, :, None] * w
    assert np.abs(div).max() < 1e-12 * np.abs(u).max()


# ---------------------------------------------------------------- tracers
def test_tracers_uniform_flow_and_trilinear(oracle_mod):
    p = kc.cfg_small(8, 16, 8, npart=64, ap=1e-3)
    o = oracle_mod.Oracle(p)
    mx, mz, nyp = 3 * p.nx // 2, 3 * p.nz // 2, p.ny + 1
    y = inputs.grid_y(p.ny)
    xg = np.arange(mx) * p.xl / mx
    zg = np.arange(mz) * p.zl / mz
    Y, Z, X = np.meshgrid(y, zg, xg, indexing="ij")
    # linear in y and z, constant in x: trilinear interpolation is exact away from the periodic seam
    U = 0.3 + 0.0 * X
    V = 0.05 * Y
    W = -0.2 + 0.1 * Z
    o.set("UP3D", U)
    o.set("VP3D", V)
    o.set("WP3D", W)
    rng = np.random.default_rng(7)
    xp = rng.uniform(0, p.xl, 64)
    yp = rng.uniform(-0.9, 0.9, 64)
    zp = rng.uniform(0, zg[-1] * 0.999, 64)
    for n, a in (("XPART", xp), ("YPART", yp), ("ZPART", zp)):
        o.set(n, a)
    assert o.call("init_part") == 0
    np.testing.assert_allclose(o.get("UPART"), 0.3, atol=1e-14)
    np.testing.assert_allclose(o.get("VPART"), 0.05 * yp, atol=1e-14)
    np.testing.assert_allclose(o.get("WPART"), -0.2 + 0.1 * zp, atol=1e-13)
    assert o.call("tracer_update") == 0
    np.testing.assert_allclose(o.get("XPART"), np.fmod(p.xl + xp + 0.3 * p.dt, p.xl), atol=1e-14)
    np.testing.assert_allclose(o.get("YPART"), yp + 0.05 * yp * p.dt, atol=1e-14)


def _swirl_oracle(oracle_mod, grads, p):
    """Oracle calcswirl on constant velocity gradients u_ij = grads[i][j] (spectral (0,0) mode,
    Chebyshev coefficient 0: constant in physical space)."""
    o = oracle_mod.Oracle(p)
    names = ["U11", "U12", "U13", "U21", "U22", "U23", "U31", "U32", "U33"]
    for m, name in enumerate(names):
        a = np.zeros((p.ny + 1, p.nz, p.nx // 2), dtype=np.complex128, order="F")
        a[0, 0, 0] = grads[m // 3][m % 3]
        o.set(name, a)
    assert o.call("calcswirl") == 0
    return o.get("SWIRL3D")


def test_swirl_known_answers(oracle_mod):
    """Swirl strength (helpers.f90:197-404) on uniform gradients: a solid-body rotation of rate w has
    eigenvalues 0, +-i w, so swirl = sqrt(2) w; a pure strain has real eigenvalues, swirl ~ 0; a
    rotation plus an axial strain keeps the complex pair."""
    p = kc.cfg_small(16, 16, 12)
    w = 1.7
    rot = [[0.0, -w, 0.0], [w, 0.0, 0.0], [0.0, 0.0, 0.0]]
    sw = _swirl_oracle(oracle_mod, rot, p)
    assert np.allclose(sw, math.sqrt(2.0) * w, rtol=1e-12, atol=0)
    strain = [[0.3, 0.0, 0.0], [0.0, -0.1, 0.0], [0.0, 0.0, -0.2]]
    sw = _swirl_oracle(oracle_mod, strain, p)
    assert np.abs(sw).max() < 1e-14
    # rotation w about z with strain s on z: eigenvalues s, -s/2 +- i w_eff, w_eff = sqrt(w^2 - s^2/4)... use numpy
    g = np.array([[-0.25, -w, 0.0], [w, -0.25, 0.0], [0.0, 0.0, 0.5]])
    sw = _swirl_oracle(oracle_mod, g.tolist(), p)
    lam = np.linalg.eigvals(g)
    want = math.sqrt(float(np.sum(lam.imag ** 2)))
    assert np.allclose(sw, want, rtol=1e-12, atol=0)


def test_flowstats_laminar_poiseuille(oracle_mod):
    """writeoutputs statistics (helpers.f90:1227-1438) on laminar Poiseuille u = 1.5 (1 - y^2)
    (U_b = 1): mass flux 1 up to the trapezoid error of the Gauss-Lobatto grid, no fluctuations,
    wall shear -+3/re (du/dy = -3y), kinetic energy 0.5 <u^2> = 0.6 in the bulk."""
    p = kc.cfg_small(16, 32, 12)
    o = oracle_mod.Oracle(p)
    iu, iv, iw = kc.initial_fields(p, amp=0.0)
    kc.load_initial(o, p, (iu, iv, iw))
    assert o.initial() == 0
    prof, scal = o.flowstats()
    y = np.cos(np.pi * np.arange(p.ny + 1) / p.ny)
    assert np.allclose(prof[0], 1.5 * (1 - y ** 2), atol=1e-12)
    assert np.abs(prof[1:5]).max() < 1e-12
    assert np.allclose(prof[5], -3.0 * y / p.re, atol=1e-12)
    dy = np.abs(np.diff(y))
    trap = np.sum(0.5 * (prof[0][1:] + prof[0][:-1]) * dy) / 2.0
    assert abs(scal[0] - trap) < 1e-14 and abs(scal[0] - 1.0) < 5e-3
    assert abs(scal[1] + 3.0 / p.re) < 1e-12 and abs(scal[2] - 3.0 / p.re) < 1e-12
    assert abs(scal[3] - 0.6) < 5e-3


def test_constant_flow_rate_recovers_poiseuille_gradient(oracle_mod):
    """Constant flow rate (flow_rate > 0, a variant the reference does not have) on the laminar
    Poiseuille profile with the wrong constant dPdx (twice the balance): each step's correction
    makes the driving gradient exactly the Poiseuille value -3/re (u'' = -3 for u = 1.5 (1 - y^2)),
    the profile stays steady and the trapezoid bulk velocity stays at its target."""
    re = 1400.0
    p0 = kc.cfg_small(16, 32, 12, re=re)
    o0 = oracle_mod.Oracle(p0)
    kc.load_initial(o0, p0, kc.initial_fields(p0, amp=0.0))
    assert o0.initial() == 0
    target = o0.flowstats()[1][0]          # the laminar profile's own trapezoid bulk velocity (~1)
    p = kc.cfg_small(16, 32, 12, re=re, r_tau=math.sqrt(6.0 / re) * re, flow_rate=target)
    o = oracle_mod.Oracle(p)
    kc.load_initial(o, p, kc.initial_fields(p0, amp=0.0))     # the U_b = 1 profile of the balanced case
    assert o.initial() == 0
    assert abs(o.dpdx() + 6.0 / re) < 1e-15
    u0 = o.get("U0")
    for _ in range(5):
        assert o.step() == 0
        assert abs(o.stats().dpdx + 3.0 / re) < 1e-9 * 3.0 / re   # delta from a 2e-5 change of Q ~ 1
    np.testing.assert_allclose(o.get("U0"), u0, atol=1e-12)
    assert abs(o.flowstats()[1][0] - target) < 1e-13
    # without the constraint the wrong gradient accelerates the flow
    q = kc.cfg_small(16, 32, 12, re=re, r_tau=math.sqrt(6.0 / re) * re)
    o2 = oracle_mod.Oracle(q)
    kc.load_initial(o2, q, kc.initial_fields(p0, amp=0.0))
    assert o2.initial() == 0 and o2.run(5) == 0
    assert o2.flowstats()[1][0] > target + 1e-3 * 5 * q.dt
    assert o2.stats().dpdx == o2.dpdx()


def test_tracer_cells_follow_fluid_interp_lookup(oracle_mod):
    """orc_tracer_cells is fluid_interp's lookup (part_track.f90:560-577): x, z cells by floor on
    the 3/2 grid with periodic wrap, y cell from the Chebyshev angle acos(2 y / yl)."""
    p = kc.cfg_small(16, 32, 12, npart=6, ap=1e-3)
    o = oracle_mod.Oracle(p)
    mx, mz = 3 * p.nx // 2, 3 * p.nz // 2
    dx, dz = p.xl / mx, p.zl / mz
    x = np.array([0.0, 0.5 * dx, 1.5 * dx, p.xl - 0.25 * dx, -0.5 * dx, 3.2])
    z = np.array([0.0, 0.5 * dz, 2.5 * dz, p.zl - 0.1 * dz, -0.5 * dz, 1.1])
    y = np.array([0.999, 0.5, 0.0, -0.5, -0.999, 0.123])
    for n, a in (("XPART", x), ("YPART", y), ("ZPART", z)):
        o.set(n, a)
    c = o.tracer_cells()
    np.testing.assert_array_equal(c[0], (np.floor(x / dx).astype(int) % mx) + 1)
    np.testing.assert_array_equal(c[1], (np.floor(z / dz).astype(int) % mz) + 1)
    kmax = np.floor(1 + p.ny / np.pi * np.arccos(2 * y / p.yl)).astype(int)
    np.testing.assert_array_equal(c[2], kmax)
    ycoord = np.cos(np.pi * np.arange(p.ny + 1) / p.ny)
    assert np.all(ycoord[kmax - 1] >= y) and np.all(ycoord[kmax] <= y)   # y lies in [y(kmin), y(kmax)]
