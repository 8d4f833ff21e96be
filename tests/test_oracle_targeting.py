"""The oracle's targeted scalar sources (solvers.f90:2164-2206) against an independent numpy
restatement on a small grid:
  - scl_flag = 5 (newtarget, helpers.f90:957-1222): the source is the swirl strength scaled to [0, 1]
    by its maximum and then to a volume integral of spts;
  - scl_flag = 4 (findmaxQ, helpers.f90:678-953): the interior local maxima of the Q criterion
    (calcQ, helpers.f90:1519-1552), the first qn of them in the reference's loop order (x outer,
    z, y inner), sorted by -Q; Gaussians of widths sigma at those with beta = exp(-alpha_poly |c|)
    above 0.8, at most 1023.
The numpy side takes its own 3/2-grid transforms (scipy DCT-I, numpy FFTs with FFTW's conventions).
"""
import numpy as np
import pytest
import scipy.fft as sfft

from polymer_dns_b200 import inputs
from tests import kmm_cases as kc

GRADS = ["U11", "U12", "U13", "U21", "U22", "U23", "U31", "U32", "U33"]


def _to_phys(p, a):
    """Spectral (nyp, nz, nxh) -> physical values on the 3/2 grid (nyp, mz, mx), as vcw3dp."""
    nyp, nz, nxh = p.ny + 1, p.nz, p.nx // 2
    mx, mz, nzh = 3 * p.nx // 2, 3 * p.nz // 2, p.nz // 2
    cw = np.ones(nyp)
    cw[0] = cw[-1] = 2.0
    jj = np.array([j if j < nzh else (mz - nz) + j for j in range(nz)])
    b = a * (cw / 2.0)[:, None, None]
    b = sfft.dct(b.real, type=1, axis=0) + 1j * sfft.dct(b.imag, type=1, axis=0)
    s = np.zeros((nyp, mz, mx // 2 + 1), complex)
    s[:, jj, :nxh] = b
    s = np.fft.ifft(s, axis=1) * mz
    s[:, :, 0] = s[:, :, 0].real
    return np.fft.irfft(s, n=mx, axis=2) * mx


def _setup(oracle_mod, flag, seed, **kw):
    p = kc.cfg_small(16, 16, 12, dt=1e-6, scalar_on=1, scl_flag=flag, src_start=0, src_stop=100, **kw)
    o = oracle_mod.Oracle(p)
    rng = np.random.default_rng(seed)
    f = {n: kc.random_spectral(rng, p) for n in GRADS + ["U", "V", "W", "OMX", "OMY", "OMZ", "SCALAR"]}
    for n, a in f.items():
        o.set(n, a)
    return p, o, f


def _ly(y):
    nyp = len(y)
    ly = np.empty(nyp)
    ly[0] = abs(y[1] - y[0]) / 2.0
    ly[-1] = abs(y[-1] - y[-2]) / 2.0
    ly[1:-1] = np.abs(y[2:] - y[1:-1]) / 2.0 + np.abs(y[1:-1] - y[:-2]) / 2.0
    return ly


def test_newtarget_is_normalised_swirl(oracle_mod):
    """The source against the oracle's calcswirl (pinned by its own known answers) to rounding, and
    against numpy's eigenvalues to the closed form's conditioning (the Cardano expression of eig,
    helpers.f90:197-275, loses digits where two eigenvalues nearly coincide); its volume integral
    is spts."""
    p, o, f = _setup(oracle_mod, 5, 21, spts=2.5)
    assert o.call("vcw3dp") == 0
    sc = o.get("SCSOURCE")
    y = inputs.grid_y(p.ny)
    mx, mz = 3 * p.nx // 2, 3 * p.nz // 2
    vol = (p.xl / mx) * (p.zl / mz) * _ly(y)[:, None, None]
    assert o.call("calcswirl") == 0
    sw = o.get("SWIRL3D")
    want = sw / sw.max()
    want = want * (p.spts / np.sum(want * vol))
    assert kc.rel_err(sc, want) < 1e-13
    assert abs(np.sum(sc * vol) - p.spts) < 1e-12 * p.spts
    # swirl strength: the imaginary parts of the gradient tensor's eigenvalues (helpers.f90:339-404)
    g = [_to_phys(p, f[n]) for n in GRADS]
    lam = np.linalg.eigvals(np.stack(g, axis=-1).reshape(-1, 3, 3))
    swn = np.sqrt(np.sum(lam.imag ** 2, axis=1)).reshape(sc.shape)
    wn = swn / swn.max()
    wn = wn * (p.spts / np.sum(wn * vol))
    assert kc.rel_err(sc, wn) < 1e-4


def _numpy_findmaxq(p, f):
    """Targets and source of scl_flag = 4 restated with numpy."""
    nyp, ny = p.ny + 1, p.ny
    mx, mz = 3 * p.nx // 2, 3 * p.nz // 2
    g = [_to_phys(p, f[n]) for n in GRADS]
    u11, u12, u13, u21, u22, u23, u31, u32, u33 = g
    q = 0.5 * (-2.0 * (u12 * u21 + u13 * u31 + u23 * u32) - (u11 ** 2 + u22 ** 2 + u33 ** 2))
    nq = -q
    beta = np.exp(-p.alpha_poly * np.abs(_to_phys(p, f["SCALAR"])))
    # interior strict minima of -Q below zero, in the loop order x outer, z, y inner (0-based here)
    c = nq[1:ny, 1:mz - 1, 1:mx - 1]
    m = (c < 0)
    for ax in range(3):
        for sh in (1, -1):
            m &= c < np.roll(nq, sh, axis=ax)[1:ny, 1:mz - 1, 1:mx - 1]
    iy, iz, ix = np.nonzero(m)
    iy, iz, ix = iy + 1, iz + 1, ix + 1
    order = np.lexsort((iy, iz, ix))[:32768]          # x slowest, y fastest
    iy, iz, ix = iy[order], iz[order], ix[order]
    vals = nq[iy, iz, ix]
    srt = np.argsort(vals, kind="stable")              # no ties among these values
    targets = []
    for n in srt:
        if len(targets) == 1023:
            break
        if beta[iy[n], iz[n], ix[n]] > 0.8:
            targets.append((ix[n] + 1, iy[n] + 1, iz[n] + 1))   # 1-based x, y, z
    y = inputs.grid_y(p.ny)
    dx, dz = p.xl / mx, p.zl / mz
    X = (np.arange(mx) * dx)[None, None, :]
    Z = (np.arange(mz) * dz)[None, :, None]
    Y = y[:, None, None]
    sc = np.zeros((nyp, mz, mx))
    for kk, ii, jj in targets:
        bx = (X - dx * (kk - 1)) ** 2 / (2.0 * p.sigmax ** 2)
        bz = (Z - dz * (jj - 1)) ** 2 / (2.0 * p.sigmaz ** 2)
        by = (Y - y[ii - 1]) ** 2 / (2.0 * p.sigmay ** 2)
        tot = bx + by + bz
        ok = (bx < 18.0) & (bx + bz < 18.0) & (tot < 18.0)
        sc += np.where(ok, p.deltat * np.exp(-tot), 0.0)
    return np.array(targets, dtype=np.int32).reshape(-1, 3), sc


def test_findmaxq_targets_and_source(oracle_mod):
    p, o, f = _setup(oracle_mod, 4, 22, alpha_poly=0.4, sigmax=0.6, sigmay=0.2, sigmaz=0.3, deltat=0.7)
    assert o.call("vcw3dp") == 0
    tg = o.target_list()
    want, sc = _numpy_findmaxq(p, f)
    assert 0 < len(want) < 1023   # some targets placed, some candidates rejected by beta
    assert np.array_equal(tg, want)
    assert kc.rel_err(o.get("SCSOURCE"), sc) < 1e-12


def test_findmaxq_caps_at_1023_targets(oracle_mod):
    """Every beta above 0.8 (alpha_poly = 0) and more minima than targets: 1023 are placed."""
    p = kc.cfg_small(48, 32, 48, dt=1e-6, scalar_on=1, scl_flag=4, src_start=0, src_stop=100, alpha_poly=0.0,
                     sigmax=0.05, sigmay=0.05, sigmaz=0.05, deltat=1.0)
    o = oracle_mod.Oracle(p)
    rng = np.random.default_rng(23)
    for n in GRADS:
        a = rng.standard_normal((p.ny + 1, p.nz, p.nx // 2)) + 1j * rng.standard_normal((p.ny + 1, p.nz, p.nx // 2))
        a[:, p.nz // 2, :] = 0.0
        a[:, 0, 0] = a[:, 0, 0].real
        for j in range(1, p.nz // 2):
            a[:, p.nz - j, 0] = np.conj(a[:, j, 0])
        o.set(n, np.asfortranarray(a))
    assert o.call("vcw3dp") == 0
    assert len(o.target_list()) == 1023


def test_source_zero_outside_window(oracle_mod):
    p, o, f = _setup(oracle_mod, 5, 24, spts=1.0)
    o2 = oracle_mod.Oracle(kc.cfg_small(16, 16, 12, dt=1e-6, scalar_on=1, scl_flag=5, src_start=5, src_stop=9,
                                        spts=1.0))
    for n, a in f.items():
        o2.set(n, a)
    assert o2.call("vcw3dp") == 0
    assert np.abs(o2.get("SCSOURCE")).max() == 0.0
