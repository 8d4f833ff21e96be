"""Shared cases for the parity tests: seeded inputs at sizes the oracle finishes in seconds."""
import math

import numpy as np

from polymer_dns_b200 import abi, inputs

SPECTRAL_STATE = ["V", "OMY", "FN", "FNM1", "GN", "GNM1", "U", "W", "OMX", "OMZ"]
MEAN_STATE = ["U0", "W0", "H1N", "H1NM1", "H3N", "H3NM1"]


def cfg_small(nx=32, ny=32, nz=32, **kw):
    """The laminar-plus-perturbation channel (Re_bulk 2800 on 2h: re = 1400, U_b = 1)."""
    re = kw.pop("re", 1400.0)
    r_tau = kw.pop("r_tau", math.sqrt(3.0 / re) * re)   # dPdx = -3/re keeps the laminar U_b = 1 steady
    base = dict(nx=nx, ny=ny, nz=nz, dt=0.01, re=re, r_tau=r_tau, xl=4 * math.pi, zl=2 * math.pi, yl=2.0,
                flow_select=1, theta=0.5)
    base.update(kw)
    return abi.default_params(**base)


def initial_fields(p, profile="laminar", amp=0.05, kmax=4, seed=0):
    return inputs.channel_initial(p.nx, p.ny, p.nz, p.xl, p.yl, p.zl, p.re, p.r_tau, profile, amp, kmax, seed)


def load_initial(ctx, p, fields, scalar=None):
    iu, iv, iw = fields
    setter = ctx.upload if hasattr(ctx, "upload") else ctx.set
    setter("INITU", iu)
    setter("INITV", iv)
    setter("INITW", iw)
    if scalar is not None:
        setter("INITSCL", scalar)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def random_spectral(rng, p, hermitian=True):
    """Random spectral field (nyp,nz,nxh) with the reference's symmetries (norm-consistent)."""
    nyp, nz, nxh = p.ny + 1, p.nz, p.nx // 2
    a = rng.standard_normal((nyp, nz, nxh)) + 1j * rng.standard_normal((nyp, nz, nxh))
    # decay with mode number so derivatives stay O(1)
    ky = np.arange(nyp)[:, None, None]
    kz = np.minimum(np.arange(nz), nz - np.arange(nz))[None, :, None]
    kx = np.arange(nxh)[None, None, :]
    a *= np.exp(-0.15 * ky - 0.2 * kz - 0.2 * kx)
    if hermitian:
        a[:, 0, 0] = a[:, 0, 0].real
        for j in range(1, nz // 2):
            a[:, nz - j, 0] = np.conj(a[:, j, 0])
        a[:, nz // 2, :] = 0.0
    return np.asfortranarray(a)
