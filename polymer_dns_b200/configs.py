"""The named workloads: run parameters and seeded synthetic inputs.

    cfg1  32 x 33 x 32 channel, Lx = 4 pi, Lz = 2 pi, dt = 0.01, Re_bulk = 2800 (re = 1400, U_b = 1),
          constant flow rate, laminar Poiseuille + divergence-free perturbation of amplitude 0.05
          from random-phase modes |kx|, |kz| <= 4 (seed 0).
    cfg2  the Re_tau = 180 channel on 128 x 129 x 128 (Lx = 4 pi, Lz = 4 pi / 3, dt = 0.005,
          re = 2800 so U_b ~ 1 in outer units, dPdx = -(Re_tau / re)^2): log-law mean + 10 % rms
          divergence-free noise (seed 1), passive scalar (Sc = 1, uniform source, Dirichlet walls),
          100,000 tracers (seed 2, RK3).
    cfg3  cfg2 + FENE-P polymer (Wi = 20, beta = 0.9, L^2 = 900, artificial diffusivity 1e-3) + the
          Goldstein feedback force (alpha = -400, beta = -40) on a spanwise cylinder of radius 0.25
          at x = pi, y = 0.
    cfg5  the Re_tau = 395 channel on 384 x 257 x 384 (Lx = 2 pi, Lz = pi, dt = 0.002, re = Re_b / 2 from
          Dean's correlation Re_tau = 0.09 Re_b^0.88, so U_b ~ 1), polymer + scalar + IB cylinder +
          1,000,000 tracers (seed 3).

Unit mapping to the reference's dns.config values (main_dns.f90:934-1068):
  - re = 1 / nu with the half-height h = 1 (yl = 2); dPdx = -(Re_tau / re)^2 (init_flow.f90:117).
  - Goldstein alpha, beta -> gain = -alpha dt, ugain = -beta.  The feedback force is
    f = alpha int_0^t u dt' + beta u; the reference accumulates the integral as a plain running sum
    fxintg += u (no dt) and applies drag = -ugain u - gain fxintg (solvers.f90:2996-3001), so
    int u dt' = dt fxintg gives gain = -alpha dt (= 2 at dt = 0.005) and ugain = -beta (= 40).
    Reading gain = -alpha = 400 instead makes the feedback loop of the explicit (AB2) step unstable:
    the amplification factor of u_(n+1) = u_n + dt (3/2 f_n - 1/2 f_(n-1)), f_n = -ugain u_n -
    gain S_n, S_n = S_(n-1) + u_n, has modulus 1.59 at dt = 0.005 (0.92 with gain = 2), and the
    128 x 129 x 128 run leaves CFL 1 within four steps.
  - FENE-P: zlmax = L = 30, qbeta = beta, tpoly = Wi (code time units), ipeter = 1 (FENE-P), and
    diffpoly such that the conformation diffusivity 1 / (re diffpoly) is the stated 1e-3.
  - The cylinder's solid y-planes lie above the reference's spreading limit kmaxsurf (an x index,
    main_dns.f90:1526-1535, applied at solvers.f90:3069), so with the reference's test the
    cylinder receives no force; cfg3 / cfg5 set ib_spread_all = 1 so the Goldstein force acts.
Inputs are synthetic and seeded; no public dataset is involved.
"""
import math

import numpy as np

from . import abi, inputs

NAMES = ("cfg1", "cfg2", "cfg3", "cfg5")


def make(name, precision=0, grid=None, **overrides):
    """(params, init-recipe, description) of a named workload.  grid = N runs the cfg2 / cfg3 workload
    at N x (N+1) x N (small cases for profiles and oracle comparisons)."""
    if name == "cfg1":
        re = 1400.0
        kw = dict(nx=32, ny=32, nz=32, dt=0.01, re=re, r_tau=math.sqrt(3 * re), xl=4 * math.pi, zl=2 * math.pi,
                  flow_rate=1.0, precision=precision)
        init = dict(profile="laminar", amp=0.05, kmax=4, seed=0)
        desc = "cfg1 32x33x32 laminar+perturbation, constant flow rate (U_b = 1), 100-step case"
    elif name in ("cfg2", "cfg3"):
        re, r_tau = 2800.0, 180.0
        kw = dict(nx=128, ny=128, nz=128, dt=0.005, re=re, r_tau=r_tau, xl=4 * math.pi, zl=4 * math.pi / 3,
                  scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=1.0, npart=100000, ap=1e-3, tracer_scheme=1,
                  precision=precision)
        desc = "Re_tau=180 channel 128x129x128, scalar (Sc=1, uniform source, Dirichlet walls), 100k RK3 tracers"
        if name == "cfg3":
            kw.update(polymer_on=1, zlmax=30.0, tpoly=20.0, qbeta=0.9, diffpoly=1.0 / (re * 1e-3),
                      gain=400.0 * kw["dt"], ugain=40.0, ib_spread_all=1)
            desc += (", FENE-P (Wi=20, beta=0.9, L^2=900, diffusivity 1e-3), Goldstein IB (alpha=-400, beta=-40) on a "
                     "cylinder r=0.25 at (pi,0)")
        if grid:
            kw.update(nx=grid, ny=grid, nz=grid)
            desc = desc.replace("128x129x128", "%dx%dx%d" % (grid, grid + 1, grid))
        init = dict(profile="loglaw", amp=0.1, kmax=8, seed=1)
    elif name == "cfg5":
        r_tau = 395.0
        re = 10 ** (math.log10(r_tau / 0.09) / 0.88) / 2.0   # Dean: Re_tau = 0.09 Re_b^0.88; re = Re_b / 2
        kw = dict(nx=384, ny=256, nz=384, dt=0.002, re=re, r_tau=r_tau, xl=2 * math.pi, zl=math.pi,
                  scalar_on=1, diff=1.0, scalar_bc=1, scalar_q=1.0, npart=1000000, ap=1e-3, tracer_scheme=1,
                  polymer_on=1, zlmax=30.0, tpoly=20.0, qbeta=0.9, diffpoly=1.0 / (re * 1e-3), gain=400.0 * 0.002,
                  ugain=40.0, ib_spread_all=1, precision=precision)
        init = dict(profile="loglaw", amp=0.1, kmax=8, seed=3)
        desc = ("Re_tau=395 channel 384x257x384, scalar, 1M RK3 tracers, FENE-P (Wi=20, beta=0.9, L^2=900), "
                "Goldstein IB cylinder r=0.25 at (pi,0)")
    else:
        raise ValueError("unknown workload %s" % name)
    kw.update(overrides)
    return abi.default_params(**kw), init, desc


def build_inputs(p, init, name, particle_seed=None):
    """(initial u, v, w physical fields, dict of the other uploads) for a workload: the initial
    scalar (zero), the seeded uniform tracers, and the cylinder imatrix of cfg3 / cfg5."""
    f = inputs.channel_initial(p.nx, p.ny, p.nz, p.xl, p.yl, p.zl, p.re, p.r_tau, init["profile"], init["amp"],
                               init["kmax"], init["seed"])
    extra = {}
    if p.scalar_on:
        extra["INITSCL"] = np.zeros_like(f[0])
    if p.npart > 0:
        seed = particle_seed if particle_seed is not None else (3 if name == "cfg5" else 2)
        x, y, z = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, seed)
        extra.update(XPART=x, YPART=y, ZPART=z)
    if name in ("cfg3", "cfg5"):
        extra["IMATRIX"] = inputs.cylinder_imatrix(p.nx, p.ny, p.nz, p.xl, p.yl, math.pi, 0.0, 0.25)
    return f, extra


def load(f, extra, setter):
    """Upload / set the initial fields and extras through `setter(name, array)`."""
    setter("INITU", f[0])
    setter("INITV", f[1])
    setter("INITW", f[2])
    for k, v in extra.items():
        setter(k, v)
