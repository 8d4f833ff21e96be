"""Seeded synthetic inputs for the channel workloads.

The reference builds its initial field from a laminar profile only
(init_flow.f90:82-144) and reads particles / geometry from files written by
unseeded generators (setup/particles/generator.f90:198-203, geometry/Geom.f90).
These recipes replace them with seeded host-side generators so the GPU run and
the CPU oracle start from identical physical fields:

* ``channel_initial``: mean profile (laminar Poiseuille, or a Reichardt log-law
  profile in outer units) plus a divergence-free perturbation built from random
  phase stream-function modes that vanish with their wall-normal derivative at
  both walls (no-slip), so the field is exactly representable on the grid and
  solenoidal by construction;
* ``uniform_particles``: tracer positions uniformly distributed in the box;
* ``cylinder_imatrix``: a spanwise (z-aligned) solid cylinder on the 3/2 grid
  (imatrix type 1 cells, solvers.f90:2996-3002).
"""
import math

import numpy as np


def grid_y(ny, yl=2.0):
    """ycoord(k) = cos((k-1) pi/ny) yl/2 (main_dns.f90:1112-1117)."""
    return np.cos(np.arange(ny + 1) * math.pi / ny) * (yl / 2.0)


def reichardt(yplus, kappa=0.41):
    return (1.0 / kappa) * np.log1p(kappa * yplus) + 7.8 * (1.0 - np.exp(-yplus / 11.0) - (yplus / 11.0) * np.exp(-yplus / 3.0))


def _perturbation(nx, ny, nz, xl, yl, zl, kmax, seed):
    """Divergence-free no-slip perturbation on the (nyp,nz,nx) physical grid.

    Each mode is a y-profile times a (z, x) wave, so every component is assembled as one
    matrix product (profiles: nyp x M) @ (waves: M x nz*nx)."""
    rng = np.random.default_rng(seed)
    y = grid_y(ny, yl) / (yl / 2.0)                      # in [-1, 1]
    x = np.arange(nx) * xl / nx
    z = np.arange(nz) * zl / nz
    a, b = 2 * math.pi / xl, 2 * math.pi / zl
    E2, dE2 = (1 - y ** 2) ** 2, -4 * y * (1 - y ** 2)   # psi, d psi/dy vanish at the walls
    E1 = 1 - y ** 2
    prof = {"u": [], "v": [], "w": []}
    wave = {"u": [], "v": [], "w": []}

    def add(comp, py, pw):
        prof[comp].append(py)
        wave[comp].append(pw.ravel())

    for kx in range(0, kmax + 1):
        for kz in range(-kmax, kmax + 1):
            if kx == 0 and kz <= 0:
                continue
            ph = b * kz * z[:, None] + a * kx * x[None, :]   # (nz, nx)
            for comp in range(3):
                amp = rng.standard_normal()
                phase = rng.uniform(0, 2 * math.pi)
                c0, c1 = rng.standard_normal(2) * [1.0, 0.5]
                P = c0 + c1 * y
                dP = c1
                cs, sn = np.cos(ph + phase), np.sin(ph + phase)
                if comp == 0:      # psi1(x,y,z): u = dpsi/dy, v = -dpsi/dx
                    add("u", amp * (dE2 * P + E2 * dP), cs)
                    add("v", amp * E2 * P * a * kx, sn)
                elif comp == 1:    # psi2: w = dpsi/dy, v = -dpsi/dz
                    add("w", amp * (dE2 * P + E2 * dP), cs)
                    add("v", amp * E2 * P * b * kz, sn)
                else:              # psi3: u = dpsi/dz, w = -dpsi/dx (no v)
                    add("u", -amp * E1 * P * b * kz, sn)
                    add("w", amp * E1 * P * a * kx, sn)
    out = []
    for comp in ("u", "v", "w"):
        if prof[comp]:
            f = np.stack(prof[comp], axis=1) @ np.stack(wave[comp], axis=0)
        else:
            f = np.zeros((ny + 1, nz * nx))
        out.append(f.reshape(ny + 1, nz, nx))
    return tuple(out)


def channel_initial(nx, ny, nz, xl, yl, zl, re, r_tau, profile="laminar", amp=0.05, kmax=4, seed=0):
    """Physical initial fields initu, initv, initw, each (nyp, nz, nx) float64 in Fortran order.

    profile "laminar": U = -re dPdx/2 (1-y^2) with dPdx = -2/yl (2 R_tau/(yl re))^2 (init_flow.f90:117-133);
    profile "loglaw":  U = u_tau U+(y+) (Reichardt), u_tau = R_tau/re, y+ = (1-|y|) R_tau.
    The perturbation is scaled to an rms speed of `amp` over the grid points.
    """
    y = grid_y(ny, yl) / (yl / 2.0)
    if profile == "laminar":
        dpdx = -2.0 / yl * (2.0 * r_tau / (yl * re)) ** 2
        U = -re * dpdx / 2.0 * (1.0 - y ** 2)
    elif profile == "loglaw":
        utau = r_tau / re
        U = utau * reichardt((1.0 - np.abs(y)) * r_tau)
    else:
        raise ValueError(profile)
    u, v, w = _perturbation(nx, ny, nz, xl, yl, zl, kmax, seed)
    rms = math.sqrt(float(np.mean(u * u + v * v + w * w)))
    s = amp / rms if rms > 0 else 0.0
    initu = np.asfortranarray(U[:, None, None] + s * u)
    initv = np.asfortranarray(s * v)
    initw = np.asfortranarray(s * w)
    return initu, initv, initw


def uniform_particles(npart, xl, yl, zl, ap, seed):
    """Tracer positions, uniform in [0,xl) x [-yl/2+ap, yl/2-ap] x [0,zl)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, xl, npart)
    y = rng.uniform(-yl / 2.0 + ap, yl / 2.0 - ap, npart)
    z = rng.uniform(0.0, zl, npart)
    return x, y, z


def cylinder_imatrix(nx, ny, nz, xl, yl, xc=math.pi, yc=0.0, radius=0.25):
    """imatrix (nyp, mz, mx) int32: 1 inside a z-aligned cylinder, 0 elsewhere (3/2 grid, x = (k-1) xl/mx)."""
    mx, mz = 3 * nx // 2, 3 * nz // 2
    y = grid_y(ny, yl)
    x = np.arange(mx) * xl / mx
    inside = ((x[None, :] - xc) ** 2 + (y[:, None] - yc) ** 2) <= radius ** 2     # (nyp, mx)
    im = np.zeros((ny + 1, mz, mx), dtype=np.int32, order="F")
    im[:, :, :] = inside[:, None, :].astype(np.int32)
    return im
