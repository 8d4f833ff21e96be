"""Inertial particles (particle_flag > 0) in the oracle: known answers of the Maxey-Riley RK4
integrator of part_track.f90:617-1075.

In a quiescent channel (zero velocity, zero pressure gradient) every fluid term vanishes, so a
particle obeys dv/dt = -k v + a with a = -gravity (Pi_f - Pi_p) and k = Pi_f C_D 3/(8 ap)
(Stokes drag, CD_switch = 1) or k = 0 (CD_switch = 0).  RK4 is exact for a constant
acceleration and multiplies the deviation from the terminal velocity by R(-k h) = 1 - kh +
(kh)^2/2 - (kh)^3/6 + (kh)^4/24 per substep h = dt/substep otherwise.  These pin the stage
structure, the substep count (part_track.f90:296-356), the wall clamp and elastic bounce
(part_track.f90:728-738), the running maximum umax1 and the particle CFL stop
(part_track.f90:213-222).
"""
import math

import numpy as np
import pytest

from oracle import pyoracle
from polymer_dns_b200 import abi
from tests import kmm_cases as kc


def _quiescent(npart, **kw):
    base = dict(r_tau=0.0, particle_flag=1, npart=npart, ap=1e-3, ratio=2.0, c_mu=1.0)
    base.update(kw)
    return kc.cfg_small(16, 16, 16, **base)


def _start(p, y):
    o = pyoracle.Oracle(p)
    z = np.zeros((p.ny + 1, p.nz, p.nx))
    kc.load_initial(o, p, (z, z, z))
    n = p.npart
    o.set("XPART", np.linspace(0.1, p.xl - 0.1, n))
    o.set("YPART", np.asarray(y, dtype=float))
    o.set("ZPART", np.linspace(0.2, p.zl - 0.2, n))
    st = o.initial()
    return o, st


def test_constant_acceleration_is_exact_and_bounces():
    g = 0.5
    p = _quiescent(4, gravity=g, cd_switch=0)
    pi_f, pi_p = 1.0 / (p.ratio + 0.5), p.ratio / (p.ratio + 0.5)
    a = -g * (pi_f - pi_p)                       # ratio 2: a = +0.2 (towards the top wall)
    ybot = p.ap - 1.0
    height = 1.0 - p.ap
    y0 = np.array([-0.5, 0.0, 0.3, height - 2e-4])
    o, st = _start(p, y0)
    assert st == 0
    assert np.all(o.get("VPART") == 0.0)         # init_part: the fluid's velocity
    x0, z0 = o.get("XPART"), o.get("ZPART")
    dt = p.dt
    bounced = False
    for n in range(1, 6):
        assert o.step() == 0
        y, v = o.get("YPART"), o.get("VPART")
        t = n * dt
        for j in range(3):
            assert abs(y[j] - (y0[j] + 0.5 * a * t * t)) <= 1e-13, (n, j)
            assert abs(v[j] - a * t) <= 1e-13, (n, j)
        # the last particle reaches the top wall: clamped to Height, v reverses there
        if y[3] == height:
            assert v[3] < 0.0
            bounced = True
        np.testing.assert_allclose(o.get("XPART"), x0, rtol=0, atol=1e-14)
        np.testing.assert_allclose(o.get("ZPART"), z0, rtol=0, atol=1e-14)
        assert not o.get("UPART").any() and not o.get("WPART").any()
    assert bounced
    assert ybot < y.min()


def test_stokes_drag_terminal_approach_with_substeps():
    g = 1.0
    p = _quiescent(3, gravity=g, cd_switch=1, ap=1e-3, ratio=2.0, re=1400.0, dt=0.01)
    pi_f, pi_p = 1.0 / (p.ratio + 0.5), p.ratio / (p.ratio + 0.5)
    tau = p.re * p.ap ** 2 / (6.0 * pi_f)
    nsub = math.ceil(max(1.0, 2.0 * p.dt / tau))
    assert nsub > 1
    c_d = 16.0 / (2 * p.ap * p.re) * p.c_mu
    k = pi_f * c_d * 3.0 / (8.0 * p.ap)
    a = -g * (pi_f - pi_p)
    vinf = a / k
    h = p.dt / nsub
    z = -k * h
    R = 1 + z + z * z / 2 + z ** 3 / 6 + z ** 4 / 24
    o, st = _start(p, [-0.2, 0.0, 0.2])
    assert st == 0
    vmax = 0.0
    for n in range(1, 4):
        assert o.step() == 0
        v = o.get("VPART")
        want = vinf + (0.0 - vinf) * R ** (n * nsub)
        np.testing.assert_allclose(v, want, rtol=1e-12, atol=0)
        vmax = max(vmax, abs(want))
        s = o.stats()
        assert abs(s.pumax - vmax) <= 1e-12 * vmax
        assert abs(s.pcfl - vmax * p.dt / p.ap) <= 1e-12 * s.pcfl


def test_particle_cfl_stop():
    """p_cfl = umax1 dt / ap >= 10 stops the reference (part_track.f90:217-221); umax1 is the
    running maximum over every earlier update."""
    g = 20.0
    p = _quiescent(2, gravity=g, cd_switch=0, ap=1e-5, dt=0.002)
    pi_f, pi_p = 1.0 / (p.ratio + 0.5), p.ratio / (p.ratio + 0.5)
    a = abs(g * (pi_f - pi_p))
    o, st = _start(p, [-0.5, -0.4])
    assert st == 0
    for n in range(1, 20):
        st = o.step()
        pcfl = a * n * p.dt * p.dt / p.ap
        if pcfl >= 10.0:
            assert st == abi.ERR_PCFL
            break
        assert st == 0, n
    else:
        pytest.fail("the particle CFL never reached 10")


def test_tracers_untouched_by_inertial_fields():
    """particle_flag = 0 keeps the tracer path: tracers follow the fluid, so gravity and drag
    play no part."""
    p = _quiescent(2, particle_flag=0, gravity=1.0)
    o, st = _start(p, [-0.2, 0.2])
    assert st == 0
    assert o.step() == 0
    assert not o.get("VPART").any()
