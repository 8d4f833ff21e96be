"""Inertial particles (particle_flag > 0) on the GPU: the Maxey-Riley RK4 integrator of
part_track.f90:617-1075 against the oracle and against its known answers.

Tolerances: particle positions and velocities after `initial` agree with the oracle to the
routine bar (1e-12 relative); after a few steps, the physical fields the integrator reads
(vorticity, velocity gradient, Laplacian on the 3/2 grid, the previous step's copies) and the
particles to the whole-run bar of the FP64 drop-in (1e-10 relative).
"""
import math

import numpy as np
import pytest

from polymer_dns_b200 import abi, inputs
from tests import kmm_cases as kc

pytestmark = pytest.mark.gpu

ROUTINE_TOL = 1e-12
RUN_TOL = 1e-10
PART = ("XPART", "YPART", "ZPART", "UPART", "VPART", "WPART")


@pytest.fixture(scope="module")
def rt():
    from polymer_dns_b200 import build, runtime
    build.build()
    return runtime


def _setup(ctx, p, fields, parts):
    setter = ctx.upload if hasattr(ctx, "upload") else ctx.set
    kc.load_initial(ctx, p, fields)
    for name, arr in zip(("XPART", "YPART", "ZPART"), parts):
        setter(name, arr)
    return ctx.initial()


def _get(ctx, name):
    return ctx.download(name) if hasattr(ctx, "download") else ctx.get(name)


@pytest.mark.parametrize("cd_switch,grid", [(2, (32, 32, 32)), (3, (16, 32, 24)), (1, (32, 32, 32))])
def test_inertial_matches_oracle(rt, cd_switch, grid):
    from oracle import pyoracle
    p = kc.cfg_small(*grid, particle_flag=1, npart=300, ap=0.002, ratio=2.0, gravity=0.1, cd_switch=cd_switch,
                     c_mu=1.0)
    fields = kc.initial_fields(p, amp=0.1, seed=31)
    parts = inputs.uniform_particles(p.npart, p.xl, p.yl, p.zl, p.ap, 7)
    g = rt.KmmContext(p)
    o = pyoracle.Oracle(p)
    assert _setup(g, p, fields, parts) == 0
    assert _setup(o, p, fields, parts) == 0
    for name in PART:
        e = kc.rel_err(_get(g, name), _get(o, name))
        assert e <= ROUTINE_TOL, ("initial", name, e)
    for _ in range(4):
        assert g.step() == 0
        assert o.step() == 0
    for name in ("WX3D", "WZ3D", "U12P3D", "U31P3D", "LVP3D", "UOLD", "LWNM1"):
        e = kc.rel_err(_get(g, name), _get(o, name))
        assert e <= RUN_TOL, (name, e)
    for name in PART:
        e = kc.rel_err(_get(g, name), _get(o, name))
        assert e <= RUN_TOL, (name, e)
    sg, so = g.stats(), o.stats()
    assert abs(sg.pumax - so.pumax) <= RUN_TOL * so.pumax
    assert sg.pumax > 0.0
    g.close()


def test_inertial_known_answer_stokes_settling(rt):
    """Quiescent channel, Stokes drag and gravity: the velocity approaches the terminal one by
    the RK4 factor R(-k h) per substep (the substep count of part_track.f90:296-356)."""
    g_ = 1.0
    p = kc.cfg_small(16, 16, 16, r_tau=0.0, particle_flag=1, npart=64, ap=1e-3, ratio=2.0, c_mu=1.0, gravity=g_,
                     cd_switch=1)
    pi_f, pi_p = 1.0 / (p.ratio + 0.5), p.ratio / (p.ratio + 0.5)
    tau = p.re * p.ap ** 2 / (6.0 * pi_f)
    nsub = math.ceil(max(1.0, 2.0 * p.dt / tau))
    k = pi_f * 16.0 / (2 * p.ap * p.re) * p.c_mu * 3.0 / (8.0 * p.ap)
    vinf = -g_ * (pi_f - pi_p) / k
    z = -k * p.dt / nsub
    R = 1 + z + z * z / 2 + z ** 3 / 6 + z ** 4 / 24
    zero = np.zeros((p.ny + 1, p.nz, p.nx))
    parts = (np.linspace(0.1, p.xl - 0.1, p.npart), np.linspace(-0.8, 0.8, p.npart),
             np.linspace(0.2, p.zl - 0.2, p.npart))
    with rt.KmmContext(p) as g:
        assert _setup(g, p, (zero, zero, zero), parts) == 0
        for n in range(1, 4):
            assert g.step() == 0
            np.testing.assert_allclose(g.download("VPART"), vinf * (1 - R ** (n * nsub)), rtol=1e-12, atol=0)
        assert not g.download("UPART").any()


def test_inertial_particle_cfl_stop(rt):
    p = kc.cfg_small(16, 16, 16, r_tau=0.0, particle_flag=1, npart=2, ap=1e-5, ratio=2.0, gravity=20.0, cd_switch=0,
                     dt=0.002)
    a = abs(20.0 * (1.0 / 2.5 - 2.0 / 2.5))
    zero = np.zeros((p.ny + 1, p.nz, p.nx))
    parts = (np.array([1.0, 2.0]), np.array([-0.5, -0.4]), np.array([1.0, 2.0]))
    with rt.KmmContext(p) as g:
        assert _setup(g, p, (zero, zero, zero), parts) == 0
        for n in range(1, 20):
            st = g.call("step", allow=(abi.ERR_PCFL,))
            if a * n * p.dt * p.dt / p.ap >= 10.0:
                assert st == abi.ERR_PCFL
                break
            assert st == 0
        else:
            pytest.fail("the particle CFL never reached 10")
