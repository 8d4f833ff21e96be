"""The mixed form's y (Chebyshev) transforms as 3xTF32 tcgen05 GEMMs (KMM_OPT_TC_DCT = 1) against
the same form with FP32 FFT transforms and against the FP64 drop-in.

Both mixed variants carry reduced-precision rounding in the transforms: 3xTF32 products (each
operand split into two TF32 parts, about 22 significant bits) accumulated in FP32 over the ny + 1
terms of each sum, or FP32 butterflies (log2 of the length rounding steps).  After 3 polymer + IB
+ scalar steps both stay within the mixed form's bar of 1e-5 relative of the FP64 state; the
tensor-core form is measured at about 1e-7 .. 5e-7 there, several times the FFT form's error.
"""
import numpy as np
import pytest

from polymer_dns_b200 import abi, configs
from tests import kmm_cases as kc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    from polymer_dns_b200 import build, runtime
    build.build()
    return runtime


@pytest.mark.parametrize("n", [32, 64, 96, 128])
def test_tensor_core_y_transforms_track_fp64(rt, n):
    ctxs = {}
    for name, prec, tc in (("fp64", 0, 0), ("fft", 1, 0), ("tc", 1, 1)):
        p, init, _ = configs.make("cfg3", precision=prec, grid=n, npart=500)
        f, extra = configs.build_inputs(p, init, "cfg3")
        g = rt.KmmContext(p)
        g.call("set_option", abi.OPT_TC_DCT, tc)
        configs.load(f, extra, g.upload)
        assert g.initial() == 0
        ctxs[name] = g
    for _ in range(3):
        for g in ctxs.values():
            assert g.step() == 0
    worst = 0.0
    for name in ("V", "OMY", "FN", "GN", "U0", "SCALAR", "C11", "C12", "C22", "QP12"):
        a64 = ctxs["fp64"].download(name)
        at, af = ctxs["tc"].download(name), ctxs["fft"].download(name)
        e_tc, e_fft = kc.rel_err(at, a64), kc.rel_err(af, a64)
        worst = max(worst, e_tc)
        assert e_tc <= 1e-5, "%s tc vs fp64 %.3e (fft %.3e)" % (name, e_tc, e_fft)
    assert worst > 1e-12                 # the tensor-core form really runs at reduced precision
    assert not np.array_equal(ctxs["tc"].download("V"), ctxs["fft"].download("V"))
    for g in ctxs.values():
        g.close()
