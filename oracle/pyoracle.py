"""Python handle on the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded by tests/, the smoke check and bench.py's CPU legs; the product never
imports this module.  It wraps oracle/liborc.so (built by oracle/Makefile) with
the same routine names as the product's C-ABI so both sides are driven alike.
"""
import ctypes
import os
import subprocess

import numpy as np

from polymer_dns_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liborc.so")
_lib = None


def build(force=False):
    """Compile liborc.so from oracle/kmm_oracle.c (gcc, OpenMP)."""
    src = os.path.join(_HERE, "kmm_oracle.c")
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liborc.so"])
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_ctx_create.argtypes = [ctypes.POINTER(abi.KmmParams), ctypes.POINTER(vp)]
        L.orc_ctx_destroy.argtypes = [vp]
        L.orc_field.argtypes = [vp, i]
        L.orc_field.restype = vp
        L.orc_field_size.argtypes = [vp, i, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(i)]
        L.orc_get_stats.argtypes = [vp, ctypes.POINTER(abi.KmmStats)]
        L.orc_dpdx.argtypes = [vp]
        L.orc_dpdx.restype = d
        for name, args in [
            ("orc_copy", [vp, i, i]), ("orc_zero", [vp, i]), ("orc_set_it", [vp, i]),
            ("orc_cderiv", [vp, i, i]), ("orc_wallderiv", [vp, i, i, i, i, i]),
            ("orc_gradv", [vp]), ("orc_gradscl", [vp]), ("orc_derivscji", [vp]), ("orc_gfcn", [vp]),
            ("orc_phirhs", [vp, i, i, i, d]), ("orc_solve", [vp, i, d, i]),
            ("orc_penta", [vp, i, d, i, d, d, d, d]), ("orc_uzero", [vp, i]),
            ("orc_phi_from_v", [vp]), ("orc_influence", [vp]), ("orc_veloc", [vp]), ("orc_vort", [vp]),
            ("orc_nonlin", [vp]), ("orc_vcw3dp", [vp]), ("orc_norm", [vp, i]), ("orc_xyzfft", [vp, i, i]),
            ("orc_polynl", [vp]), ("orc_polyforce", [vp]), ("orc_subforce", [vp]), ("orc_filter", [vp]),
            ("orc_initial", [vp]), ("orc_step", [vp]), ("orc_run", [vp, i]),
            ("orc_tracer_update", [vp]), ("orc_init_part", [vp]), ("orc_calcswirl", [vp]),
        ]:
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = i
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_flowstats.argtypes = [vp, dp, dp]
        L.orc_flowstats.restype = i
        L.orc_tracer_cells.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_size_t]
        L.orc_tracer_cells.restype = i
        L.orc_target_list.argtypes = [vp, ctypes.POINTER(ctypes.c_int), i]
        L.orc_target_list.restype = i
        L.orc_set_threads.argtypes = [i]
        L.orc_set_threads.restype = i
        L.orc_dct1.argtypes = [i, dp, dp]
        L.orc_fft.argtypes = [i, dp, dp, i]
        L.orc_rfft.argtypes = [i, dp, dp]
        L.orc_irfft.argtypes = [i, dp, dp]
        _lib = L
    return _lib


def set_threads(n):
    """OpenMP threads of the oracle's parallel loops (n <= 0: all host cores); returns the count."""
    return int(lib().orc_set_threads(int(n)))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def dct1(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lib().orc_dct1(len(x), _dp(x), _dp(out))
    return out


def fft(x, sign=-1):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().orc_fft(len(x), _dp(x.view(np.float64)), _dp(out.view(np.float64)), sign)
    return out


def rfft(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(len(x) // 2 + 1, np.complex128)
    lib().orc_rfft(len(x), _dp(x), _dp(out.view(np.float64)))
    return out


def irfft(X, n):
    X = np.ascontiguousarray(X, dtype=np.complex128)
    out = np.empty(n, np.float64)
    lib().orc_irfft(n, _dp(X.view(np.float64)), _dp(out))
    return out


class Oracle:
    """One oracle context: host-resident fields in the reference's Fortran layout."""

    def __init__(self, params):
        self.params = params
        self.L = lib()
        self.h = ctypes.c_void_p()
        st = self.L.orc_ctx_create(ctypes.byref(params), ctypes.byref(self.h))
        if st:
            raise RuntimeError("orc_ctx_create failed: %s" % abi.STATUS_NAMES.get(st, st))
        self.nx, self.ny, self.nz, self.npart = params.nx, params.ny, params.nz, params.npart

    def close(self):
        if self.h:
            self.L.orc_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _id(self, f):
        return abi.FIELD[f] if isinstance(f, str) else int(f)

    def field(self, f):
        """numpy view (Fortran order) of the oracle's storage for field f."""
        fid = self._id(f)
        n = ctypes.c_size_t()
        eb = ctypes.c_int()
        if self.L.orc_field_size(self.h, fid, ctypes.byref(n), ctypes.byref(eb)):
            raise KeyError(f)
        ptr = self.L.orc_field(self.h, fid)
        kind, dt = abi.field_kind(fid)
        shape = abi.field_shape(fid, self.nx, self.ny, self.nz, self.npart)
        nbytes = n.value * eb.value
        buf = (ctypes.c_char * nbytes).from_address(ptr)
        arr = np.frombuffer(buf, dtype=np.dtype(dt))
        return arr.reshape(shape, order="F")

    def get(self, f):
        return self.field(f).copy(order="F")

    def set(self, f, value):
        dst = self.field(f)
        dst[...] = np.asarray(value).reshape(dst.shape, order="F") if np.ndim(value) else value

    def call(self, name, *args):
        fn = getattr(self.L, "orc_" + name)
        conv = [self._id(a) if isinstance(a, str) else a for a in args]
        return fn(self.h, *conv)

    def stats(self):
        s = abi.KmmStats()
        self.L.orc_get_stats(self.h, ctypes.byref(s))
        return s

    def dpdx(self):
        return self.L.orc_dpdx(self.h)

    def tracer_cells(self):
        """orc_tracer_cells: (3, npart) int32 1-based interpolation cells (imin, jmin, kmax)."""
        cells = np.zeros(3 * self.npart, np.int32)
        st = self.L.orc_tracer_cells(self.h, cells.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), cells.size)
        if st:
            raise RuntimeError("orc_tracer_cells returned %d" % st)
        return cells.reshape(3, self.npart)

    def target_list(self):
        """orc_target_list: (n, 3) int32 1-based (x, y, z) grid indices of the last scl_flag = 4
        source's targets, in placement order."""
        buf = np.zeros(3 * 1023, np.int32)
        n = self.L.orc_target_list(self.h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), buf.size)
        if n < 0:
            raise RuntimeError("orc_target_list returned %d" % n)
        return buf[:3 * n].reshape(n, 3)

    def flowstats(self):
        """(prof[7][nyp], scal[4]) of orc_flowstats: umean, urms, vrms, wrms, R12, T12, ke profiles;
        massflux, top / bottom wall shear, bulk kinetic energy."""
        prof = np.zeros((7, self.ny + 1))
        scal = np.zeros(4)
        st = self.L.orc_flowstats(self.h, _dp(prof), _dp(scal))
        if st:
            raise RuntimeError("orc_flowstats returned %d" % st)
        return prof, scal

    # convenience mirrors of the kmm_* entry points
    def initial(self):
        return self.call("initial")

    def step(self):
        return self.call("step")

    def run(self, n):
        return self.call("run", n)
