"""Python handle on libkmm_b200.so through its C ABI (include/kmm.h).

This is the host-side mirror of the reference's Fortran calls: each method has
the name of the reference subroutine it replaces and takes field names where the
Fortran routine takes arrays.  There is no CPU fallback: if the CUDA library is
missing or no GPU is visible, constructing a context raises.
"""
import ctypes
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkmm_b200.so")
_lib = None

# name -> argtypes after the context pointer
_ROUTINES = {
    "cderiv": "ii", "wallderiv": "iiiii", "gradv": "", "gradscl": "", "derivscji": "", "gfcn": "",
    "phirhs": "iiid", "solve": "idi", "penta": "ididddd", "uzero": "i", "phi_from_v": "", "influence": "",
    "veloc": "", "vort": "", "nonlin": "", "vcw3dp": "", "norm": "i", "xyzfft": "ii", "polynl": "",
    "polyforce": "", "subforce": "", "filter": "", "initial": "", "step": "", "run": "i",
    "tracer_update": "", "init_part": "", "copy": "ii", "zero": "i", "set_it": "i", "sync": "",
    "set_option": "ii", "calcswirl": "",
}
_CT = {"i": ctypes.c_int, "d": ctypes.c_double}


class KmmError(RuntimeError):
    def __init__(self, status, where, message=""):
        self.status = status
        super().__init__("%s returned %s%s" % (where, abi.STATUS_NAMES.get(status, status),
                                                (": " + message) if message else ""))


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libkmm_b200.so is missing: build it with `python -m polymer_dns_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.kmm_ctx_create.argtypes = [ctypes.POINTER(abi.KmmParams), ctypes.c_int, ctypes.POINTER(vp)]
        L.kmm_ctx_create.restype = ctypes.c_int
        L.kmm_ctx_destroy.argtypes = [vp]
        L.kmm_ctx_destroy.restype = ctypes.c_int
        L.kmm_last_error.argtypes = [vp]
        L.kmm_last_error.restype = ctypes.c_char_p
        L.kmm_abi_version.restype = ctypes.c_int
        L.kmm_field_size.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
        L.kmm_field_size.restype = ctypes.c_int
        for fn in ("kmm_upload", "kmm_download"):
            getattr(L, fn).argtypes = [vp, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
            getattr(L, fn).restype = ctypes.c_int
        L.kmm_get_stats.argtypes = [vp, ctypes.POINTER(abi.KmmStats)]
        L.kmm_get_stats.restype = ctypes.c_int
        L.kmm_set_timing.argtypes = [vp, ctypes.c_int]
        L.kmm_set_timing.restype = ctypes.c_int
        L.kmm_get_stage_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.kmm_get_stage_times.restype = ctypes.c_int
        L.kmm_launch_count.argtypes = [vp]
        L.kmm_launch_count.restype = ctypes.c_longlong
        L.kmm_event_record.argtypes = [vp, ctypes.c_int]
        L.kmm_event_record.restype = ctypes.c_int
        L.kmm_event_elapsed.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.kmm_event_elapsed.restype = ctypes.c_int
        L.kmm_ensemble_step.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.kmm_ensemble_step.restype = ctypes.c_int
        L.kmm_ensemble_run.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.kmm_ensemble_run.restype = ctypes.c_int
        L.kmm_flowstats.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.kmm_flowstats.restype = ctypes.c_int
        L.kmm_xyzfft_noalloc.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
        L.kmm_xyzfft_noalloc.restype = ctypes.c_int
        L.kmm_tracer_cells.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_size_t]
        L.kmm_tracer_cells.restype = ctypes.c_int
        L.kmm_wait_selftest.argtypes = [vp, ctypes.c_double]
        L.kmm_wait_selftest.restype = ctypes.c_int
        L.kmm_target_list.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.kmm_target_list.restype = ctypes.c_int
        L.kmm_bind_host.argtypes = [vp, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
        L.kmm_bind_host.restype = ctypes.c_int
        L.kmm_run_host.argtypes = [vp, ctypes.c_int]
        L.kmm_run_host.restype = ctypes.c_int
        for name, sig in _ROUTINES.items():
            f = getattr(L, "kmm_" + name)
            f.argtypes = [vp] + [_CT[c] for c in sig]
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def exported_symbols():
    """Names the library must export (every entry point declared in include/kmm.h)."""
    base = ["kmm_ctx_create", "kmm_ctx_destroy", "kmm_last_error", "kmm_abi_version", "kmm_field_size",
            "kmm_upload", "kmm_download", "kmm_get_stats", "kmm_set_timing", "kmm_get_stage_times",
            "kmm_launch_count", "kmm_event_record", "kmm_event_elapsed", "kmm_xyzfft_noalloc", "kmm_flowstats",
            "kmm_ensemble_step", "kmm_ensemble_run", "kmm_tracer_cells", "kmm_wait_selftest",
            "kmm_target_list", "kmm_bind_host", "kmm_run_host"]
    return base + ["kmm_" + n for n in _ROUTINES]


def xyzfft_noalloc(phys_dev_ptr, spec_dev_ptr, nx, ny, nz, stream=None):
    """kmm_xyzfft_noalloc on raw device pointers (no context, no device allocation)."""
    return lib().kmm_xyzfft_noalloc(ctypes.c_void_p(phys_dev_ptr), ctypes.c_void_p(spec_dev_ptr), int(nx), int(ny),
                                    int(nz), ctypes.c_void_p(stream) if stream else None)


def ensemble_run(ctxs, nsteps=1):
    """kmm_ensemble_run over KmmContext objects; returns the per-member status list (raises on
    argument errors only, as a member's CFL or NaN status is data for the caller)."""
    n = len(ctxs)
    arr = (ctypes.c_void_p * n)(*[c.h.value for c in ctxs])
    st = (ctypes.c_int * n)()
    rc = lib().kmm_ensemble_run(arr, n, int(nsteps), st)
    if rc == abi.ERR_ARG:
        raise KmmError(rc, "kmm_ensemble_run")
    return list(st)


class KmmContext:
    """A device context holding every field mirror of one channel run."""

    def __init__(self, params, device=0):
        self.params = params
        self.L = lib()
        self.h = ctypes.c_void_p()
        st = self.L.kmm_ctx_create(ctypes.byref(params), int(device), ctypes.byref(self.h))
        if st:
            raise KmmError(st, "kmm_ctx_create")
        self.nx, self.ny, self.nz, self.npart = params.nx, params.ny, params.nz, params.npart

    def close(self):
        if self.h:
            self.L.kmm_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _id(self, f):
        return abi.FIELD[f] if isinstance(f, str) else int(f)

    def error(self):
        m = self.L.kmm_last_error(self.h)
        return m.decode() if m else ""

    def _check(self, st, where, allow=()):
        if st and st not in allow:
            raise KmmError(st, where, self.error())
        return st

    def upload(self, f, arr):
        fid = self._id(f)
        _, dt = abi.field_kind(fid)
        a = np.asarray(arr, dtype=np.dtype(dt))
        a = np.asfortranarray(a.reshape(abi.field_shape(fid, self.nx, self.ny, self.nz, self.npart), order="F"))
        self._check(self.L.kmm_upload(self.h, fid, a.ctypes.data, a.nbytes), "kmm_upload(%s)" % f)

    def download(self, f):
        fid = self._id(f)
        _, dt = abi.field_kind(fid)
        shape = abi.field_shape(fid, self.nx, self.ny, self.nz, self.npart)
        a = np.empty(shape, dtype=np.dtype(dt), order="F")
        self._check(self.L.kmm_download(self.h, fid, a.ctypes.data, a.nbytes), "kmm_download(%s)" % f)
        return a

    def call(self, name, *args, allow=()):
        conv = [self._id(a) if isinstance(a, str) else a for a in args]
        st = getattr(self.L, "kmm_" + name)(self.h, *conv)
        return self._check(st, "kmm_" + name, allow)

    def stats(self):
        s = abi.KmmStats()
        self._check(self.L.kmm_get_stats(self.h, ctypes.byref(s)), "kmm_get_stats")
        return s

    def set_timing(self, on):
        self._check(self.L.kmm_set_timing(self.h, int(on)), "kmm_set_timing")

    def stage_times(self):
        n = 8
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int * n)()
        self._check(self.L.kmm_get_stage_times(self.h, ms, cnt, n), "kmm_get_stage_times")
        names = ["column", "dct_fwd", "zfft_bwd", "xphys", "xfwd", "zfft_fwd", "dct_bwd", "post"]
        return {names[i]: (ms[i], cnt[i]) for i in range(n)}

    def launch_count(self):
        return int(self.L.kmm_launch_count(self.h))

    def event_record(self, slot):
        self._check(self.L.kmm_event_record(self.h, slot), "kmm_event_record")

    def event_elapsed(self, a, b):
        ms = ctypes.c_double()
        self._check(self.L.kmm_event_elapsed(self.h, a, b, ctypes.byref(ms)), "kmm_event_elapsed")
        return ms.value

    def upload_ptr(self, f, ptr, nbytes):
        """Upload from a raw host pointer (e.g. pinned memory) in the reference layout."""
        fid = self._id(f)
        self._check(self.L.kmm_upload(self.h, fid, ctypes.c_void_p(ptr), nbytes), "kmm_upload(%s)" % f)

    def download_ptr(self, f, ptr, nbytes):
        fid = self._id(f)
        self._check(self.L.kmm_download(self.h, fid, ctypes.c_void_p(ptr), nbytes), "kmm_download(%s)" % f)

    def bind_host(self, f, ptr, nbytes):
        """kmm_bind_host: make the host array at `ptr` (reference layout, page-locked for
        asynchronous copies) the home of field `f` for run_host; ptr = 0 unbinds."""
        fid = self._id(f)
        self._check(self.L.kmm_bind_host(self.h, fid, ctypes.c_void_p(ptr) if ptr else None, int(nbytes)),
                    "kmm_bind_host(%s)" % f)

    def unbind_host(self):
        self._check(self.L.kmm_bind_host(self.h, -1, None, 0), "kmm_bind_host")

    def run_host(self, n, allow=()):
        """kmm_run_host: n steps with the bound fields uploaded before and downloaded after every
        step.  Returns the status (statuses in `allow` are returned, others raise)."""
        return self._check(self.L.kmm_run_host(self.h, int(n)), "kmm_run_host", allow)

    def tracer_cells(self):
        """kmm_tracer_cells: the 1-based interpolation cell (imin, jmin, kmax) of every particle,
        shape (3, npart) int32, as part_track.f90:560-577 looks it up."""
        cells = np.zeros(3 * self.npart, np.int32)
        self._check(self.L.kmm_tracer_cells(self.h, cells.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), cells.size),
                    "kmm_tracer_cells")
        return cells.reshape(3, self.npart)

    def target_list(self):
        """kmm_target_list: (n, 3) int32 1-based (x, y, z) grid indices of the last scl_flag = 4
        source's targets, in placement order."""
        buf = np.zeros(3 * 1023, np.int32)
        n = int(self.L.kmm_target_list(self.h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), buf.size))
        if n < 0:
            raise KmmError(-n, "kmm_target_list")
        return buf[:3 * n].reshape(n, 3)

    def wait_selftest(self, limit_ms):
        """kmm_wait_selftest: status of a bounded wait on a barrier nothing arrives on
        (KMM_ERR_TIMEOUT expected)."""
        return int(self.L.kmm_wait_selftest(self.h, float(limit_ms)))

    def flowstats(self):
        """(prof[7][nyp], scal[4]) of kmm_flowstats: umean, urms, vrms, wrms, R12, T12, ke profiles;
        bulk velocity, top / bottom wall shear, bulk kinetic energy."""
        prof = np.zeros((7, self.ny + 1))
        scal = np.zeros(4)
        dp = ctypes.POINTER(ctypes.c_double)
        self._check(self.L.kmm_flowstats(self.h, prof.ctypes.data_as(dp), scal.ctypes.data_as(dp)), "kmm_flowstats")
        return prof, scal

    def save_restart(self, path, c_path=None):
        """outputs/last-restart (and c-last-restart when due) of the current state, in the
        reference's unformatted record layout (main_dns.f90:775-794)."""
        from . import restart
        restart.save(self.download, self.params, self.stats().it, path, c_path)

    def load_restart(self, path, c_path=None):
        """Upload setup/restart (and setup/c-restart) before `initial` with irstrt >= 1
        (main_dns.f90:1742-1916)."""
        from . import restart
        restart.load(self.upload, self.params, path, c_path)

    # mirrors of the reference's main-program blocks
    def initial(self):
        return self.call("initial")

    def step(self):
        return self.call("step")

    def run(self, n):
        return self.call("run", n)
