"""ctypes mirror of include/kmm.h: the run-parameter struct, field ids and status codes.

The struct members follow the order in which ``setstuff`` reads dns.config
(FFTW_DNS/code/src/dns/main_dns.f90:934-1068).  tests/test_abi_header.py checks
that this module and the header agree.
"""
import ctypes

KMM_ABI_VERSION = 1

# options (enum kmm_option)
OPT_ENSEMBLE_GRAPH = 9
OPT_FUSED, OPT_COLUMN_BLOCKED, OPT_GRAPH, OPT_ZTMA, OPT_WAIT_LIMIT_MS, OPT_XBIG, OPT_TC_DCT, OPT_DERIVED_INPUTS = (
    1, 2, 3, 4, 5, 6, 7, 8)

# status codes (enum kmm_status)
OK, ERR_ARG, ERR_CUDA, ERR_CFL, ERR_NAN, ERR_INTERP, ERR_TIMEOUT, ERR_NOMEM, ERR_UNSUPPORTED, ERR_PCFL = range(10)
STATUS_NAMES = {
    OK: "KMM_OK", ERR_ARG: "KMM_ERR_ARG", ERR_CUDA: "KMM_ERR_CUDA", ERR_CFL: "KMM_ERR_CFL",
    ERR_NAN: "KMM_ERR_NAN", ERR_INTERP: "KMM_ERR_INTERP", ERR_TIMEOUT: "KMM_ERR_TIMEOUT",
    ERR_NOMEM: "KMM_ERR_NOMEM", ERR_UNSUPPORTED: "KMM_ERR_UNSUPPORTED", ERR_PCFL: "KMM_ERR_PCFL",
}

_PARAM_FIELDS = [
    ("nsteps", ctypes.c_int), ("iprnfrq", ctypes.c_int),
    ("dt", ctypes.c_double), ("gain", ctypes.c_double), ("ugain", ctypes.c_double), ("theta", ctypes.c_double),
    ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nx", ctypes.c_int),
    ("bftail", ctypes.c_int),
    ("yl", ctypes.c_double), ("zl", ctypes.c_double), ("xl", ctypes.c_double), ("re", ctypes.c_double),
    ("xstart", ctypes.c_double), ("uinf", ctypes.c_double),
    ("kwall", ctypes.c_int), ("perturbtime", ctypes.c_int),
    ("r_tau", ctypes.c_double), ("gravity", ctypes.c_double),
    ("irstrt", ctypes.c_int), ("crstrt", ctypes.c_int), ("print3d", ctypes.c_int), ("geomtype", ctypes.c_int),
    ("particle_flag", ctypes.c_int), ("flow_select", ctypes.c_int),
    ("itarget", ctypes.c_int), ("ipeter", ctypes.c_int), ("ipolyflag", ctypes.c_int), ("scl_flag", ctypes.c_int),
    ("npart", ctypes.c_int), ("new_part", ctypes.c_int),
    ("ratio", ctypes.c_double), ("ap", ctypes.c_double), ("c_mu", ctypes.c_double),
    ("cd_switch", ctypes.c_int),
    ("zlmax", ctypes.c_double), ("tpoly", ctypes.c_double), ("alpha_poly", ctypes.c_double),
    ("diffpoly", ctypes.c_double), ("c11z", ctypes.c_double), ("c22z", ctypes.c_double),
    ("c33z", ctypes.c_double), ("qbeta", ctypes.c_double),
    ("diff", ctypes.c_double), ("deltat", ctypes.c_double), ("sigmax", ctypes.c_double),
    ("sigmay", ctypes.c_double), ("sigmaz", ctypes.c_double),
    ("src_start", ctypes.c_int), ("src_stop", ctypes.c_int), ("scltarg", ctypes.c_int),
    ("cadence", ctypes.c_int),
    ("spts", ctypes.c_double),
    ("scalar_on", ctypes.c_int), ("polymer_on", ctypes.c_int),
    ("scalar_bc", ctypes.c_int),
    ("scalar_q", ctypes.c_double),
    ("tracer_scheme", ctypes.c_int),
    ("precision", ctypes.c_int),
    ("ib_spread_all", ctypes.c_int),
    ("flow_rate", ctypes.c_double),
]


class KmmParams(ctypes.Structure):
    _fields_ = _PARAM_FIELDS


class KmmStats(ctypes.Structure):
    _fields_ = [("cflmax", ctypes.c_double), ("umax", ctypes.c_double), ("it", ctypes.c_int), ("status", ctypes.c_int),
                ("pumax", ctypes.c_double), ("pcfl", ctypes.c_double), ("dpdx", ctypes.c_double)]


def _enum(names, start=0):
    return {n: start + i for i, n in enumerate(names)}


SPECTRAL_NAMES = (
    ["U", "V", "W", "OMX", "OMY", "OMZ", "FN", "FNM1", "GN", "GNM1",
     "U11", "U12", "U13", "U21", "U22", "U23", "U31", "U32", "U33", "LU", "LV", "LW",
     "GF1", "GF2", "WRKC", "WRK1",
     "SCALAR", "SCLX", "SCLY", "SCLZ", "SCN", "SCNM1",
     "C11", "C12", "C13", "C21", "C22", "C23", "C31", "C32", "C33",
     "C11N", "C12N", "C13N", "C22N", "C23N", "C33N",
     "C11NM1", "C12NM1", "C13NM1", "C22NM1", "C23NM1", "C33NM1",
     "STR11N", "STR12N", "STR13N", "STR22N", "STR23N", "STR33N",
     "STR11NM1", "STR12NM1", "STR13NM1", "STR22NM1", "STR23NM1", "STR33NM1",
     "QP11", "QP12", "QP13", "QP22", "QP23", "QP33",
     "T1", "T2", "T3"]
    + ["DC%d%d%d" % (i, j, k) for i in (1, 2, 3) for j in (1, 2, 3) for k in (1, 2, 3)]
    + ["CSOURCE"]
)
MEAN_NAMES = ["U0", "W0", "H1N", "H1NM1", "H3N", "H3NM1", "UXMEAN"]
WALL_NAMES = ["BCTOP", "BCBOT", "DNV1B", "DNV1T", "DNV2B", "DNV2T", "DENOM", "C1", "C2"]
PHYS_NAMES = (["FXINTG", "FYINTG", "FZINTG", "UP3D", "VP3D", "WP3D", "SWIRL3D", "WX3D", "WY3D", "WZ3D"]
              + ["U%d%dP3D" % (i, j) for i in (1, 2, 3) for j in (1, 2, 3)]
              + ["LUP3D", "LVP3D", "LWP3D", "UOLD", "VOLD", "WOLD", "LUNM1", "LVNM1", "LWNM1", "SCSOURCE"])
PART_NAMES = ["XPART", "YPART", "ZPART", "UPART", "VPART", "WPART", "SWIRLPART"]
INIT_NAMES = ["INITU", "INITV", "INITW", "INITSCL"]

FIELD = {}
FIELD.update(_enum(SPECTRAL_NAMES, 0))
FIELD["NSPECTRAL"] = len(SPECTRAL_NAMES)
FIELD.update(_enum(MEAN_NAMES, 200))
FIELD.update(_enum(WALL_NAMES, 300))
FIELD.update(_enum(PHYS_NAMES, 400))
FIELD["IMATRIX"] = 500
FIELD.update(_enum(PART_NAMES, 600))
FIELD.update(_enum(INIT_NAMES, 700))

globals().update({"F_" + k: v for k, v in FIELD.items()})


def field_kind(fid):
    """(kind, dtype-name) of a field id: spectral/mean/wall/phys/imatrix/part/init."""
    if 0 <= fid < 200:
        return "spectral", "complex128"
    if 200 <= fid < 300:
        return "mean", "float64"
    if 300 <= fid < 400:
        return "wall", "complex128"
    if 400 <= fid < 500:
        return "phys", "float64"
    if fid == 500:
        return "imatrix", "int32"
    if 600 <= fid < 700:
        return "part", "float64"
    if 700 <= fid < 800:
        return "init", "float64"
    raise ValueError("unknown field id %r" % fid)


def field_shape(fid, nx, ny, nz, npart=0):
    """Fortran-order shape of a field, as the reference declares it (main_dns.f90:23-100)."""
    nyp, nxh, mx, mz = ny + 1, nx // 2, 3 * nx // 2, 3 * nz // 2
    kind, _ = field_kind(fid)
    return {
        "spectral": (nyp, nz, nxh),
        "mean": (nyp,),
        "wall": (nz, nxh),
        "phys": (nyp, mz, mx),
        "imatrix": (nyp, mz, mx),
        "part": (npart,),
        "init": (nyp, nz, nx),
    }[kind]


def default_params(**kw):
    """Reference defaults for a plain channel (flow_select = 1, theta = 0.5), overridable by keyword."""
    p = KmmParams()
    base = dict(nsteps=1, iprnfrq=1000, dt=0.01, gain=50.0, ugain=50.0, theta=0.5,
                ny=32, nz=32, nx=32, bftail=0, yl=2.0, zl=6.283185307179586, xl=12.566370614359172,
                re=1400.0, xstart=0.0, uinf=0.0, kwall=0, perturbtime=0, r_tau=64.80740698407860,
                gravity=0.0, irstrt=0, crstrt=0, print3d=0, geomtype=0, particle_flag=0, flow_select=1,
                itarget=0, ipeter=1, ipolyflag=1, scl_flag=0, npart=0, new_part=0, ratio=0.0, ap=1e-3,
                c_mu=1.0, cd_switch=0, zlmax=30.0, tpoly=20.0, alpha_poly=0.0, diffpoly=1000.0,
                c11z=1.0, c22z=1.0, c33z=1.0, qbeta=0.9, diff=1.0, deltat=0.0, sigmax=0.01, sigmay=0.01,
                sigmaz=0.01, src_start=0, src_stop=-1, scltarg=0, cadence=1000000, spts=0.0,
                scalar_on=0, polymer_on=0, scalar_bc=0, scalar_q=0.0, tracer_scheme=0, precision=0,
                ib_spread_all=0, flow_rate=0.0)
    base.update(kw)
    for k, v in base.items():
        if not hasattr(p, k):
            raise AttributeError("kmm_params has no member %r" % k)
        setattr(p, k, v)
    return p
