"""ctypes mirror of include/galaxy_gpu.h (structs and constants).

The C header is the contract; this module only restates it for Python
callers (tests, bench.py and the host-side helpers in this package).
"""
import ctypes as C

GX_OK = 0
GX_ERR_ARG = -1
GX_ERR_CUDA = -2
GX_ERR_STATE = -3
GX_ERR_NOMEM = -4
GX_ERR_TIMEOUT = -5
GX_ERR_RANGE = -6
GX_ERR_DEVICE = -7

GX_RMAP_STDPOL = 0
GX_RMAP_LOG = 1
GX_SOFT_PLUMMER = 1
GX_SOFT_SPLINE = 2
GX_PREC_MIXED = 0
GX_PREC_FP64 = 1
GX_PREC_MIXED_TC05 = 2
GX_FLAG_COMPENSATED = 1
GX_FLAG_QUADRATIC = 2
GX_FLAG_WHOLE_GRID = 4
GX_FLAG_SORTED_DEPOSIT = 8
GX_FLAG_PLANE_SPLIT = 16
GX_FLAG_ROWBLOCK_TRANSFORMS = 32
GX_OP_SUM, GX_OP_MIN, GX_OP_MAX = 0, 1, 2
GX_DT_INT32, GX_DT_FLOAT32 = 0, 1

GX_GRID_MASS = 0
GX_GRID_FR = 1
GX_GRID_FT = 2
GX_GRID_FZ = 3
GX_GRID_POT = 4
GX_GRID_FX = 5
GX_GRID_FY = 6

GX_GREEN_FR = 0
GX_GREEN_FT = 1
GX_GREEN_FZ = 2
GX_GREEN_POT = 3

GX_MAX_SKIP = 16


class GxConfig(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32),
        ("nr", C.c_int32),
        ("na", C.c_int32),
        ("ngz", C.c_int32),
        ("dzg", C.c_float),
        ("ng", C.c_int32),
        ("nsect", C.c_int32),
        ("nskip", C.c_int32),
        ("skip", C.c_int32 * GX_MAX_SKIP),
        ("rmap", C.c_int32),
        ("rmap_a", C.c_float),
        ("rmap_r0", C.c_float),
        ("softl", C.c_float),
        ("tsoft", C.c_int32),
        ("pmass", C.c_float),
        ("halo", C.c_int32),
        ("halo_v2", C.c_float),
        ("halo_rc", C.c_float),
        ("precision", C.c_int32),
        ("flags", C.c_int32),
        ("device", C.c_int32),
    ]


class GxGeometry(C.Structure):
    _fields_ = [
        ("nr", C.c_int32),
        ("na", C.c_int32),
        ("ngz", C.c_int32),
        ("ng", C.c_int32),
        ("mmax", C.c_int32),
        ("nsect", C.c_int32),
        ("mesh", C.c_int32),
        ("alpha", C.c_float),
        ("ua", C.c_float),
        ("uoffs", C.c_float),
        ("rinh", C.c_float),
        ("rgrid", C.c_float),
        ("zm", C.c_float),
        ("thmax", C.c_float),
        ("nact", C.c_int32),
        ("lg", C.c_uint8 * 260),
    ]


class GxDiag(C.Structure):
    _fields_ = [
        ("ke", C.c_double),
        ("pe", C.c_double),
        ("lz", C.c_double),
        ("virial", C.c_double),
        ("a2_re", C.c_double),
        ("a2_im", C.c_double),
        ("n_on_grid", C.c_int64),
    ]


class GxSfpBasis(C.Structure):
    _fields_ = [
        ("k", C.c_int32),
        ("minm", C.c_int32),
        ("maxm", C.c_int32),
        ("minn", C.c_int32),
        ("maxn", C.c_int32),
        ("nsect", C.c_int32),
        ("nrtab", C.c_int32),
        ("roots", C.c_void_p),
        ("xcoeff", C.c_void_p),
    ]


def make_config(ndim, nr, na, ngz=1, dzg=0.0, ng=1, nsect=1, skip=(),
                rmap=GX_RMAP_STDPOL, rmap_a=0.0, rmap_r0=0.0, softl=1.0,
                tsoft=GX_SOFT_PLUMMER, pmass=1.0, halo=0, halo_v2=0.0,
                halo_rc=1.0, precision=GX_PREC_MIXED, flags=0, device=0):
    """Build a GxConfig from the reference's card values (p2dset/p3dset)."""
    c = GxConfig()
    c.ndim = ndim
    c.nr = nr
    c.na = na
    c.ngz = ngz if ndim == 3 else 1
    c.dzg = dzg
    c.ng = ng
    c.nsect = nsect
    c.nskip = len(skip)
    for i, s in enumerate(skip):
        c.skip[i] = s
    c.rmap = rmap
    c.rmap_a = rmap_a
    c.rmap_r0 = rmap_r0
    c.softl = softl
    c.tsoft = tsoft
    c.pmass = pmass
    c.halo = halo
    c.halo_v2 = halo_v2
    c.halo_rc = halo_rc
    c.precision = precision
    c.flags = flags
    c.device = device
    return c
