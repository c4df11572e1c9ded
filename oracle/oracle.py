"""ctypes driver of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, to check results against.  The product path
(galaxy_b200) never imports this module.

Every function wraps one restated reference routine; see gx_oracle.h for
the layouts and gx_oracle_tmpl.h for the file:line of each restatement.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from galaxy_b200._abi import GxConfig, GxGeometry, GxDiag, GxSfpBasis

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
        _setup(_lib)
    return _lib


def _setup(L):
    P = C.c_void_p
    i64 = C.c_int64
    L.ox_geometry.argtypes = [C.POINTER(GxConfig), C.POINTER(GxGeometry), C.c_char_p, C.c_int]
    L.ox_green_size.argtypes = [C.POINTER(GxConfig)]
    L.ox_green_size.restype = i64
    L.ox_direct_size.argtypes = [C.POINTER(GxConfig)]
    L.ox_direct_size.restype = i64
    for s in ("f64", "f32"):
        getattr(L, "ox_green_" + s).argtypes = [C.POINTER(GxConfig), P, P]
        getattr(L, "ox_weight_" + s).argtypes = [C.POINTER(GxConfig), C.c_int, i64, P, P, P, P]
        getattr(L, "ox_massgn_" + s).argtypes = [C.POINTER(GxConfig), i64, P, P, P, P, P]
        getattr(L, "ox_findf_" + s).argtypes = [C.POINTER(GxConfig), P, P, C.c_int, C.c_int,
                                                C.c_int, P]
        getattr(L, "ox_polcat_" + s).argtypes = [C.POINTER(GxConfig), P]
        getattr(L, "ox_grdacc_" + s).argtypes = [C.POINTER(GxConfig), i64, P, P, C.c_int, P, P]
        getattr(L, "ox_masset_" + s).argtypes = [C.POINTER(GxConfig), i64, P, P, P]
        getattr(L, "ox_step_" + s).argtypes = [C.POINTER(GxConfig), P, i64, P, P, P, C.c_int,
                                               C.c_int, P]
        getattr(L, "ox_particle_pass_" + s).argtypes = [C.POINTER(GxConfig), i64, P, P, P, P]
        getattr(L, "ox_direct_field_" + s).argtypes = [C.POINTER(GxConfig), P, C.c_int, P, P,
                                                       P, P, C.c_int, P]
    L.ox_set_threads.argtypes = [C.c_int]
    L.ox_ajfun.argtypes = [C.POINTER(GxSfpBasis), C.c_int, C.c_int, C.c_double]
    L.ox_ajfun.restype = C.c_double
    L.ox_ajder.argtypes = [C.POINTER(GxSfpBasis), C.c_int, C.c_int, C.c_double]
    L.ox_ajder.restype = C.c_double
    L.ox_sfp_coeffs.argtypes = [C.POINTER(GxSfpBasis), i64, P, C.c_int, C.c_double, C.c_double, P]
    L.ox_sfp_acc.argtypes = [C.POINTER(GxSfpBasis), P, i64, P, C.c_int, C.c_double, P, P]
    L.ox_icheck.argtypes = [C.POINTER(GxConfig), i64, P, P, P, C.c_double, C.POINTER(GxDiag)]
    L.ox_adj_forward.argtypes = [C.POINTER(GxConfig), P, i64, P, C.c_int, P, P]
    L.ox_adj_gradient.argtypes = [C.POINTER(GxConfig), P, i64, P, C.c_int, P, P, P]


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _dt(prec):
    return (np.float64, "f64") if prec == 64 else (np.float32, "f32")


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with {rc}")


def set_threads(n):
    """Host threads of the restated loops (1 = sequential reference order)."""
    return lib().ox_set_threads(int(n))


def geometry(cfg):
    g = GxGeometry()
    err = C.create_string_buffer(256)
    rc = lib().ox_geometry(C.byref(cfg), C.byref(g), err, 256)
    if rc != 0:
        raise ValueError(err.value.decode())
    return g


def nkz(cfg):
    return cfg.ngz + 1 if cfg.ndim == 3 else 1


def green(cfg, prec=64, direct=False):
    """Transformed Green table [4][ng][nkz][is][ir] (and the direct one)."""
    dt, s = _dt(prec)
    g = geometry(cfg)
    G = np.zeros(lib().ox_green_size(C.byref(cfg)), dtype=dt)
    D = np.zeros(lib().ox_direct_size(C.byref(cfg)), dtype=dt) if direct else None
    _chk(getattr(lib(), "ox_green_" + s)(C.byref(cfg), _p(G), _p(D)), "green")
    G = G.reshape(4, g.ng, nkz(cfg), g.nr, g.nr)
    if direct:
        D = D.reshape(4, g.nr, g.nr, nkz(cfg), g.na // 2 + 1)
        return G, D
    return G


def weight(cfg, pos, old=False, prec=64):
    dt, s = _dt(prec)
    pos = np.ascontiguousarray(pos, dtype=dt)
    n = pos.shape[0]
    key = np.zeros(n, np.int32)
    wt = np.zeros((n, 27 if (cfg.ndim == 3 and cfg.flags & 2) else 8), dt)
    on = np.zeros(n, np.uint8)
    _chk(getattr(lib(), "ox_weight_" + s)(C.byref(cfg), int(old), n, _p(pos), _p(key), _p(wt),
                                           _p(on)), "weight")
    return key, wt, on


def masset(cfg, pos, prec=64):
    """Scaled mass array and 1-based active ring range (jrad, krad)."""
    dt, s = _dt(prec)
    pos = np.ascontiguousarray(pos, dtype=dt)
    g = geometry(cfg)
    mass = np.zeros(g.mesh, dt)
    jrk = np.zeros(2, np.int32)
    _chk(getattr(lib(), "ox_masset_" + s)(C.byref(cfg), pos.shape[0], _p(pos), _p(mass),
                                           _p(jrk)), "masset")
    return mass, (int(jrk[0]), int(jrk[1]))


def findf(cfg, G, mass, lpot=True, jrk=None, prec=64, polar=True):
    """Fields [4][mesh] (radial, azimuthal, vertical, potential) or, with
    polar=False, Cartesian (fx, fy, fz, potential) after polcat."""
    dt, s = _dt(prec)
    g = geometry(cfg)
    G = np.ascontiguousarray(G, dtype=dt)
    mass = np.ascontiguousarray(mass, dtype=dt)
    if jrk is None:
        jrk = (1, g.nr)
    f = np.zeros((4, g.mesh), dt)
    _chk(getattr(lib(), "ox_findf_" + s)(C.byref(cfg), _p(G), _p(mass), int(lpot), jrk[0],
                                          jrk[1], _p(f)), "findf")
    if not polar:
        _chk(getattr(lib(), "ox_polcat_" + s)(C.byref(cfg), _p(f)), "polcat")
    return f


def grdacc(cfg, pos, fields, phys=True, prec=64):
    dt, s = _dt(prec)
    pos = np.ascontiguousarray(pos, dtype=dt)
    fields = np.ascontiguousarray(fields, dtype=dt)
    n = pos.shape[0]
    acc = np.zeros((n, cfg.ndim), dt)
    pot = np.zeros(n, dt)
    _chk(getattr(lib(), "ox_grdacc_" + s)(C.byref(cfg), n, _p(pos), _p(fields), int(phys),
                                           _p(acc), _p(pot)), "grdacc")
    return acc, pot


def step(cfg, G, pos, nsteps, phys=False, prec=64):
    """Advance AoS particle records nsteps (masset first).  Returns
    (pos, mass, fields-of-last-solve)."""
    dt, s = _dt(prec)
    pos = np.array(pos, dtype=dt, copy=True, order="C")
    G = np.ascontiguousarray(G, dtype=dt)
    g = geometry(cfg)
    mass, jrk = masset(cfg, pos, prec)
    jrk = np.array(jrk, np.int32)
    f = np.zeros((4, g.mesh), dt)
    _chk(getattr(lib(), "ox_step_" + s)(C.byref(cfg), _p(G), pos.shape[0], _p(pos), _p(mass),
                                         _p(jrk), nsteps, int(phys), _p(f)), "step")
    return pos, mass, f


def particle_pass(cfg, pos, fields, prec=32):
    """One step's particle loop in place on pos (grdacc, stpgrp, massgn,
    scaled); returns the new mass array and ring range."""
    dt, s = _dt(prec)
    assert pos.dtype == dt and pos.flags.c_contiguous
    g = geometry(cfg)
    mass = np.zeros(g.mesh, dt)
    jrk = np.zeros(2, np.int32)
    fields = np.ascontiguousarray(fields, dtype=dt)
    _chk(getattr(lib(), "ox_particle_pass_" + s)(C.byref(cfg), pos.shape[0], _p(pos), _p(fields),
                                                  _p(mass), _p(jrk)), "particle_pass")
    return mass, (int(jrk[0]), int(jrk[1]))


def direct_field(cfg, D, masses, lpot=True, prec=64):
    """Direct convolution for point masses [(ring, spoke, plane, m)], 1-based."""
    dt, s = _dt(prec)
    g = geometry(cfg)
    D = np.ascontiguousarray(D, dtype=dt)
    mr = np.array([m[0] for m in masses], np.int32)
    mt = np.array([m[1] for m in masses], np.int32)
    mz = np.array([m[2] for m in masses], np.int32)
    mm = np.array([m[3] for m in masses], dt)
    f = np.zeros((4, g.mesh), dt)
    _chk(getattr(lib(), "ox_direct_field_" + s)(C.byref(cfg), _p(D), len(masses), _p(mr),
                                                 _p(mt), _p(mz), _p(mm), int(lpot), _p(f)),
         "direct_field")
    return f


def icheck(cfg, pos, acc=None, pot=None, pmass=1.0):
    pos = np.ascontiguousarray(pos, np.float64)
    acc = None if acc is None else np.ascontiguousarray(acc, np.float64)
    pot = None if pot is None else np.ascontiguousarray(pot, np.float64)
    d = GxDiag()
    _chk(lib().ox_icheck(C.byref(cfg), pos.shape[0], _p(pos), _p(acc), _p(pot), pmass,
                         C.byref(d)), "icheck")
    return d


def ajfun(basis, m, n, r):
    return lib().ox_ajfun(C.byref(basis.c), m, n, float(r))


def ajder(basis, m, n, r):
    return lib().ox_ajder(C.byref(basis.c), m, n, float(r))


def sfp_coeffs(basis, pos, maxr, pmass=1.0):
    """sfpadd over all particles (table + Lagrange, FP64), scaled; layout
    [maxn + 1][2 maxm + 1], cosine at +m, sine at -m."""
    pos = np.ascontiguousarray(pos, np.float64)
    out = np.zeros((basis.maxn + 1) * (2 * basis.maxm + 1), np.float64)
    _chk(lib().ox_sfp_coeffs(C.byref(basis.c), pos.shape[0], _p(pos), pos.shape[1], float(maxr),
                             float(pmass), _p(out)), "sfp_coeffs")
    return out.reshape(basis.maxn + 1, 2 * basis.maxm + 1)


def sfp_acc(basis, coeff, pos, maxr):
    pos = np.ascontiguousarray(pos, np.float64)
    coeff = np.ascontiguousarray(coeff, np.float64)
    acc = np.zeros((pos.shape[0], 2), np.float64)
    pot = np.zeros(pos.shape[0], np.float64)
    _chk(lib().ox_sfp_acc(C.byref(basis.c), _p(coeff), pos.shape[0], _p(pos), pos.shape[1],
                          float(maxr), _p(acc), _p(pot)), "sfp_acc")
    return acc, pot


def adj_forward(cfg, G, pos, nsteps):
    """J = |A2| after masset + nsteps FP64 steps of the records pos (n x 4,
    2D), A2 = mean e^{2 i phi} over all particles (gx_oracle_adj.h)."""
    L = lib()
    q = np.ascontiguousarray(pos, np.float64).copy()
    G = np.ascontiguousarray(G, np.float64)
    a2 = np.zeros(2)
    J = np.zeros(1)
    _chk(L.ox_adj_forward(C.byref(cfg), _p(G), len(q), _p(q), int(nsteps), _p(a2), _p(J)),
         "ox_adj_forward")
    return float(J[0]), complex(a2[0], a2[1]), q


def adj_gradient(cfg, G, pos, nsteps):
    """(J, grad [n][4] = dJ/d(x, y, vx, vy), dJ/d(halo_rc, halo_v2)) in FP64"""
    L = lib()
    q = np.ascontiguousarray(pos, np.float64)
    G = np.ascontiguousarray(G, np.float64)
    grad = np.zeros((len(q), 4))
    dth = np.zeros(2)
    J = np.zeros(1)
    _chk(L.ox_adj_gradient(C.byref(cfg), _p(G), len(q), _p(q), int(nsteps), _p(grad), _p(dth),
                           _p(J)), "ox_adj_gradient")
    return float(J[0]), grad, dth


class OxZones(C.Structure):
    _fields_ = [("nzones", C.c_int32), ("nstep", C.c_int32 * 8), ("zbr", C.c_double * 8),
                ("istep", C.c_int32), ("lstep", (C.c_int32 * 2) * 8),
                ("jrk", (C.c_int32 * 2) * 8)]


class ZoneRun:
    """FP64 run with multiple time-step zones (gx_oracle_zone.h): loadup's
    zone assignment and velocity scaling, masset, steps, unload.  pos holds
    velocities in zone-step units between setup and records()."""

    def __init__(self, cfg, G, pos, nstep, zbr):
        L = lib()
        for name, at in (("ox_zone_setup", [C.POINTER(GxConfig), C.POINTER(OxZones), C.c_int64,
                                            C.c_void_p, C.c_void_p]),
                         ("ox_zone_unscale", [C.POINTER(GxConfig), C.POINTER(OxZones),
                                              C.c_int64, C.c_void_p, C.c_void_p]),
                         ("ox_zone_masset", [C.POINTER(GxConfig), C.POINTER(OxZones), C.c_int64,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p]),
                         ("ox_zone_step", [C.POINTER(GxConfig), C.POINTER(OxZones), C.c_void_p,
                                           C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_int])):
            getattr(L, name).argtypes = at
        self.cfg = cfg
        self.G = np.ascontiguousarray(G, np.float64)
        self.z = OxZones()
        self.z.nzones = len(nstep)
        for i, (s, r) in enumerate(zip(nstep, zbr)):
            self.z.nstep[i] = int(s)
            self.z.zbr[i] = float(r)
        self.pos = np.array(pos, np.float64, copy=True, order="C")
        n = len(self.pos)
        self.zone = np.zeros(n, np.int32)
        g = geometry(cfg)
        self.zm = np.zeros((len(nstep), g.mesh))
        self.zo = np.zeros((len(nstep), g.mesh))
        self.jrk = np.zeros(2, np.int32)
        _chk(L.ox_zone_setup(C.byref(cfg), C.byref(self.z), n, _p(self.pos), _p(self.zone)),
             "zone_setup")
        _chk(L.ox_zone_masset(C.byref(cfg), C.byref(self.z), n, _p(self.pos), _p(self.zone),
                              _p(self.zm), _p(self.zo), _p(self.jrk)), "zone_masset")

    def step(self, nsteps):
        _chk(lib().ox_zone_step(C.byref(self.cfg), C.byref(self.z), _p(self.G), len(self.pos),
                                _p(self.pos), _p(self.zone), _p(self.zm), _p(self.zo),
                                _p(self.jrk), int(nsteps)), "zone_step")

    @property
    def mass(self):
        return self.zm[0]

    def records(self):
        """particle records with velocities in base-step units"""
        q = self.pos.copy()
        _chk(lib().ox_zone_unscale(C.byref(self.cfg), C.byref(self.z), len(q), _p(q),
                                   _p(self.zone)), "zone_unscale")
        return q


def danl(cfg, mass, lscale, ts):
    """density harmonics [nr][ng] complex of a mass array (densty.f 'danl')"""
    L = lib()
    L.ox_danl.argtypes = [C.POINTER(GxConfig), C.c_void_p, C.c_double, C.c_void_p]
    g = geometry(cfg)
    m = np.ascontiguousarray(mass, np.float64)
    w = np.zeros(2 * g.ng * g.nr)
    _chk(L.ox_danl(C.byref(cfg), _p(m), 1.0 / (lscale * ts * ts), _p(w)), "danl")
    half = g.ng * g.nr
    return (w[:half] + 1j * w[half:]).reshape(g.nr, g.ng)
