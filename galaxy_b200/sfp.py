"""Abel-Jacobi basis data for the SFP entry points (host side).

The basis is the reference's set k (SRC/lib15/ajsetup.f:23-58): per (m, n),
n roots and k + 1 coefficients of the polynomial in 1 - r^2 of
U_nm(r) = pi/sqrt(2) r^m [sum_i c_i (1 - r^2)^i] prod_j (r^2 - root_j^2)
(ajfun.f:33-47).  `Basis` keeps the arrays alive and builds the GxSfpBasis
struct the C ABI takes.
"""
import json

import numpy as np

from ._abi import GxSfpBasis


class Basis:
    def __init__(self, k, roots, xcoeff, maxm, maxn, minm=0, minn=0, nsect=1, nrtab=1001):
        """roots[(m, n)] -> n roots; xcoeff[(m, n)] -> k + 1 coefficients."""
        self.k, self.maxm, self.maxn = k, maxm, maxn
        self.minm, self.minn, self.nsect, self.nrtab = minm, minn, nsect, nrtab
        self.roots = np.zeros((maxm + 1, maxn + 1, max(maxn, 1)), np.float64)
        self.xcoeff = np.zeros((maxm + 1, maxn + 1, k + 1), np.float64)
        for m in range(maxm + 1):
            for n in range(maxn + 1):
                r = roots[(m, n)]
                self.roots[m, n, :len(r)] = r
                self.xcoeff[m, n, :] = xcoeff[(m, n)]
        self.c = GxSfpBasis(k, minm, maxm, minn, maxn, nsect, nrtab,
                            self.roots.ctypes.data, self.xcoeff.ctypes.data)

    @classmethod
    def from_json(cls, path, maxm=None, maxn=None, **kw):
        d = json.load(open(path))
        maxm = d["maxm"] if maxm is None else maxm
        maxn = d["maxn"] if maxn is None else maxn
        roots = {tuple(int(v) for v in key.split(",")): val for key, val in d["roots"].items()}
        xc = {tuple(int(v) for v in key.split(",")): val for key, val in d["xcoeff"].items()}
        return cls(d["k"], roots, xc, maxm, maxn, **kw)

    def functions(self):
        return [(m, n) for m in range(self.minm, self.maxm + 1, self.nsect)
                for n in range(self.minn, self.maxn + 1)]


class Sfp:
    """SFP coefficient sum and forces on one GPU (a GxSfp)."""

    def __init__(self, basis, maxr, device=0):
        import ctypes as C
        from . import lib, GxError, GX_OK
        from ._abi import GxSfpBasis
        self._C, self._E, self._OK = C, GxError, GX_OK
        L = lib()
        P = C.c_void_p
        L.gx_sfp_init.argtypes = [C.POINTER(GxSfpBasis), C.c_double, C.c_int, C.POINTER(P)]
        L.gx_sfp_destroy.argtypes = [P]
        L.gx_sfp_destroy.restype = None
        L.gx_sfp_last_error.argtypes = [P]
        L.gx_sfp_last_error.restype = C.c_char_p
        L.gx_sfp_load.argtypes = [P, P, C.c_int64, C.c_int]
        L.gx_sfp_sum.argtypes = [P, C.c_int, C.c_double, P]
        L.gx_sfp_acc.argtypes = [P, P, P, P]
        L.gx_sfp_last_ms.argtypes = [P, C.POINTER(C.c_float), C.POINTER(C.c_int64)]
        L.gx_sfp_step.argtypes = [P, C.c_int, C.c_double, C.c_int, C.c_double, P]
        L.gx_sfp_unload.argtypes = [P, P]
        self._L = L
        self.basis = basis
        self._h = C.c_void_p()
        rc = L.gx_sfp_init(C.byref(basis.c), float(maxr), device, C.byref(self._h))
        if rc != GX_OK:
            raise GxError(rc, L.gx_sfp_last_error(None).decode())
        self.n = 0

    def _chk(self, rc):
        if rc != self._OK:
            raise self._E(rc, self._L.gx_sfp_last_error(self._h).decode())

    def close(self):
        if self._h:
            self._L.gx_sfp_destroy(self._h)
            self._h = self._C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def load(self, coords):
        coords = np.ascontiguousarray(coords, dtype=np.float32)
        self.n = coords.shape[0]
        self._chk(self._L.gx_sfp_load(self._h, coords.ctypes.data, self.n, coords.shape[1]))

    def sum(self, pmass=1.0, precision=0):
        b = self.basis
        out = np.zeros((b.maxn + 1) * (2 * b.maxm + 1), np.float64)
        self._chk(self._L.gx_sfp_sum(self._h, precision, float(pmass), out.ctypes.data))
        return out.reshape(b.maxn + 1, 2 * b.maxm + 1)

    def acc(self, coeff):
        coeff = np.ascontiguousarray(coeff, np.float64)
        acc = np.zeros((self.n, 2), np.float32)
        pot = np.zeros(self.n, np.float32)
        self._chk(self._L.gx_sfp_acc(self._h, coeff.ctypes.data, acc.ctypes.data, pot.ctypes.data))
        return acc, pot

    def step(self, nsteps, dt, pmass=1.0, precision=0):
        """nsteps leapfrog steps in the particles' own SFP field (positions
        and velocities from `load`); returns the coefficients of the final
        positions."""
        b = self.basis
        out = np.zeros((b.maxn + 1) * (2 * b.maxm + 1), np.float64)
        self._chk(self._L.gx_sfp_step(self._h, int(nsteps), float(dt), precision, float(pmass),
                                      out.ctypes.data))
        return out.reshape(b.maxn + 1, 2 * b.maxm + 1)

    def unload(self):
        """The particles as (n, 4) records: x, y, vx, vy."""
        out = np.zeros((self.n, 4), np.float32)
        self._chk(self._L.gx_sfp_unload(self._h, out.ctypes.data))
        return out

    def last_ms(self):
        ms = self._C.c_float()
        nl = self._C.c_int64()
        self._chk(self._L.gx_sfp_last_ms(self._h, self._C.byref(ms), self._C.byref(nl)))
        return ms.value, nl.value
