"""Ensemble of independent 2D discs on one GPU (a GxEnsemble).

The discs share one polar grid geometry and Green table; every step of all
of them is one persistent launch (gx_ensemble_step in
galaxy_b200/csrc/gx_ensemble.cu).  Each disc follows the single-disc run
(SRC/progs/galaxy.f:107-148: findf, getacc + stpgrp, massgn).
"""
import ctypes as C

import numpy as np


class Ensemble:
    """ndisc discs: records[d] is an (n_d, 4) array of x, y, vx, vy in grid
    units, pmass[d] the particle mass of disc d; cfg a 2D GxConfig."""

    def __init__(self, cfg, records, pmass, max_steps):
        from . import lib, GxError, GX_OK
        from ._abi import GxConfig
        self._E, self._OK = GxError, GX_OK
        L = lib()
        P = C.c_void_p
        i64p = C.POINTER(C.c_int64)
        ip = C.POINTER(C.c_int)
        L.gx_ensemble_create.argtypes = [C.POINTER(GxConfig), C.c_int, i64p, P, P, C.c_int,
                                         C.POINTER(P)]
        L.gx_ensemble_destroy.argtypes = [P]
        L.gx_ensemble_destroy.restype = None
        L.gx_ensemble_last_error.argtypes = [P]
        L.gx_ensemble_last_error.restype = C.c_char_p
        L.gx_ensemble_tune.argtypes = [P, ip, ip]
        L.gx_ensemble_config.argtypes = [P, ip, ip, ip, ip]
        L.gx_ensemble_step.argtypes = [P, C.c_int]
        L.gx_ensemble_steps_done.argtypes = [P, i64p]
        L.gx_ensemble_a2.argtypes = [P, P, C.c_int64]
        L.gx_ensemble_unload.argtypes = [P, P]
        L.gx_ensemble_last_ms.argtypes = [P, C.POINTER(C.c_float), i64p]
        self._L = L
        self.ndisc = len(records)
        self.counts = np.array([len(r) for r in records], np.int64)
        coords = np.ascontiguousarray(
            np.concatenate([np.asarray(r, np.float32).reshape(-1, 4) for r in records]), np.float32)
        pm = np.ascontiguousarray(pmass, np.float32)
        self.h = P()
        rc = L.gx_ensemble_create(C.byref(cfg), self.ndisc,
                                  self.counts.ctypes.data_as(i64p), pm.ctypes.data,
                                  coords.ctypes.data, int(max_steps), C.byref(self.h))
        if rc != GX_OK:
            raise GxError(rc, L.gx_ensemble_last_error(None).decode())

    def _chk(self, rc):
        if rc != self._OK:
            raise self._E(rc, self._L.gx_ensemble_last_error(self.h).decode())

    def tune(self):
        t, c = C.c_int(), C.c_int()
        self._chk(self._L.gx_ensemble_tune(self.h, C.byref(t), C.byref(c)))
        return t.value, c.value

    def config(self):
        v = [C.c_int() for _ in range(4)]
        self._chk(self._L.gx_ensemble_config(self.h, *[C.byref(x) for x in v]))
        return dict(threads=v[0].value, chunk=v[1].value, grid=v[2].value, graph=bool(v[3].value))

    def step(self, nsteps=1):
        self._chk(self._L.gx_ensemble_step(self.h, int(nsteps)))

    def steps_done(self):
        n = C.c_int64()
        self._chk(self._L.gx_ensemble_steps_done(self.h, C.byref(n)))
        return n.value

    def a2(self):
        """(steps_done + 1, ndisc) complex: mean of e^{2 i phi} over each
        disc's particles on the grid after each step."""
        s = self.steps_done()
        out = np.zeros((s + 1, self.ndisc, 2), np.float64)
        self._chk(self._L.gx_ensemble_a2(self.h, out.ctypes.data, out.size))
        return out[..., 0] + 1j * out[..., 1]

    def unload(self):
        """list of (n_d, 4) arrays, disc by disc."""
        out = np.zeros((int(self.counts.sum()), 4), np.float32)
        self._chk(self._L.gx_ensemble_unload(self.h, out.ctypes.data))
        return np.split(out, np.cumsum(self.counts)[:-1])

    def last_ms(self):
        ms, n = C.c_float(), C.c_int64()
        self._chk(self._L.gx_ensemble_last_ms(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def close(self):
        if self.h:
            self._L.gx_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
