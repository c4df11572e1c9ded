"""galaxy_b200 -- B200-native polar-grid particle-mesh step of GALAXY v15.

The compute lives in the in-tree CUDA library ``libgalaxy_gpu.so`` (C ABI
in ``include/galaxy_gpu.h``).  This module is the host-side mirror of the
lib15 routine interface for the path (grdset, greenm, loadup, masset,
findf, getacc, step, tmcent, icheck), one method per reference routine with
the same meaning and error behaviour: every failure raises ``GxError`` with
the library's message, as the reference stops in ``crash``
(SRC/lib15/crash.f:1-38).  There is no CPU fallback: importing the package
fails if the library is missing.
"""
import ctypes as C
import os

import numpy as np

from ._abi import (GxConfig, GxDiag, GxGeometry, make_config, GX_OK, GX_PREC_FP64,
                   GX_PREC_MIXED, GX_RMAP_LOG, GX_RMAP_STDPOL, GX_SOFT_PLUMMER,
                   GX_SOFT_SPLINE, GX_GRID_MASS, GX_GRID_FR, GX_GRID_FT, GX_GRID_FZ,
                   GX_GRID_POT, GX_GRID_FX, GX_GRID_FY, GX_GREEN_FR, GX_GREEN_FT,
                   GX_GREEN_FZ, GX_GREEN_POT, GX_FLAG_COMPENSATED,
                   GX_FLAG_QUADRATIC, GX_FLAG_WHOLE_GRID, GX_FLAG_SORTED_DEPOSIT,
                   GX_FLAG_PLANE_SPLIT, GX_FLAG_ROWBLOCK_TRANSFORMS)

__all__ = ["Galaxy", "GxError", "GxConfig", "GxDiag", "GxGeometry", "make_config", "lib",
           "LIB_PATH"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libgalaxy_gpu.so")
_lib = None


class GxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"galaxy_gpu error {code}: {msg}")
        self.code = code


def lib():
    """Load libgalaxy_gpu.so (built by galaxy_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m galaxy_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        i64 = C.c_int64
        L.gx_grdset.argtypes = [C.POINTER(GxConfig), C.POINTER(P)]
        L.gx_destroy.argtypes = [P]
        L.gx_destroy.restype = None
        L.gx_last_error.argtypes = [P]
        L.gx_last_error.restype = C.c_char_p
        L.gx_geometry.argtypes = [P, C.POINTER(GxGeometry)]
        L.gx_greenm.argtypes = [P]
        L.gx_green_get.argtypes = [P, C.c_int, P, i64]
        L.gx_loadup.argtypes = [P, P, i64]
        L.gx_unload.argtypes = [P, P]
        L.gx_weight.argtypes = [P, P, i64, C.c_int, P, P]
        L.gx_masset.argtypes = [P]
        L.gx_set_mass.argtypes = [P, P]
        L.gx_findf.argtypes = [P, C.c_int]
        L.gx_findf_polar.argtypes = [P, C.c_int]
        L.gx_get_grid.argtypes = [P, C.c_int, P]
        L.gx_getacc.argtypes = [P, P, P]
        L.gx_step.argtypes = [P, C.c_int, C.c_int]
        L.gx_tmcent.argtypes = [P, C.c_int]
        L.gx_icheck.argtypes = [P, C.POINTER(GxDiag)]
        L.gx_last_step_ms.argtypes = [P, C.POINTER(C.c_float)]
        L.gx_last_launch_count.argtypes = [P, C.POINTER(C.c_int64)]
        L.gx_comm_unique_id.argtypes = [C.c_char_p]
        L.gx_comm_init.argtypes = [P, C.c_char_p, C.c_int, C.c_int]
        L.gx_comm_host.argtypes = [P, C.c_int, C.c_int, P, P]
        L.gx_host_alloc.argtypes = [i64, C.POINTER(P)]
        L.gx_host_free.argtypes = [P]
        L.gx_set_profile.argtypes = [P, C.c_int]
        L.gx_phase_ms.argtypes = [P, P, P]
        L.gx_adjoint.argtypes = [P, C.c_int, C.c_int, P, P, P, P]
        L.gx_set_zones.argtypes = [P, C.c_int32, P, P]
        L.gx_zone_info.argtypes = [P, P, P]
        L.gx_zone_rings.argtypes = [P, P]
        L.gx_danl.argtypes = [P, C.c_double, P]
        _lib = L
    return _lib


class PinnedArray:
    """numpy view of page-locked host memory allocated by the library."""

    def __init__(self, shape, dtype=np.float32):
        nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self._p = C.c_void_p()
        rc = lib().gx_host_alloc(nbytes, C.byref(self._p))
        if rc != GX_OK:
            raise GxError(rc, "gx_host_alloc failed")
        buf = (C.c_char * nbytes).from_address(self._p.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    @property
    def ptr(self):
        return self._p.value

    def free(self):
        if self._p:
            self.array = None
            lib().gx_host_free(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Galaxy:
    """One polar grid and its particles on one GPU (a GxCtx)."""

    def __init__(self, cfg):
        self._L = lib()
        self._h = C.c_void_p()
        rc = self._L.gx_grdset(C.byref(cfg), C.byref(self._h))
        if rc != GX_OK:
            raise GxError(rc, self._L.gx_last_error(None).decode())
        self.cfg = cfg
        self.geo = GxGeometry()
        self._L.gx_geometry(self._h, C.byref(self.geo))
        self.ndim = cfg.ndim
        self.n = 0

    # -- plumbing ---------------------------------------------------------
    def _chk(self, rc):
        if rc != GX_OK:
            raise GxError(rc, self._L.gx_last_error(self._h).decode())

    def close(self):
        if self._h:
            self._L.gx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def mesh(self):
        return self.geo.mesh

    # -- lib15 routines -----------------------------------------------------
    def greenm(self):
        self._chk(self._L.gx_greenm(self._h))

    def green(self, gtype):
        g = self.geo
        nkz = g.ngz + 1 if self.ndim == 3 else 1
        out = np.zeros(g.ng * nkz * g.nr * g.nr, np.float64)
        self._chk(self._L.gx_green_get(self._h, gtype, _ptr(out), out.size))
        return out.reshape(g.ng, nkz, g.nr, g.nr)

    def loadup(self, coords):
        coords = np.ascontiguousarray(coords, dtype=np.float32)
        assert coords.ndim == 2 and coords.shape[1] == 2 * self.ndim
        self.n = coords.shape[0]
        self._chk(self._L.gx_loadup(self._h, _ptr(coords), self.n))

    def loadup_ptr(self, ptr, n):
        """loadup from a host pointer (e.g. pinned memory) of n records."""
        self.n = int(n)
        self._chk(self._L.gx_loadup(self._h, C.c_void_p(ptr), self.n))

    def unload_ptr(self, ptr):
        self._chk(self._L.gx_unload(self._h, C.c_void_p(ptr)))

    def set_comm(self, comm):
        """Bind to the ranks of a torch.distributed job (one rank per GPU)."""
        import torch.distributed as dist
        rank, world = dist.get_rank(), dist.get_world_size()
        buf = C.create_string_buffer(128)
        if rank == 0:
            self._chk(self._L.gx_comm_unique_id(buf))
        uid = comm.broadcast_bytes(buf.raw) if hasattr(comm, "broadcast_bytes") else None
        if uid is None:
            obj = [bytes(buf.raw)]
            dist.broadcast_object_list(obj, src=0)
            uid = obj[0]
        self._chk(self._L.gx_comm_init(self._h, uid, world, rank))

    def unload(self):
        out = np.zeros((self.n, 2 * self.ndim), np.float32)
        self._chk(self._L.gx_unload(self._h, _ptr(out)))
        return out

    def weight(self, coords, old=False):
        coords = np.ascontiguousarray(coords, dtype=np.float32)
        n = coords.shape[0]
        ncl = np.zeros(n, np.int32)
        quad = self.ndim == 3 and (self.cfg.flags & GX_FLAG_QUADRATIC)
        wt = np.zeros((n, 27 if quad else 8), np.float32)
        self._chk(self._L.gx_weight(self._h, _ptr(coords), n, int(old), _ptr(ncl), _ptr(wt)))
        return ncl, wt

    def masset(self):
        self._chk(self._L.gx_masset(self._h))

    def set_mass(self, mass):
        mass = np.ascontiguousarray(mass, dtype=np.float32).ravel()
        assert mass.size == self.mesh
        self._chk(self._L.gx_set_mass(self._h, _ptr(mass)))

    def findf(self, lpot=True):
        self._chk(self._L.gx_findf(self._h, int(lpot)))

    def findf_polar(self, lpot=True):
        self._chk(self._L.gx_findf_polar(self._h, int(lpot)))

    def grid(self, which):
        out = np.zeros(self.mesh, np.float32)
        self._chk(self._L.gx_get_grid(self._h, which, _ptr(out)))
        return out

    def getacc(self, want_pot=True):
        acc = np.zeros((self.n, self.ndim), np.float32)
        pot = np.zeros(self.n, np.float32) if want_pot else None
        self._chk(self._L.gx_getacc(self._h, _ptr(acc), _ptr(pot) if want_pot else None))
        return (acc, pot) if want_pot else acc

    def step(self, nsteps=1, phys=False):
        self._chk(self._L.gx_step(self._h, nsteps, int(phys)))

    def adjoint(self, nsteps, ckpt_every=50):
        """Gradient of J = |A2(t_final)| after nsteps steps (2D, mixed path)
        with respect to the loaded records and the halo parameters:
        returns (J, grad [n, 4] = dJ/d(x, y, vx, vy) in load order,
        dJ/d(halo_rc, halo_v2), reversal drift).  The context keeps its
        initial particles."""
        n = self.n
        J = np.zeros(1, np.float64)
        grad = np.zeros((n, 4), np.float32)
        dth = np.zeros(2, np.float64)
        drift = np.zeros(1, np.float32)
        self._chk(self._L.gx_adjoint(self._h, int(nsteps), int(ckpt_every), _ptr(J), _ptr(grad),
                                     _ptr(dth), _ptr(drift)))
        return float(J[0]), grad, dth, float(drift[0])

    def set_zones(self, nstep, zbr):
        """Multiple time-step zones (before loadup): zone i steps every
        nstep[i] base steps and holds the particles at radius >= zbr[i]
        (grid units; nstep[0] = 1, zbr[0] unused)."""
        nstep = np.ascontiguousarray(nstep, np.int32)
        zbr = np.ascontiguousarray(zbr, np.float32)
        assert nstep.size == zbr.size
        self._chk(self._L.gx_set_zones(self._h, int(nstep.size), _ptr(nstep), _ptr(zbr)))

    def zone_info(self):
        """(zone code of every particle in load order, 1..nzones or
        nzones + 1 off the grid; the step counter)"""
        zone = np.zeros(self.n, np.int32)
        istep = np.zeros(1, np.int32)
        self._chk(self._L.gx_zone_info(self._h, _ptr(zone), _ptr(istep)))
        return zone, int(istep[0])

    def zone_rings(self):
        """((jrs, krs) source rings, (jrf, krf) field rings) of the next
        step's solve, 1-based inclusive"""
        r = np.zeros(4, np.int32)
        self._chk(self._L.gx_zone_rings(self._h, _ptr(r)))
        return (int(r[0]), int(r[1])), (int(r[2]), int(r[3]))

    def tmcent(self, start=True):
        self._chk(self._L.gx_tmcent(self._h, int(start)))

    def icheck(self):
        d = GxDiag()
        self._chk(self._L.gx_icheck(self._h, C.byref(d)))
        return d

    def danl(self, lscale, ts):
        """Density harmonics of the grid rings (densty.f 'danl'):
        complex array [nr][ng], m = 0 the ring's surface density sum over
        spokes, m >= 1 the harmonic divided by it."""
        g = self.geo
        w = np.zeros(2 * g.ng * g.nr, np.float32)
        self._chk(self._L.gx_danl(self._h, 1.0 / (lscale * ts * ts), _ptr(w)))
        half = g.ng * g.nr
        return (w[:half] + 1j * w[half:]).reshape(g.nr, g.ng)

    def last_step_ms(self):
        v = C.c_float()
        self._chk(self._L.gx_last_step_ms(self._h, C.byref(v)))
        return v.value

    PHASES = ("fwd", "conv", "syn", "push", "sort", "deposit", "combine", "other")

    def set_profile(self, on=True):
        self._chk(self._L.gx_set_profile(self._h, int(on)))

    def phase_ms(self):
        ms = np.zeros(8, np.float32)
        cnt = np.zeros(8, np.int64)
        self._chk(self._L.gx_phase_ms(self._h, _ptr(ms), _ptr(cnt)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.PHASES) if cnt[i]}

    def last_launch_count(self):
        v = C.c_int64()
        self._chk(self._L.gx_last_launch_count(self._h, C.byref(v)))
        return v.value
