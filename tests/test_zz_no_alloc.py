"""GPU test of gx_massgn_noalloc, the mass-assignment entry point that
allocates no memory (for callers that may not allocate device memory while
they deposit mass).  It is called through the C ABI on device buffers the
test owns and must reproduce the mass array of the existing gx_masset path
of the same particles, on two calls in a row (the second call finds the
shared working array holding the first call's contents).  This file is
collected last so a failure here stops a `-x` run only after every other
test ran."""
import ctypes as C

import numpy as np
import pytest

from galaxy_b200 import (Galaxy, lib, make_config, GX_GRID_MASS, GX_OK, GX_RMAP_LOG,
                         GX_RMAP_STDPOL)
from galaxy_b200._abi import GxConfig, GX_ERR_RANGE
from galaxy_b200.disk import kt_disk

pytestmark = pytest.mark.gpu


def _setup(L):
    L.gx_massgn_noalloc.argtypes = [C.POINTER(GxConfig), C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_void_p]
    return L


CASES = {
    "3d": (make_config(3, 32, 64, ngz=15, dzg=0.1, ng=9, rmap=GX_RMAP_LOG,
                       rmap_a=float(np.log(100.0) / 31), rmap_r0=0.05, softl=0.2, tsoft=1),
           dict(ndim=3, rmax=4.5, z0=0.1, lscale=1.0)),
    "2d": (make_config(2, 40, 64, ng=9, rmap=GX_RMAP_STDPOL, softl=1.0, tsoft=1),
           dict(ndim=2, rmax=5.0, z0=0.1, lscale=5.0)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_massgn_matches_masset_twice(case):
    import torch
    cfg, d = CASES[case]
    rec, pm = kt_disk(150000, seed=21, rmax=d["rmax"], ndim=d["ndim"], z0=d["z0"],
                      lscale=d["lscale"])
    cfg.pmass = pm
    with Galaxy(cfg) as gal:
        gal.loadup(rec)
        gal.masset()
        ref = gal.grid(GX_GRID_MASS).astype(np.float64)
    L = _setup(lib())
    coords = torch.from_numpy(rec).cuda()
    outs = []
    for _ in range(2):
        out = torch.full((gal.mesh,), -1.0, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        rc = L.gx_massgn_noalloc(C.byref(cfg), coords.data_ptr(), rec.shape[0], out.data_ptr(),
                                 None)
        assert rc == GX_OK
        outs.append(out.cpu().numpy().astype(np.float64))
    scale = ref.max()
    for m in outs:
        # fixed-point quanta 2^-20 (gx_masset) and 2^-32 (this entry point)
        assert np.abs(m - ref).max() / scale < 2e-6
        assert abs(m.sum() - ref.sum()) / ref.sum() < 1e-6
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_massgn_on_a_caller_stream():
    """Work queued on a caller's stream (a torch stream handle): the call
    returns before the work completes, the caller synchronises that stream,
    and the result equals gx_masset's.  A warm-up call with n = 0 first, as
    a caller does at set-up; the caller's current device is unchanged."""
    import torch
    cfg, d = CASES["3d"]
    rec, pm = kt_disk(100000, seed=22, rmax=d["rmax"], ndim=d["ndim"], z0=d["z0"],
                      lscale=d["lscale"])
    cfg.pmass = pm
    with Galaxy(cfg) as gal:
        gal.loadup(rec)
        gal.masset()
        ref = gal.grid(GX_GRID_MASS).astype(np.float64)
        mesh = gal.mesh
    L = _setup(lib())
    coords = torch.from_numpy(rec).cuda()
    out = torch.full((mesh,), -1.0, dtype=torch.float32, device="cuda")
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    dev = torch.cuda.current_device()
    assert L.gx_massgn_noalloc(C.byref(cfg), None, 0, out.data_ptr(), st.cuda_stream) == GX_OK
    st.synchronize()
    assert float(out.abs().max()) == 0.0  # no particles: an empty mesh
    rc = L.gx_massgn_noalloc(C.byref(cfg), coords.data_ptr(), rec.shape[0], out.data_ptr(),
                             st.cuda_stream)
    assert rc == GX_OK
    st.synchronize()
    assert torch.cuda.current_device() == dev
    m = out.cpu().numpy().astype(np.float64)
    assert np.abs(m - ref).max() / ref.max() < 2e-6
    assert abs(m.sum() - ref.sum()) / ref.sum() < 1e-6


def test_noalloc_rejects_mesh_beyond_limit():
    import torch
    L = _setup(lib())
    cfg = make_config(3, 160, 256, ngz=125, dzg=0.04, ng=4, rmap=GX_RMAP_LOG,
                      rmap_a=float(np.log(100.0) / 159), rmap_r0=0.05, softl=0.1, tsoft=1)
    out = torch.zeros(8, device="cuda")
    coords = torch.zeros(6, device="cuda")
    rc = L.gx_massgn_noalloc(C.byref(cfg), coords.data_ptr(), 1, out.data_ptr(), None)
    assert rc == GX_ERR_RANGE
