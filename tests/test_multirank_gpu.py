"""The library's multi-rank path, run: two ranks of a gloo process group, each
with its own context on the same GPU and half of the particles, bound with
gx_comm_host so that the library's exchanges (MIN/MAX of the active ring
range, SUM of the forward spectrum; with GX_FLAG_PLANE_SPLIT each rank
contracts only its vertical wavenumbers and the ranks SUM the contracted
spectra, SRC/lib15_mpi/p3convp.f:180-190, 276-326) go through the host.
The reduced fields must be the single-context fields of all the particles
and the ranks' particles after a few steps the single-context run's
(FP32 sums in another order: 1e-6).  No kernel of one rank waits on the
other: the exchanges are host all-reduces between launches."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case(name):
    from galaxy_b200 import make_config, GX_RMAP_LOG, GX_RMAP_STDPOL, GX_FLAG_PLANE_SPLIT
    from galaxy_b200.disk import kt_disk
    if name == "2d":
        cfg = make_config(2, 40, 64, ng=9, rmap=GX_RMAP_STDPOL, softl=1.0, tsoft=1)
        rec, pm = kt_disk(60000, seed=3, rmax=5.0, ndim=2, dt=0.025, lscale=5.0)
    else:
        nr = 32
        cfg = make_config(3, nr, 64, ngz=15, dzg=0.1, ng=9, rmap=GX_RMAP_LOG,
                          rmap_a=float(np.log(100.0) / (nr - 1)), rmap_r0=0.05, softl=0.2, tsoft=1)
        rec, pm = kt_disk(60000, seed=4, rmax=4.5, ndim=3, z0=0.1, dt=0.025)
        if name == "3d-split":
            cfg.flags = GX_FLAG_PLANE_SPLIT
    cfg.pmass = pm
    return cfg, rec


def _fields(gal, nd):
    from galaxy_b200 import GX_GRID_FR, GX_GRID_FT, GX_GRID_FZ, GX_GRID_POT, GX_GRID_MASS
    ks = (GX_GRID_FR, GX_GRID_FT) + ((GX_GRID_FZ,) if nd == 3 else ()) + (GX_GRID_POT,)
    return np.stack([gal.grid(k) for k in ks]).astype(np.float64), gal.grid(GX_GRID_MASS)


def _worker(rank, world, port, outdir, names):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from galaxy_b200 import Galaxy
        from galaxy_b200.dist import RankComm
        comm = RankComm()
        res = {}
        for name in names:
            cfg, rec = _case(name)
            mine = np.ascontiguousarray(rec[rank::world])
            with Galaxy(cfg) as gal:
                comm.attach_host(gal)
                gal.greenm()
                gal.loadup(mine)
                gal.masset()
                gal.findf_polar(True)
                f, m = _fields(gal, cfg.ndim)
                gal.step(3)
                pos = gal.unload()
            res[name] = (f, m, pos)
        np.save(os.path.join(outdir, f"rank{rank}.npy"), np.array([res], dtype=object))
    finally:
        dist.destroy_process_group()


NAMES = ("2d", "3d", "3d-split")


def test_two_ranks_through_the_library_reproduce_one_context(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), NAMES), nprocs=world,
                       join=True, start_method="spawn")
    from galaxy_b200 import Galaxy
    res = [np.load(tmp_path / f"rank{r}.npy", allow_pickle=True)[0] for r in range(world)]
    for name in NAMES:
        cfg, rec = _case(name)
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.loadup(rec)
            gal.masset()
            gal.findf_polar(True)
            f1, m1 = _fields(gal, cfg.ndim)
            gal.step(3)
            pos1 = gal.unload()
        msum = res[0][name][1].astype(np.float64) + res[1][name][1].astype(np.float64)
        assert np.abs(msum - m1).max() <= 1e-6 * np.abs(m1).max(), name
        for r in range(world):
            f, _, pos = res[r][name]
            for t in range(f.shape[0]):
                e = np.linalg.norm(f[t] - f1[t]) / np.linalg.norm(f1[t])
                assert e < 1e-6, (name, r, t, e)
            ref = pos1[r::world]
            d = np.abs(pos - ref).max(axis=1) / np.abs(ref).max()
            assert np.mean(d > 1e-6) < 1e-3 and d.max() < 1e-4, (name, r, d.max())
