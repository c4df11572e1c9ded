"""The particle decomposition across ranks, on CPU with two gloo ranks.

Each rank deposits its own share of the particles (the oracle's massgn +
scaled); the ranks then reduce the active ring range with MIN/MAX and the
grid with SUM, as gx_comm.cu does on the device (there the sum is taken
over the forward spectrum, a linear function of the mass).  The reduced
mass and ring range must equal the single-rank ones of all the particles,
and the field of the reduced mass the single-rank field; the field is
linear in the mass, so the sum of the ranks' fields is that field too.
Also checked: RankComm's broadcast of the 128-byte communicator id, its
barrier and its max over ranks (the bench's device time of a step)."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _cfgs():
    from galaxy_b200 import make_config, GX_RMAP_LOG, GX_RMAP_STDPOL
    c2 = make_config(2, 32, 64, ng=5, rmap=GX_RMAP_STDPOL, softl=1.0, tsoft=1, pmass=1.0)
    c3 = make_config(3, 24, 32, ngz=15, dzg=0.1, ng=5, rmap=GX_RMAP_LOG,
                     rmap_a=float(np.log(100.0) / 23), rmap_r0=0.05, softl=0.2, tsoft=1,
                     pmass=1.0)
    return c2, c3


def _worker(rank, world, port, outdir):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from galaxy_b200.dist import RankComm
        from galaxy_b200.disk import kt_disk
        from oracle import oracle as ox
        comm = RankComm()
        res = {}
        # communicator id: rank 0's bytes reach every rank
        uid = bytes(range(128)) if rank == 0 else bytes(128)
        res["uid_ok"] = comm.broadcast_bytes(uid) == bytes(range(128))
        comm.barrier()
        res["max"] = comm.max(10.0 + rank)
        for name, cfg in zip(("2d", "3d"), _cfgs()):
            nd = cfg.ndim
            rec, pm = kt_disk(4000, seed=5, rmax=4.0, ndim=nd, z0=0.1, dt=0.025)
            cfg.pmass = pm
            pos = rec.astype(np.float64)
            mine = pos[rank::world]
            m_loc, jrk_loc = ox.masset(cfg, mine, prec=64)
            m_sum = comm.sum_array(m_loc)
            jrk = comm.ring_range(jrk_loc)
            m_all, jrk_all = ox.masset(cfg, pos, prec=64)
            G = ox.green(cfg, 64)
            f_red = ox.findf(cfg, G, m_sum, lpot=True, jrk=jrk, prec=64)
            f_all = ox.findf(cfg, G, m_all, lpot=True, jrk=tuple(jrk_all), prec=64)
            f_loc = ox.findf(cfg, G, m_loc, lpot=True, jrk=jrk, prec=64)
            f_sum = comm.sum_array(f_loc)
            scale = np.abs(f_all).max()
            res[name] = dict(
                mass=float(np.abs(m_sum - m_all).max() / np.abs(m_all).max()),
                jrk=(tuple(jrk), tuple(int(v) for v in jrk_all)),
                field=float(np.abs(f_red - f_all).max() / scale),
                linear=float(np.abs(f_sum - f_all).max() / scale))
        np.save(os.path.join(outdir, f"rank{rank}.npy"), np.array([res], dtype=object))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_single_rank_solve(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        res = np.load(tmp_path / f"rank{r}.npy", allow_pickle=True)[0]
        assert res["uid_ok"]
        assert res["max"] == 11.0
        for name in ("2d", "3d"):
            d = res[name]
            assert d["mass"] < 1e-13, (name, d)
            assert d["jrk"][0] == d["jrk"][1], (name, d)
            assert d["field"] < 1e-12, (name, d)
            assert d["linear"] < 1e-12, (name, d)
