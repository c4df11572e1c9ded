"""Host side of the particle decomposition across ranks (one process per GPU).

The reference's MPI overlay splits the particles among ranks, each rank
keeping a full copy of the grid (SRC/lib15_mpi/massum.f:54-65,
p2manlp.f:164-233, p3manlp.f:102).  Here torch.distributed carries the
host-side plumbing (rank 0's NCCL id to every rank, barriers, the max over
ranks of the device-timed step), and the library's own NCCL communicator
carries the per-step exchange (gx_comm.cu: MIN/MAX of the active ring range,
SUM of the forward spectrum, and with the plane split SUM of the contracted
spectra); or, for ranks on a CPU process group, the same exchanges run
through the host (attach_host, gx_comm_host).
"""


class RankComm:
    """torch.distributed helpers of a job with one rank per GPU; on a CPU
    process group (gloo) the reductions run on host tensors."""

    def __init__(self):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.device = "cuda" if dist.get_backend() == "nccl" else "cpu"

    def attach(self, gal):
        """Bind a Galaxy context to the ranks (gx_comm_unique_id on rank 0,
        broadcast, gx_comm_init on every rank)."""
        gal.set_comm(self)

    def attach_host(self, gal):
        """Bind a Galaxy context to the ranks through the host (gx_comm_host):
        the library's exchanges become all-reduces of host tensors over this
        process group (e.g. gloo)."""
        import ctypes as C
        import numpy as np
        from ._abi import GX_OP_SUM, GX_OP_MIN, GX_DT_INT32
        torch, dist = self.torch, self.dist
        ops = {GX_OP_SUM: dist.ReduceOp.SUM, GX_OP_MIN: dist.ReduceOp.MIN}

        def reduce(user, op, dtype, data, count):
            try:
                ct = C.c_int32 if dtype == GX_DT_INT32 else C.c_float
                arr = np.ctypeslib.as_array((ct * int(count)).from_address(data))
                t = torch.from_numpy(arr)  # the library's host buffer, reduced in place
                dist.all_reduce(t, op=ops.get(op, dist.ReduceOp.MAX))
                return 0
            except Exception:  # reported by the library as GX_ERR_STATE
                return 1

        fn = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64)(reduce)
        gal._host_reduce = fn  # the callback lives as long as the context
        gal._chk(gal._L.gx_comm_host(gal._h, self.world, self.rank, fn, None))

    def broadcast_bytes(self, b):
        obj = [bytes(b) if self.rank == 0 else None]
        self.dist.broadcast_object_list(obj, src=0)
        return obj[0]

    def barrier(self):
        self.dist.barrier()

    def max(self, v):
        t = self.torch.tensor([float(v)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_array(self, a):
        """element-wise sum over ranks of a numpy array (FP64 on the wire)"""
        import numpy as np
        # a copy: the reduction runs in place and must not touch the caller's array
        t = self.torch.from_numpy(np.array(a, np.float64, copy=True)).to(self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def ring_range(self, jrk):
        """MIN/MAX over ranks of the 1-based active ring range (massum.f:54-65)"""
        lo = self.torch.tensor([int(jrk[0])], dtype=self.torch.int64, device=self.device)
        hi = self.torch.tensor([int(jrk[1])], dtype=self.torch.int64, device=self.device)
        self.dist.all_reduce(lo, op=self.dist.ReduceOp.MIN)
        self.dist.all_reduce(hi, op=self.dist.ReduceOp.MAX)
        return int(lo.item()), int(hi.item())
