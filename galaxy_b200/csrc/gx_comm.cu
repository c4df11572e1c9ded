// gx_comm.cu -- multi-GPU exchange of the mixed path over NCCL.
//
// The reference's MPI overlay decomposes by particles: every rank keeps a
// full copy of the grid, deposits its own particles, reduces the active
// ring range with MIN/MAX (SRC/lib15_mpi/massum.f:54-65) and sums the
// Fourier coefficients of the active harmonics after its local transform
// (SRC/lib15_mpi/p2manlp.f:164-233, p3manlp.f:102); every rank then runs
// the radial contraction and synthesis redundantly.  Here the same two
// exchanges run on the context stream: an all-reduce (min, max) of the
// ring range before the forward transform and an all-reduce (sum) of the
// forward spectrum after it.  NCCL is loaded at run time (dlopen of
// libnccl.so.2), so the library shares the copy a host process (e.g. torch)
// already has and has no link-time dependency on it.
#include <dlfcn.h>
#include <nccl.h>
#include <string.h>

#include <mutex>

#include "gx_common.cuh"

namespace {
struct NcclApi {
    void* h = nullptr;
    decltype(&ncclGetUniqueId) getUniqueId = nullptr;
    decltype(&ncclCommInitRank) commInitRank = nullptr;
    decltype(&ncclAllReduce) allReduce = nullptr;
    decltype(&ncclCommDestroy) commDestroy = nullptr;
    decltype(&ncclGetErrorString) errorString = nullptr;
    std::string err;
};

NcclApi* nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* names[] = {"libnccl.so.2", "libnccl.so"};
        for (const char* nm : names) {
            api.h = dlopen(nm, RTLD_NOW | RTLD_GLOBAL);
            if (api.h) break;
        }
        if (!api.h) {
            api.err = "libnccl.so.2 not found";
            return;
        }
        api.getUniqueId = (decltype(api.getUniqueId))dlsym(api.h, "ncclGetUniqueId");
        api.commInitRank = (decltype(api.commInitRank))dlsym(api.h, "ncclCommInitRank");
        api.allReduce = (decltype(api.allReduce))dlsym(api.h, "ncclAllReduce");
        api.commDestroy = (decltype(api.commDestroy))dlsym(api.h, "ncclCommDestroy");
        api.errorString = (decltype(api.errorString))dlsym(api.h, "ncclGetErrorString");
        if (!api.getUniqueId || !api.commInitRank || !api.allReduce || !api.commDestroy) {
            api.err = "NCCL symbols missing";
            api.h = nullptr;
        }
    });
    return api.h ? &api : nullptr;
}
}  // namespace

#define GX_NCCL(ctx, call)                                                         \
    do {                                                                           \
        ncclResult_t r_ = (call);                                                  \
        if (r_ != ncclSuccess) {                                                   \
            NcclApi* a_ = nccl();                                                  \
            (ctx)->err = std::string("NCCL: ") +                                   \
                         (a_ && a_->errorString ? a_->errorString(r_) : "error");  \
            return GX_ERR_CUDA;                                                    \
        }                                                                          \
    } while (0)

extern "C" int gx_comm_unique_id(char* id128) {
    if (!id128) return GX_ERR_ARG;
    NcclApi* a = nccl();
    if (!a) return GX_ERR_STATE;
    ncclUniqueId id;
    if (a->getUniqueId(&id) != ncclSuccess) return GX_ERR_CUDA;
    memcpy(id128, &id, sizeof id);
    return GX_OK;
}

extern "C" int gx_comm_init(GxCtx* c, const char* id128, int nranks, int rank) {
    if (!c || !id128 || nranks < 1 || rank < 0 || rank >= nranks) return GX_ERR_ARG;
    if (c->fp64) return c->err = "the multi-GPU exchange runs on the mixed path", GX_ERR_ARG;
    NcclApi* a = nccl();
    if (!a) return c->err = "NCCL unavailable", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    ncclUniqueId id;
    memcpy(&id, id128, sizeof id);
    ncclComm_t comm = nullptr;
    GX_NCCL(c, a->commInitRank(&comm, nranks, id, rank));
    c->comm = comm;
    c->host_fn = nullptr;
    c->nranks = nranks;
    c->rank = rank;
    return GX_OK;
}

// NCCL is loaded only when a communicator is bound: loading the system copy
// into a process that later imports a framework bundling a newer libnccl.so.2
// would shadow that copy
void gx_comm_destroy(GxCtx* c) {
    if (!c->comm) return;
    NcclApi* a = nccl();
    if (a) a->commDestroy((ncclComm_t)c->comm);
    c->comm = nullptr;
}

extern "C" int gx_comm_host(GxCtx* c, int nranks, int rank, gx_host_reduce_fn fn, void* user) {
    if (!c || !fn || nranks < 1 || rank < 0 || rank >= nranks) return GX_ERR_ARG;
    if (c->fp64) return c->err = "the multi-GPU exchange runs on the mixed path", GX_ERR_ARG;
    gx_comm_destroy(c);
    c->host_fn = fn;
    c->host_user = user;
    c->nranks = nranks;
    c->rank = rank;
    return GX_OK;
}

// one exchange through the host: device -> host, the caller's reduction,
// host -> device (all on the context stream, synchronised)
static int host_reduce(GxCtx* c, void* dptr, int64_t count, int dtype, int op) {
    const size_t bytes = (size_t)count * 4;
    if (c->host_buf.size() < bytes) c->host_buf.resize(bytes);
    void* h = c->host_buf.data();
    GX_CUDA(c, cudaMemcpyAsync(h, dptr, bytes, cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->host_fn(c->host_user, op, dtype, h, count) != 0)
        return c->err = "the host reduction of the ranks failed", GX_ERR_STATE;
    GX_CUDA(c, cudaMemcpyAsync(dptr, h, bytes, cudaMemcpyHostToDevice, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

// MIN/MAX of the 1-based active ring range (massum.f:54-65)
int gx_comm_reduce_range(GxCtx* c) {
    if (c->nranks < 2) return GX_OK;
    if (c->host_fn) {
        int rc = host_reduce(c, c->jrk_d, 1, GX_DT_INT32, GX_OP_MIN);
        return rc ? rc : host_reduce(c, c->jrk_d + 1, 1, GX_DT_INT32, GX_OP_MAX);
    }
    if (!c->comm) return GX_OK;
    NcclApi* a = nccl();
    GX_NCCL(c, a->allReduce(c->jrk_d, c->jrk_d, 1, ncclInt32, ncclMin, (ncclComm_t)c->comm,
                            c->stream));
    GX_NCCL(c, a->allReduce(c->jrk_d + 1, c->jrk_d + 1, 1, ncclInt32, ncclMax,
                            (ncclComm_t)c->comm, c->stream));
    return GX_OK;
}

// MIN/MAX of the planes holding mass (the step's own solve skips the rest)
int gx_comm_reduce_planes(GxCtx* c, int32_t* zr) {
    if (c->nranks < 2) return GX_OK;
    if (c->host_fn) {
        int rc = host_reduce(c, zr, 1, GX_DT_INT32, GX_OP_MIN);
        return rc ? rc : host_reduce(c, zr + 1, 1, GX_DT_INT32, GX_OP_MAX);
    }
    if (!c->comm) return GX_OK;
    NcclApi* a = nccl();
    GX_NCCL(c, a->allReduce(zr, zr, 1, ncclInt32, ncclMin, (ncclComm_t)c->comm, c->stream));
    GX_NCCL(c, a->allReduce(zr + 1, zr + 1, 1, ncclInt32, ncclMax, (ncclComm_t)c->comm, c->stream));
    return GX_OK;
}

static int reduce_sum_f32(GxCtx* c, float* p, size_t count) {
    if (c->nranks < 2) return GX_OK;
    if (c->host_fn) return host_reduce(c, p, (int64_t)count, GX_DT_FLOAT32, GX_OP_SUM);
    if (!c->comm) return GX_OK;
    NcclApi* a = nccl();
    GX_NCCL(c, a->allReduce(p, p, count, ncclFloat32, ncclSum, (ncclComm_t)c->comm, c->stream));
    return GX_OK;
}

// sum of the forward spectrum over ranks (p2manlp.f:208, p3manlp.f:102)
int gx_comm_reduce_spectrum(GxCtx* c) {
    return reduce_sum_f32(c, reinterpret_cast<float*>(c->specS),
                          (size_t)4 * c->spec.nact * c->g.nkz * c->g.nr);
}

// the plane split's exchange: every rank contracted its own vertical
// wavenumbers and left the others zero, so the sum over ranks is every
// rank's full contracted spectrum (p3convp.f:276-326 sends and receives
// the planes)
int gx_comm_reduce_conv(GxCtx* c) {
    return reduce_sum_f32(c, reinterpret_cast<float*>(c->specO),
                          (size_t)4 * 4 * c->spec.nact * c->g.nkz * c->g.nr);
}

bool gx_plane_split(const GxCtx* c) {
    return (c->cfg.flags & GX_FLAG_PLANE_SPLIT) && c->nranks > 1 && c->g.ndim == 3 &&
           (c->comm || c->host_fn);
}
