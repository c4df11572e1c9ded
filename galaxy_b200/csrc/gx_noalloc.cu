// gx_noalloc.cu -- mass assignment that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they deposit
// mass: a host code that owns a fixed device memory pool and forbids any
// other allocation (a Fortran driver that places its own arrays), a time
// loop that must not stall on the allocator, or code running where
// cudaMalloc is not permitted.  gx_massgn_noalloc gives them massgn
// (SRC/lib15/massgn.f:68-89, 140-172, with scaled.f:89-92) on their own
// device buffers: the caller passes the particle records and the output
// mesh; the only working memory is the file-scope array g_massgn_scratch
// below, a fixed 2^22-cell fixed-point accumulator (32 MiB) that every GPU
// loading this library holds until the process exits.  The call uses no
// cudaMalloc, cudaFree or other allocating routine.
#include <mutex>

#include "gx_common.cuh"

#define GX_NOALLOC_MAX_MESH (1 << 22)

// one int64 fixed-point (2^-32 of a particle) accumulator per mesh cell
static __device__ __align__(256) unsigned long long g_massgn_scratch[GX_NOALLOC_MAX_MESH];

__global__ void k_na_clear(unsigned long long* __restrict__ acc, int mesh) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < mesh) acc[i] = 0ull;
}

__global__ void k_na_deposit(DevGeo g, const float* __restrict__ coords, int64_t n,
                             unsigned long long* __restrict__ acc) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nw = 2 * g.ndim;
    const float* q = coords + i * nw;
    const CellW c = gx_cell(g, q[0], q[1], (g.ndim == 3) ? q[2] : 0.f, false);
    if (c.key < 0) return;
    float w[8];
    int ic[8];
    gx_weights(g, c, w);
    const int nc = gx_corners(g, c.key, ic);
    for (int k = 0; k < nc; k++) {
        if (ic[k] < 0) continue;
        const long long v = __double2ll_rn((double)w[k] * 4294967296.0);
        atomicAdd(&acc[ic[k]], (unsigned long long)v);  // two's complement sum
    }
}

__global__ void k_na_finish(const unsigned long long* __restrict__ acc, int mesh, float pmass,
                            float* __restrict__ mass) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < mesh) mass[i] = (float)((double)(long long)acc[i] * (1.0 / 4294967296.0)) * pmass;
}

static std::mutex g_na_mutex;
static void* g_na_ptr[256];

// failures are reported by return code only (no message buffer to fill)
static inline int na_fail(int rc, const char*) { return rc; }

// the caller's current device, put back on every return path
struct NaDeviceGuard {
    int prev = -1;
    NaDeviceGuard() {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~NaDeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Device address of the scratch array on the current device, looked up once
// per device.  Host code must not pass g_massgn_scratch itself to a kernel:
// on the host that name is only a stand-in for the device symbol.  With lazy
// module loading (CUDA's default) the first lookup on a device also loads
// this file's module, which is when that device reserves the array.  The
// cached address is only valid until the device is reset: a caller that
// runs cudaDeviceReset between calls is not supported.
static int na_scratch(int dev, void** ptr) {
    if (dev < 0 || dev >= 256) return na_fail(GX_ERR_CUDA, "gx_massgn_noalloc: device out of range");
    std::lock_guard<std::mutex> lk(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_massgn_scratch);
        if (e != cudaSuccess || !p)
            return na_fail(GX_ERR_CUDA, "gx_massgn_noalloc: cudaGetSymbolAddress failed");
        g_na_ptr[dev] = p;
    }
    *ptr = g_na_ptr[dev];
    return GX_OK;
}

// one launch, its own launch status (not an error left pending by earlier,
// unrelated work of the process)
static int na_launch(const void* fn, unsigned grid, cudaStream_t st, void** args) {
    if (grid == 0) return GX_OK;
    cudaError_t e = cudaLaunchKernel(fn, dim3(grid), dim3(256), args, 0, st);
    return (e == cudaSuccess) ? GX_OK : na_fail(GX_ERR_CUDA, "gx_massgn_noalloc: launch failed");
}

extern "C" int gx_massgn_noalloc(const GxConfig* cfg, const float* d_coords, int64_t n,
                                 float* d_mass, void* stream) {
    if (!cfg || n < 0 || !d_mass || (n > 0 && !d_coords))
        return na_fail(GX_ERR_ARG, "gx_massgn_noalloc: null argument");
    if (cfg->precision != GX_PREC_MIXED)
        return na_fail(GX_ERR_ARG, "gx_massgn_noalloc: mixed-precision cells only");
    if (cfg->flags & GX_FLAG_QUADRATIC)
        return na_fail(GX_ERR_ARG, "gx_massgn_noalloc: the linear scheme only");
    GxCtx tmp;
    tmp.cfg = *cfg;
    std::string err;
    int rc = setgrd(cfg, &tmp.geo, err);
    if (rc) return na_fail(rc, "gx_massgn_noalloc: invalid grid configuration");
    fill_devgeo(&tmp);
    DevGeo g = tmp.g;
    if (g.mesh > GX_NOALLOC_MAX_MESH)
        return na_fail(GX_ERR_RANGE, "gx_massgn_noalloc: mesh larger than 4194304 cells");
    NaDeviceGuard guard;
    if (cudaSetDevice(cfg->device) != cudaSuccess)
        return na_fail(GX_ERR_CUDA, "gx_massgn_noalloc: cannot select the device");
    void* p = nullptr;
    rc = na_scratch(cfg->device, &p);
    if (rc) return rc;
    unsigned long long* acc = (unsigned long long*)p;
    cudaStream_t st = (cudaStream_t)stream;
    int mesh = g.mesh;
    float pmass = cfg->pmass;
    const unsigned gm = (unsigned)((mesh + 255) / 256);
    void* a_clear[] = {&acc, &mesh};
    rc = na_launch((const void*)k_na_clear, gm, st, a_clear);
    if (rc) return rc;
    if (n > 0) {
        void* a_dep[] = {&g, &d_coords, &n, &acc};
        rc = na_launch((const void*)k_na_deposit, (unsigned)((n + 255) / 256), st, a_dep);
        if (rc) return rc;
    }
    void* a_fin[] = {&acc, &mesh, &pmass, &d_mass};
    rc = na_launch((const void*)k_na_finish, gm, st, a_fin);
    if (rc) return rc;
    if (!stream && cudaStreamSynchronize(st) != cudaSuccess)
        return na_fail(GX_ERR_CUDA, "gx_massgn_noalloc: kernel failed");
    return GX_OK;
}
