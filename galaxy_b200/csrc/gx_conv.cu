// gx_conv.cu -- radial contraction of the 3D field solve with the Green
// table streamed through shared memory by bulk copies.
//
// p3conv.f:137-230: for every active harmonic m, vertical wavenumber kz and
// field type t (radial, azimuthal, vertical, potential) the output spectrum
// at ring ir is sum_is G_t[m][kz][is][ir] * S[m][kz][is] with the cc/cs/sc/ss
// mixing of the type.  Each Green entry is used for 4 MACs and read once per
// step, so the kernel's job is to keep the HBM pipe full.
//
// Persistent CTAs of 8 consumer warps and 1 producer warp.  Work items are
// (m, kz) pairs dealt round-robin to CTAs.  The producer walks the same tile
// sequence as the consumers -- items, then valid types, then chunks of rows
// (source rings js..ks) of the nr x nr matrix -- and copies each tile, a
// contiguous block of rows, into a ring of NST shared-memory stages with
// cp.async.bulk; an mbarrier per stage counts the bytes in (full) and the
// consumer warps out (empty).  The item's spectrum (nr float4) comes the same
// way into a double buffer.  Every wait is bounded: on time-out the CTA
// raises the device error word, drains its own copies in flight (bounded)
// and returns; a consumer warp that timed out keeps taking the named
// barriers so that its partners are not left waiting.
#include <algorithm>

#include "gx_bulk.cuh"
#include "gx_common.cuh"

namespace {
constexpr int MAXST = 8;                      // most stages in the ring
template <int NCW>
__device__ __forceinline__ void consumer_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(NCW * 32) : "memory");
}

struct ConvArgs {
    DevGeo g;
    int nact, tmask, nitems, rows_per_tile, nst;
    int nkr, ksplit, krank;  // plane split: this rank's kz are krank + ksplit q, q < nkr
    const float* G;
    const float4* S;
    float4* O;
    const int32_t* jrk;
    int32_t* errword;
    int act_m[260];  // m of each active harmonic
};

// the type t of item (a, kz) has a Green matrix (p3conv.f:173-226)
__device__ __forceinline__ bool type_valid(const DevGeo& g, int t, int m, int k) {
    if (t == 1) return (m >= 1) && (m <= min(g.ng, g.mmax - 1) - 1);
    if (t == 2) return (k >= 1) && (k <= g.ngz - 1);
    return true;
}
}  // namespace

// NJ = ceil(nr / 128): groups of 128 output rings per lane (4 per lane each)
template <int NJ, int NCW, int MINB>
__global__ void __launch_bounds__((NCW + 1) * 32, MINB) k_conv_bulk(ConvArgs A) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const DevGeo& g = A.g;
    const int nr = g.nr, nkz = g.nkz;
    const int R = A.rows_per_tile, NST = A.nst;
    const size_t stage_floats = (size_t)R * nr;
    float* stage = reinterpret_cast<float*>(smraw);
    float4* part = reinterpret_cast<float4*>(stage + NST * stage_floats);   // [NCW][nr]
    float4* Sbuf = part + NCW * nr;                                          // [2][nr]
    uint64_t* full = reinterpret_cast<uint64_t*>(Sbuf + 2 * nr);
    uint64_t* empty = full + MAXST;
    uint64_t* sfull = empty + MAXST;   // [2] spectrum of the item in
    uint64_t* sempty = sfull + 2;      // [2] spectrum no longer read
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // with no mass on the grid (ks < js) no tile is copied and every output is 0
    const int js = max(A.jrk[0], 1) - 1, ks = min(A.jrk[1], nr) - 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCW);
        }
        for (int s = 0; s < 2; s++) {
            mbar_init(&sfull[s], 1);
            mbar_init(&sempty[s], NCW);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (warp == NCW) {
        // ------------------------------------------------------------ producer
        if (lane != 0) return;
        int tile = 0, li = 0, s_issued = 0;
        bool ok = true;
        for (int it = blockIdx.x; ok && it < A.nitems; it += gridDim.x, li++) {
            const int a = it / A.nkr, k = A.krank + A.ksplit * (it - a * A.nkr), m = A.act_m[a];
            // the item's spectrum into its half of the double buffer
            const int sb = li & 1;
            if (li >= 2 && !mbar_wait(&sempty[sb], ((li >> 1) - 1) & 1)) {
                ok = false;
                break;
            }
            mbar_expect_tx(&sfull[sb], (uint32_t)(nr * sizeof(float4)));
            bulk_g2s(Sbuf + sb * nr, A.S + ((size_t)a * nkz + k) * nr, (uint32_t)(nr * sizeof(float4)),
                     &sfull[sb]);
            s_issued++;
            for (int t = 0; ok && t < 4; t++) {
                if (!((A.tmask >> t) & 1) || !type_valid(g, t, m, k)) continue;
                const float* Gt = A.G + ((((size_t)t * g.ng + m) * nkz + k) * nr) * (size_t)nr;
                for (int r0 = js; r0 <= ks; r0 += R) {
                    const int rows = min(R, ks - r0 + 1);
                    const int s = tile % NST;
                    if (tile >= NST && !mbar_wait(&empty[s], ((tile / NST) - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    const uint32_t bytes = (uint32_t)(rows * nr * sizeof(float));
                    mbar_expect_tx(&full[s], bytes);
                    bulk_g2s(stage + s * stage_floats, Gt + (size_t)r0 * nr, bytes, &full[s]);
                    tile++;
                }
            }
        }
        if (!ok) {
            atomicExch(A.errword, 3);
            // drain the copies that may still be in flight (the latest phase of each buffer)
            for (int q = max(0, tile - NST); q < tile; q++) mbar_wait(&full[q % NST], (q / NST) & 1);
            for (int q = max(0, s_issued - 2); q < s_issued; q++) mbar_wait(&sfull[q & 1], (q >> 1) & 1);
        }
        return;
    }

    // ---------------------------------------------------------------- consumers
    int tile = 0, li = 0;
    bool dead = false;
    for (int it = blockIdx.x; it < A.nitems; it += gridDim.x, li++) {
        const int a = it / A.nkr, k = A.krank + A.ksplit * (it - a * A.nkr), m = A.act_m[a];
        const float4* Sb = Sbuf + (li & 1) * nr;
        if (!dead && !mbar_wait(&sfull[li & 1], (li >> 1) & 1)) {
            atomicExch(A.errword, 3);
            dead = true;
        }
        for (int t = 0; t < 4; t++) {
            if (!((A.tmask >> t) & 1)) continue;
            // ring-major output [t][ir][kz][a]: the synthesis reads a ring's
            // spectrum as one contiguous block
            const size_t ost = (size_t)nkz * A.nact;
            float4* out = A.O + ((size_t)t * nr * nkz + k) * A.nact + a;
            if (!type_valid(g, t, m, k)) {
                for (int i = threadIdx.x; i < nr; i += NCW * 32) out[i * ost] = make_float4(0, 0, 0, 0);
                continue;
            }
            float4 acc[NJ][4];
#pragma unroll
            for (int j = 0; j < NJ; j++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[j][q] = make_float4(0, 0, 0, 0);
            for (int r0 = js; r0 <= ks; r0 += R) {
                const int rows = min(R, ks - r0 + 1);
                const int s = tile % NST;
                tile++;
                if (dead) continue;
                if (!mbar_wait(&full[s], ((tile - 1) / NST) & 1)) {
                    atomicExch(A.errword, 3);
                    dead = true;
                    continue;
                }
                const float* st = stage + s * stage_floats;
                // this warp's rows of the tile (warp, warp + NCW, ...) into
                // registers first, so that the stage goes back to the
                // producer before the arithmetic: more of the table stays in
                // flight while the sums run
                static_assert(NJ == 1, "one group of 128 output rings per lane");
                constexpr int RW = 128 / NCW;  // rows per warp at most (R <= 128)
                float4 gr[RW];
#pragma unroll
                for (int u = 0; u < RW; u++) {
                    const int r = warp + NCW * u;
                    gr[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (r < rows && 4 * lane < nr)
                        gr[u] = *reinterpret_cast<const float4*>(st + (size_t)r * nr + 4 * lane);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[s]);
#pragma unroll
                for (int u = 0; u < RW; u++) {
                    const int r = warp + NCW * u;
                    if (r >= rows) break;
                    const float4 sv = Sb[r0 + r];
                    const float gv[4] = {gr[u].x, gr[u].y, gr[u].z, gr[u].w};
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float gq = gv[q];
                        float4& o = acc[0][q];
                        if (t == 0 || t == 3) {
                            o.x += gq * sv.x; o.y += gq * sv.y;
                            o.z += gq * sv.z; o.w += gq * sv.w;
                        } else if (t == 1) {
                            o.x += gq * sv.z; o.z -= gq * sv.x;
                            o.y += gq * sv.w; o.w -= gq * sv.y;
                        } else {
                            o.x += gq * sv.y; o.y -= gq * sv.x;
                            o.z += gq * sv.w; o.w -= gq * sv.z;
                        }
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NJ; j++) {
                const int ir0 = 4 * lane + 128 * j;
                if (ir0 >= nr) continue;
#pragma unroll
                for (int q = 0; q < 4; q++) part[warp * nr + ir0 + q] = acc[j][q];
            }
            consumer_sync<NCW>();
            for (int i = threadIdx.x; i < nr; i += NCW * 32) {
                float4 v = part[i];
#pragma unroll
                for (int w = 1; w < NCW; w++) {
                    const float4 p = part[w * nr + i];
                    v.x += p.x; v.y += p.y; v.z += p.z; v.w += p.w;
                }
                out[i * ost] = v;
            }
            consumer_sync<NCW>();
        }
        __syncwarp();
        if (lane == 0 && !dead) mbar_arrive(&sempty[li & 1]);
    }
}

// host side: true when the bulk path handles this geometry
bool gx_conv_bulk_ok(const DevGeo& g) { return g.ndim == 3 && g.nr % 4 == 0 && g.nr <= 128; }

int gx_conv_bulk(GxCtx* c, int nact, int tmask) {
    const DevGeo& g = c->g;
    int dev_sms = 0, smem_max = 0;
    GX_CUDA(c, cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->dev));
    GX_CUDA(c, cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
    // 8 consumer warps; tiles of whole 64 KB matrices (or 64 KB of rows): a
    // sweep on B200 found the contraction's rate set by the size of each bulk
    // copy (16 KB: 2.9 TB/s, 32 KB: 3.5, 64 KB: 3.95), not by the stage count
    constexpr int ncw = 8;
    const size_t fixed = sizeof(float4) * (size_t)g.nr * (ncw + 2) + (2 * MAXST + 4) * sizeof(uint64_t);
    const int R = std::min(g.nr, (int)(65536 / (g.nr * sizeof(float))));
    const size_t stage_bytes = (size_t)R * g.nr * sizeof(float);
    const size_t budget = std::min<size_t>((size_t)smem_max - fixed, 204800);
    int nst = (int)std::min<size_t>(MAXST, budget / stage_bytes);
    if (nst < 2) return c->err = "radial contraction: shared memory too small", GX_ERR_ARG;
    const size_t smem = nst * stage_bytes + fixed;
    ConvArgs A;
    A.g = g;
    A.nact = nact;
    A.tmask = tmask;
    // with the plane split this rank contracts the kz with kz mod nranks ==
    // rank (p3convp.f:180-190: the planes iz with mod(iz - jz, numprocs) ==
    // myid, jz = 1) and leaves the rest of the output zero for the ranks' sum
    const bool split = gx_plane_split(c);
    A.ksplit = split ? c->nranks : 1;
    A.krank = split ? c->rank : 0;
    A.nkr = (g.nkz - A.krank + A.ksplit - 1) / A.ksplit;
    A.nitems = nact * A.nkr;
    if (split)
        GX_CUDA(c, cudaMemsetAsync(c->specO, 0, sizeof(float4) * 4 * (size_t)nact * g.nkz * g.nr, c->stream));
    if (A.nitems == 0) return GX_OK;
    A.rows_per_tile = R;
    A.nst = nst;
    A.G = c->green32;
    A.S = reinterpret_cast<const float4*>(c->specS);
    A.O = reinterpret_cast<float4*>(c->specO);
    A.jrk = c->jrk_d;
    A.errword = c->errword;
    for (int i = 0; i < 260; i++) A.act_m[i] = (i < nact) ? c->spec.m[i] : 0;
    const int grid = std::min(A.nitems, dev_sms);
    GX_CUDA(c, cudaFuncSetAttribute(k_conv_bulk<1, ncw, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_conv_bulk<1, ncw, 1><<<grid, (ncw + 1) * 32, smem, c->stream>>>(A);
    GX_LAUNCHED(c);
    return GX_OK;
}
