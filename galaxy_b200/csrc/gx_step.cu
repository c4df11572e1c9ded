// gx_step.cu -- particle side of the mixed-precision path.
//
//   k_push         one pass per step over the particles in row-sorted order
//                  (getacc + stpgrp + the new cell key of massgn's weight
//                  call): old cell and weights (weight.f:61-101, 196-250),
//                  gather of the float4 field at the 4/8 corners
//                  (grdacc.f:40-84, 189-218), rigid halo (getacc.f:103-122,
//                  frhalo.f:55-56), v += a, x += v (stpgrp.f:26-32), off-grid
//                  test (offgrd.f:51-77), new ring-plane row of the key.
//   radix sort     LSD sort of the row digits of the cell keys
//                  (hist / per-digit scan / stable scatter), stable so the
//                  deposit order is fixed by the previous pass.
//   k_deposit      massgn (massgn.f:68-89, 140-172) as an owner-computes
//                  reduction: one work item = up to DEP_CH particles of one
//                  base row; warps group their 32 particles by spoke with
//                  __match_any_sync, the group leader sums the weights in
//                  lane order into warp-private shared-memory bins, bins are
//                  combined in warp order.  No atomics on floats; the result
//                  is bitwise reproducible run to run.
//   k_mass_combine every output row sums the partial rows of the base rows
//                  that feed it (same row, plane below, ring below, both) in
//                  a fixed order and applies pmass (scaled.f:89-92).
#include <algorithm>

#include "gx_common.cuh"

#define DEP_CH 2048
#define SORT_TILE 4096
#define SORT_THREADS 256
#define SORT_ITEMS (SORT_TILE / SORT_THREADS)

// ---------------------------------------------------------------------------
// radix sort of 32-bit row keys with int32 payload
__global__ void k_sort_hist(const uint32_t* __restrict__ keys, int64_t n, int shift, int bits,
                            uint32_t* __restrict__ hist, int ntile) {
    __shared__ uint32_t h[256];
    const int nb = 1 << bits;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * SORT_TILE;
    const uint32_t mask = nb - 1;
    for (int it = 0; it < SORT_ITEMS; it++) {
        int64_t i = base + it * SORT_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & mask], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < nb; d += blockDim.x) hist[(size_t)d * ntile + blockIdx.x] = h[d];
}

// exclusive scan of hist[d][0..ntile) for digit d = blockIdx.x; dtotal[d] = sum
__global__ void k_sort_scan(uint32_t* __restrict__ hist, int ntile, uint32_t* __restrict__ dtotal) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    uint32_t* h = hist + (size_t)blockIdx.x * ntile;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < ntile; base += blockDim.x) {
        int i = base + threadIdx.x;
        uint32_t v = (i < ntile) ? h[i] : 0;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t s = (lane < nw) ? wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            if (lane < nw) wsum[lane] = s;
        }
        __syncthreads();
        uint32_t wpre = (warp > 0) ? wsum[warp - 1] : 0;
        uint32_t excl = carry + wpre + x - v;
        if (i < ntile) h[i] = excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += wsum[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) dtotal[blockIdx.x] = carry;
}

// stable scatter of one tile; warp w ranks items [w*SORT_TILE/8, ...) in order
__global__ void __launch_bounds__(SORT_THREADS) k_sort_scatter(
    const uint32_t* __restrict__ kin, const int32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    int32_t* __restrict__ vout, int64_t n, int shift, int bits, const uint32_t* __restrict__ hist,
    const uint32_t* __restrict__ dtotal, int ntile) {
    __shared__ uint32_t cnt[SORT_THREADS / 32][256];
    __shared__ uint32_t dbase[256];
    const int nb = 1 << bits;
    const uint32_t mask = nb - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = SORT_THREADS / 32;
    constexpr int PERW = SORT_TILE / NW;  // items per warp
    constexpr int SUB = PERW / 32;        // sub-chunks per warp
    for (int i = threadIdx.x; i < NW * 256; i += blockDim.x) (&cnt[0][0])[i] = 0;
    // digit bases: exclusive scan of dtotal (small, done by warp 0 serially in lanes)
    if (warp == 0) {
        uint32_t run = 0;
        for (int d0 = 0; d0 < nb; d0 += 32) {
            int d = d0 + lane;
            uint32_t v = (d < nb) ? dtotal[d] : 0;
            uint32_t x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (d < nb) dbase[d] = run + x - v;
            run += __shfl_sync(0xffffffffu, x, 31);
        }
    }
    __syncthreads();
    const int64_t tbase = (int64_t)blockIdx.x * SORT_TILE + warp * PERW;
    uint32_t key[SUB];
    int32_t val[SUB];
    uint32_t rank[SUB];
#pragma unroll
    for (int s = 0; s < SUB; s++) {
        int64_t i = tbase + s * 32 + lane;
        bool act = i < n;
        key[s] = act ? kin[i] : 0xffffffffu;
        val[s] = act ? (vin ? vin[i] : (int32_t)i) : 0;
        uint32_t d = (key[s] >> shift) & mask;
        uint32_t am = __ballot_sync(0xffffffffu, act);
        uint32_t peers = __match_any_sync(0xffffffffu, act ? d : 0xffffffffu) & am;
        uint32_t before = __popc(peers & ((1u << lane) - 1));
        uint32_t base = act ? cnt[warp][d] : 0;
        rank[s] = base + before;
        __syncwarp();
        if (act && before == 0) cnt[warp][d] = base + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive offsets over warps (in warp order)
    for (int d = threadIdx.x; d < nb; d += blockDim.x) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            uint32_t c = cnt[w][d];
            cnt[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < SUB; s++) {
        int64_t i = tbase + s * 32 + lane;
        if (i < n) {
            uint32_t d = (key[s] >> shift) & mask;
            uint32_t pos = dbase[d] + hist[(size_t)d * ntile + blockIdx.x] + cnt[warp][d] + rank[s];
            kout[pos] = key[s];
            vout[pos] = val[s];
        }
    }
}

// sorts keys_in (row keys, values 0..n-1) -> sb.keys[out], sb.vals[out]; returns out index
static int row_sort(GxCtx* c, const uint32_t* keys_in, int* out_idx) {
    SortBufs& sb = c->sb;
    const int64_t n = c->n;
    const int ntile = (int)((n + SORT_TILE - 1) / SORT_TILE);
    const uint32_t* kin = keys_in;
    const int32_t* vin = nullptr;
    int o = 0;
    int rc0 = gx_phase_mark(c, PH_SORT);
    if (rc0) return rc0;
    for (int p = 0; p < sb.npass; p++) {
        int bits = sb.pass_bits[p], shift = sb.pass_shift[p];
        k_sort_hist<<<ntile, SORT_THREADS, 0, c->stream>>>(kin, n, shift, bits, sb.hist, ntile);
        GX_LAUNCHED(c);
        k_sort_scan<<<1 << bits, 1024, 0, c->stream>>>(sb.hist, ntile, sb.dtotal);
        GX_LAUNCHED(c);
        o = p & 1;
        k_sort_scatter<<<ntile, SORT_THREADS, 0, c->stream>>>(kin, vin, sb.keys[o], sb.vals[o], n,
                                                              shift, bits, sb.hist, sb.dtotal, ntile);
        GX_LAUNCHED(c);
        kin = sb.keys[o];
        vin = sb.vals[o];
    }
    *out_idx = o;
    return GX_OK;
}

// ---------------------------------------------------------------------------
// row starts of the sorted row keys; rowstart[r] = first s with key >= r,
// r = 0 .. nrow + 1 (row nrow collects the particles off the grid)
__global__ void k_rowstart(const uint32_t* __restrict__ keys, int64_t n, int nrow,
                           int32_t* __restrict__ rowstart) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s > n) return;
    int kc = (s < n) ? (int)keys[s] : nrow + 1;
    int kp = (s > 0) ? (int)keys[s - 1] : -1;
    for (int r = kp + 1; r <= kc && r <= nrow + 1; r++) rowstart[r] = (int32_t)s;
}

// work items and the active ring range (single CTA)
__global__ void k_items(const int32_t* __restrict__ rowstart, int nrow, int ngz, int nr,
                        int32_t* __restrict__ rowitem, int32_t* __restrict__ items,
                        int32_t* __restrict__ nitems, int32_t* __restrict__ jrk) {
    __shared__ int32_t wsum[32];
    __shared__ int32_t carry;
    __shared__ int32_t rmin, rmax;
    if (threadIdx.x == 0) {
        carry = 0;
        rmin = 0x7fffffff;
        rmax = -1;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < nrow; base += blockDim.x) {
        int r = base + threadIdx.x;
        int cnt = (r < nrow) ? rowstart[r + 1] - rowstart[r] : 0;
        int v = (cnt + DEP_CH - 1) / DEP_CH;
        if (cnt > 0) {
            atomicMin(&rmin, r);
            atomicMax(&rmax, r);
        }
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int s = (lane < nw) ? wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            if (lane < nw) wsum[lane] = s;
        }
        __syncthreads();
        int excl = carry + ((warp > 0) ? wsum[warp - 1] : 0) + x - v;
        if (r < nrow) {
            rowitem[r] = excl;
            int s0 = rowstart[r];
            for (int q = 0; q < v; q++) {
                int it = excl + q;
                items[3 * it + 0] = r;
                items[3 * it + 1] = s0 + q * DEP_CH;
                items[3 * it + 2] = min(s0 + (q + 1) * DEP_CH, rowstart[r + 1]);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += wsum[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        rowitem[nrow] = carry;
        *nitems = carry;
        // 1-based ring range as massgn tracks it (jrad = j + 1, krad = j + 2)
        if (rmax >= 0) {
            jrk[0] = rmin / ngz + 1;
            jrk[1] = min(rmax / ngz + 2, nr);
        } else {
            jrk[0] = nr;
            jrk[1] = 0;
        }
    }
}

// deterministic owner-computes deposit; smem: bins[8][NW][na] + scratch[8][32][NW]
template <int NW>
__global__ void __launch_bounds__(256) k_deposit(DevGeo g, const int32_t* __restrict__ items,
                                                 const int32_t* __restrict__ nitems,
                                                 const float* __restrict__ P, int64_t cap,
                                                 const int32_t* __restrict__ perm,
                                                 float* __restrict__ stage,
                                                 int32_t* __restrict__ errword) {
    extern __shared__ __align__(16) float sm[];
    const int na = g.na;
    constexpr int NQ = NW / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* bins = sm;                          // [8][NW][na]
    float* scr = sm + 8 * NW * na;             // [8][32][NW]
    float* wb = bins + warp * NW * na;
    float* ws = scr + (warp * 32 + lane) * NW;
    const int nit = *nitems;
    const float* X = P;
    const float* Y = P + cap;
    const float* Z = (g.ndim == 3) ? P + 2 * cap : nullptr;
    for (int item = blockIdx.x; item < nit; item += gridDim.x) {
        const int row = items[3 * item], s0 = items[3 * item + 1], s1 = items[3 * item + 2];
        for (int i = threadIdx.x; i < 8 * NW * na; i += blockDim.x) bins[i] = 0.f;
        __syncthreads();
        const int nsub = (s1 - s0 + 31) >> 5;
        for (int sub = warp; sub < nsub; sub += 8) {
            const int s = s0 + sub * 32 + lane;
            const bool act = s < s1;
            int jt = -1;
            float w[8];
            if (act) {
                const int p = perm[s];
                float z = Z ? Z[p] : 0.f;
                CellW cw = gx_cell(g, X[p], Y[p], z, false);
                if (cw.key < 0 || cw.key / na != row) {
                    atomicExch(errword, 1);
                } else {
                    jt = cw.key - row * na;
                    gx_weights(g, cw, w);
#pragma unroll
                    for (int k = 0; k < NW; k++) ws[k] = w[k];
                }
            }
            const bool ok = jt >= 0;
            const uint32_t am = __ballot_sync(0xffffffffu, ok);
            const uint32_t peers = __match_any_sync(0xffffffffu, ok ? jt : -1) & am;
            __syncwarp();
            if (ok && (peers & ((1u << lane) - 1)) == 0) {
                // leader: sum the group's weights in lane order
                float acc[NW];
#pragma unroll
                for (int k = 0; k < NW; k++) acc[k] = 0.f;
                uint32_t pm = peers;
                while (pm) {
                    int l = __ffs(pm) - 1;
                    pm &= pm - 1;
                    const float* src = scr + (warp * 32 + l) * NW;
#pragma unroll
                    for (int k = 0; k < NW; k++) acc[k] += src[k];
                }
#pragma unroll
                for (int k = 0; k < NW; k++) wb[k * na + jt] += acc[k];
            }
            __syncwarp();
        }
        __syncthreads();
        // combine warps in order: lo weight at j, hi weight from j - 1 (mod na)
        float* dst = stage + (size_t)item * NQ * na;
        for (int i = threadIdx.x; i < NQ * na; i += blockDim.x) {
            const int q = i / na, j = i - q * na;
            const int jm = (j == 0) ? na - 1 : j - 1;
            float v = 0.f;
            for (int w8 = 0; w8 < 8; w8++) v += bins[(w8 * NW + 2 * q) * na + j];
            for (int w8 = 0; w8 < 8; w8++) v += bins[(w8 * NW + 2 * q + 1) * na + jm];
            dst[i] = v;
        }
        __syncthreads();
    }
}

// mass[R][j] = pmass * (sum of partials of base rows R, R-1, R-ngz, R-ngz-1)
__global__ void k_mass_combine(DevGeo g, const float* __restrict__ stage,
                               const int32_t* __restrict__ rowitem, float* __restrict__ mass) {
    const int na = g.na, nrow = g.nrow;
    const int NQ = (g.ndim == 3) ? 4 : 2;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)nrow * na) return;
    const int R = (int)(i / na), j = (int)(i - (int64_t)R * na);
    const int off[4] = {0, 1, g.ngz, g.ngz + 1};
    float v = 0.f;
    for (int q = 0; q < NQ; q++) {
        const int B = R - off[q];
        if (B < 0) continue;
        for (int it = rowitem[B]; it < rowitem[B + 1]; it++)
            v += stage[((size_t)it * NQ + q) * na + j];
    }
    mass[i] = v * g.pmass;
}

// ---------------------------------------------------------------------------
// row key of a cell (nrow for particles off the grid)
__device__ __forceinline__ uint32_t row_of(const DevGeo& g, const CellW& c) {
    return (c.key >= 0) ? (uint32_t)(c.key / g.na) : (uint32_t)g.nrow;
}

__global__ void k_keys(DevGeo g, const float* __restrict__ P, int64_t cap, int64_t n,
                       uint32_t* __restrict__ keys) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float z = (g.ndim == 3) ? P[2 * cap + i] : 0.f;
    CellW c = gx_cell(g, P[i], P[cap + i], z, false);
    keys[i] = row_of(g, c);
}

// interpolated acceleration and potential at (x, y, z): grdacc + halfrc
__device__ __forceinline__ void gx_accel(const DevGeo& g, const float4* __restrict__ F, float x,
                                         float y, float z, float& ax, float& ay, float& az,
                                         float& ph) {
    ax = ay = az = ph = 0.f;
    CellW cw = gx_cell(g, x, y, z, true);
    if (cw.key < 0) return;
    float w[8];
    int ic[8];
    gx_weights(g, cw, w);
    const int nc = gx_corners(g, cw.key, ic);
    for (int k = 0; k < nc; k++) {
        if (ic[k] < 0) continue;
        const float4 f = __ldg(F + ic[k]);
        ax += f.x * w[k];
        ay += f.y * w[k];
        az += f.z * w[k];
        ph += f.w * w[k];
    }
    if (g.halo == 1) {
        // cored isothermal halo (frhalo.f:55-56): F(r) = -v^2 r / (r^2 + rc^2)
        float r2 = x * x + y * y + ((g.ndim == 3) ? z * z : 0.f);
        float rr = sqrtf(r2);
        float fr = -g.halo_v2 * rr / (r2 + g.halo_rc2);
        if (fr != 0.f) {
            fr = fr / rr;
            ax += fr * x;
            ay += fr * y;
            if (g.ndim == 3) az += fr * z;
        }
        ph += 0.5f * g.halo_v2 * logf(1.f + r2 / g.halo_rc2);
    }
}

// the fused particle pass of one step
__global__ void __launch_bounds__(256) k_push(DevGeo g, const float* __restrict__ Pin,
                                              float* __restrict__ Pout, int64_t cap, int64_t n,
                                              const int32_t* __restrict__ perm,
                                              const int32_t* __restrict__ orig_in,
                                              int32_t* __restrict__ orig_out,
                                              const float4* __restrict__ F,
                                              uint32_t* __restrict__ keys,
                                              float* __restrict__ pot) {
    int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = perm[s];
    const bool d3 = g.ndim == 3;
    float x = Pin[p], y = Pin[cap + p], z = 0.f, vx, vy, vz = 0.f;
    if (d3) {
        z = Pin[2 * cap + p];
        vx = Pin[3 * cap + p];
        vy = Pin[4 * cap + p];
        vz = Pin[5 * cap + p];
    } else {
        vx = Pin[2 * cap + p];
        vy = Pin[3 * cap + p];
    }
    const int32_t o = orig_in[p];
    float ax, ay, az, ph;
    gx_accel(g, F, x, y, z, ax, ay, az, ph);
    vx += ax;
    vy += ay;
    x += vx;
    y += vy;
    if (d3) {
        vz += az;
        z += vz;
    }
    Pout[s] = x;
    Pout[cap + s] = y;
    if (d3) {
        Pout[2 * cap + s] = z;
        Pout[3 * cap + s] = vx;
        Pout[4 * cap + s] = vy;
        Pout[5 * cap + s] = vz;
    } else {
        Pout[2 * cap + s] = vx;
        Pout[3 * cap + s] = vy;
    }
    orig_out[s] = o;
    if (pot) pot[s] = ph;
    CellW cn = gx_cell(g, x, y, z, false);
    keys[s] = row_of(g, cn);
}

// getacc for every particle at its stored position, written in load order
__global__ void k_getacc(DevGeo g, const float* __restrict__ P, int64_t cap, int64_t n,
                         const int32_t* __restrict__ origin, const float4* __restrict__ F,
                         float* __restrict__ acc, float* __restrict__ pot) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nd = g.ndim;
    float z = (nd == 3) ? P[2 * cap + i] : 0.f;
    float ax, ay, az, ph;
    gx_accel(g, F, P[i], P[cap + i], z, ax, ay, az, ph);
    const int64_t o = origin[i];
    acc[o * nd] = ax;
    acc[o * nd + 1] = ay;
    if (nd == 3) acc[o * nd + 2] = az;
    if (pot) pot[o] = ph;
}

// ---------------------------------------------------------------------------
static int deposit_sorted(GxCtx* c, const float* P, const int32_t* perm_sorted,
                          const uint32_t* keys_sorted) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    const int nrow = g.nrow;
    int rc0 = gx_phase_mark(c, PH_DEPOSIT);
    if (rc0) return rc0;
    {
        int bs = 256;
        int64_t nb = (n + 1 + bs - 1) / bs;
        k_rowstart<<<(unsigned)nb, bs, 0, c->stream>>>(keys_sorted, n, nrow, c->rowstart);
        GX_LAUNCHED(c);
    }
    k_items<<<1, 1024, 0, c->stream>>>(c->rowstart, nrow, g.ngz, g.nr, c->rowitem, c->items,
                                       c->nitems_d, c->jrk_d);
    GX_LAUNCHED(c);
    const int nw = (g.ndim == 3) ? 8 : 4;
    size_t sm = sizeof(float) * ((size_t)8 * nw * g.na + 8 * 32 * nw);
    int grid = std::min(c->maxitems, 148 * 8);
    if (nw == 8) {
        GX_CUDA(c, cudaFuncSetAttribute(k_deposit<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_deposit<8><<<grid, 256, sm, c->stream>>>(g, c->items, c->nitems_d, P, c->cap,
                                                   perm_sorted, c->stage, c->errword);
    } else {
        GX_CUDA(c, cudaFuncSetAttribute(k_deposit<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_deposit<4><<<grid, 256, sm, c->stream>>>(g, c->items, c->nitems_d, P, c->cap,
                                                   perm_sorted, c->stage, c->errword);
    }
    GX_LAUNCHED(c);
    rc0 = gx_phase_mark(c, PH_COMBINE);
    if (rc0) return rc0;
    {
        int64_t tot = (int64_t)nrow * g.na;
        int bs = 256;
        k_mass_combine<<<(unsigned)((tot + bs - 1) / bs), bs, 0, c->stream>>>(g, c->stage, c->rowitem,
                                                                             c->mass);
        GX_LAUNCHED(c);
    }
    return GX_OK;
}

int gx_mixed_masset(GxCtx* c) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    if (n == 0) {
        GX_CUDA(c, cudaMemsetAsync(c->mass, 0, sizeof(float) * g.mesh, c->stream));
        int32_t jrk[2] = {g.nr, 0};
        GX_CUDA(c, cudaMemcpyAsync(c->jrk_d, jrk, sizeof jrk, cudaMemcpyHostToDevice, c->stream));
        return GX_OK;
    }
    const float* P = c->pbuf[c->cur];
    int bs = 256;
    k_keys<<<(unsigned)((n + bs - 1) / bs), bs, 0, c->stream>>>(g, P, c->cap, n, c->pkey);
    GX_LAUNCHED(c);
    int o = 0;
    int rc = row_sort(c, c->pkey, &o);
    if (rc) return rc;
    rc = deposit_sorted(c, P, c->sb.vals[o], c->sb.keys[o]);
    if (rc) return rc;
    // the next pass processes pbuf[cur] in this sorted order
    GX_CUDA(c, cudaMemcpyAsync(c->perm, c->sb.vals[o], sizeof(int32_t) * n, cudaMemcpyDeviceToDevice,
                               c->stream));
    return gx_phase_end(c);
}

int gx_mixed_step(GxCtx* c, int nsteps, int phys) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    for (int s = 0; s < nsteps; s++) {
        const bool last = (s == nsteps - 1);
        int rc = gx_mixed_findf(c, phys && last, true);
        if (rc) return rc;
        if (n == 0) continue;
        const int nxt = c->cur ^ 1;
        int bs = 256;
        rc = gx_phase_mark(c, PH_PUSH);
        if (rc) return rc;
        k_push<<<(unsigned)((n + bs - 1) / bs), bs, 0, c->stream>>>(
            g, c->pbuf[c->cur], c->pbuf[nxt], c->cap, n, c->perm, c->origin, c->origin_tmp,
            c->field, c->pkey, (phys && last) ? c->ppot : nullptr);
        GX_LAUNCHED(c);
        std::swap(c->origin, c->origin_tmp);
        c->cur = nxt;
        int o = 0;
        rc = row_sort(c, c->pkey, &o);
        if (rc) return rc;
        rc = deposit_sorted(c, c->pbuf[c->cur], c->sb.vals[o], c->sb.keys[o]);
        if (rc) return rc;
        std::swap(c->perm, c->sb.vals[o]);
    }
    int rc = gx_phase_end(c);
    if (rc) return rc;
    c->have_field = false;
    return GX_OK;
}

int gx_mixed_getacc(GxCtx* c, float* acc, float* pot) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    if (n == 0) return GX_OK;
    int bs = 256;
    k_getacc<<<(unsigned)((n + bs - 1) / bs), bs, 0, c->stream>>>(
        g, c->pbuf[c->cur], c->cap, n, c->origin, c->field, c->pacc, c->ppot);
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaMemcpyAsync(acc, c->pacc, sizeof(float) * g.ndim * n, cudaMemcpyDeviceToHost,
                               c->stream));
    if (pot)
        GX_CUDA(c, cudaMemcpyAsync(pot, c->ppot, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    return GX_OK;
}

// ---------------------------------------------------------------------------
// weight entry point (cell numbers and weights of host particle records)
__global__ void k_weight_aos(DevGeo g, const float* __restrict__ aos, int64_t n, int old,
                             int32_t* __restrict__ ncl, float* __restrict__ wt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nw = 2 * g.ndim;
    const float* q = aos + i * nw;
    CellW c = gx_cell(g, q[0], q[1], (g.ndim == 3) ? q[2] : 0.f, old != 0);
    float w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (c.key >= 0) gx_weights(g, c, w);
    ncl[i] = c.key;
    for (int k = 0; k < 8; k++) wt[i * 8 + k] = w[k];
}

extern "C" int gx_weight(GxCtx* c, const float* coords, int64_t n, int old, int32_t* ncl, float* wt) {
    if (!c || n < 0 || (n > 0 && (!coords || !ncl || !wt))) return GX_ERR_ARG;
    if (c->fp64) return c->err = "gx_weight reports the mixed path's FP32 cells", GX_ERR_ARG;
    if (n == 0) return GX_OK;
    cudaSetDevice(c->dev);
    const int nw = 2 * c->g.ndim;
    float *daos = nullptr, *dwt = nullptr;
    int32_t* dncl = nullptr;
    GX_CUDA(c, cudaMallocAsync((void**)&daos, sizeof(float) * nw * n, c->stream));
    GX_CUDA(c, cudaMallocAsync((void**)&dwt, sizeof(float) * 8 * n, c->stream));
    GX_CUDA(c, cudaMallocAsync((void**)&dncl, sizeof(int32_t) * n, c->stream));
    GX_CUDA(c, cudaMemcpyAsync(daos, coords, sizeof(float) * nw * n, cudaMemcpyHostToDevice, c->stream));
    k_weight_aos<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, daos, n, old, dncl, dwt);
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaMemcpyAsync(ncl, dncl, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaMemcpyAsync(wt, dwt, sizeof(float) * 8 * n, cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaFreeAsync(daos, c->stream));
    GX_CUDA(c, cudaFreeAsync(dwt, c->stream));
    GX_CUDA(c, cudaFreeAsync(dncl, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}
