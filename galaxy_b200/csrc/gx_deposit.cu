// gx_deposit.cu -- deterministic mass assignment of the mixed path.
//
// massgn (SRC/lib15/massgn.f:68-89 p2d, 140-172 p3d) scatter-adds the 4 / 8
// weights of every particle into the mesh.  Here:
//
//   1. counting sort of the cell keys by their ring-plane row (one radix
//      digit of the key, ncl = (ju*ngz + jz)*na + jt + 1): the particle pass
//      counts its new rows with warp-aggregated integer atomics (k_push),
//      k_row_scan turns the counts into row starts, k_place gives every
//      particle its slot in the row-ordered permutation;
//   2. owner-computes deposit: a work item is up to DEP_CH particles of one
//      base row; the CTA forms each particle's weights from the cell key and
//      fractions the particle pass stored and adds them, as 2^-20 fixed-point integers, into shared-memory bins of the 4
//      (2D: 2) output rows the base row feeds (same row, plane above, ring
//      above, both); bins are staged per item as int32 rows;
//   3. k_mass_combine sums, per mesh row, the staged rows of the base rows
//      that feed it in int64 and converts once (x pmass, scaled.f:89-92).
//
// Every sum is an integer sum, so the mass array is bitwise reproducible
// whatever order the atomics resolve in; no floating-point atomics are used.
// The fixed-point quantum is 2^-20 of one particle's mass (9.5e-7).  Each
// particle feeds one bin per (output row, weight) and one weight to a staged
// cell, and every weight is below 1 + 1e-4 in magnitude (the linear weights
// lie in [0, 1] up to rounding; the quadratic ones reach -0.5 and 0.95 at
// the clamped rings), so a bin or staged cell holds less than
// DEP_CH (1 + 1e-4) 2^20 < 2^31 with DEP_CH = 2047: int32 never overflows.
#include <algorithm>

#include "gx_common.cuh"

#define FIXQ 1048576.0f  // 2^20

// per row: total over the counter copies, each copy's offset in the row;
// clears the counters for the next pass.  Per tile of ROW_TILE rows: the
// particles, the deposit work items and the occupied row range.  A block
// of 4 ROW_TILE threads takes one tile: thread (g, r) reads copies
// 8g .. 8g + 7 of row r (coalesced over r), so that every thread issues
// eight independent loads.
#define RR_GROUPS 4
static_assert(NCOPY % RR_GROUPS == 0, "copies split evenly over the groups");
__global__ void __launch_bounds__(ROW_TILE * RR_GROUPS) k_row_reduce(
    int nrow, uint32_t* __restrict__ rowcnt, uint32_t* __restrict__ rowfill,
    uint32_t* __restrict__ rowbase, uint32_t* __restrict__ rowtot, int32_t* __restrict__ tile) {
    constexpr int CPG = NCOPY / RR_GROUPS;  // copies per group
    __shared__ uint32_t gsum[RR_GROUPS][ROW_TILE];
    __shared__ int sh[4 * (ROW_TILE / 32)];
    const int rl = threadIdx.x % ROW_TILE, grp = threadIdx.x / ROW_TILE;
    const int r = blockIdx.x * ROW_TILE + rl;
    const size_t st = (size_t)nrow + 1;
    uint32_t v[CPG], run = 0;
    if (r <= nrow) {
#pragma unroll
        for (int k = 0; k < CPG; k++) v[k] = rowcnt[(grp * CPG + k) * st + r];
#pragma unroll
        for (int k = 0; k < CPG; k++) run += v[k];
    }
    gsum[grp][rl] = run;
    __syncthreads();
    uint32_t base = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < RR_GROUPS; q++) {
        const uint32_t x = gsum[q][rl];
        base += (q < grp) ? x : 0u;
        tot += x;
    }
    if (r <= nrow) {
#pragma unroll
        for (int k = 0; k < CPG; k++) {
            const size_t a = (grp * CPG + k) * st + r;
            rowbase[a] = base;
            base += v[k];
            rowcnt[a] = 0;
            rowfill[a] = 0;
        }
        if (grp == 0) rowtot[r] = tot;
    }
    if (grp == 0) {
        // tile statistics over the first ROW_TILE threads (warps 0 .. 7)
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        int a = (r <= nrow) ? (int)tot : 0, b = (r < nrow) ? (int)((tot + DEP_CH - 1) / DEP_CH) : 0;
        int lo = (r < nrow && tot > 0) ? r : 0x7fffffff, hi = (r < nrow && tot > 0) ? r : -1;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            sh[4 * warp] = a;
            sh[4 * warp + 1] = b;
            sh[4 * warp + 2] = lo;
            sh[4 * warp + 3] = hi;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0, b = 0, lo = 0x7fffffff, hi = -1;
        for (int w = 0; w < ROW_TILE / 32; w++) {
            a += sh[4 * w];
            b += sh[4 * w + 1];
            lo = min(lo, sh[4 * w + 2]);
            hi = max(hi, sh[4 * w + 3]);
        }
        tile[4 * blockIdx.x] = a;
        tile[4 * blockIdx.x + 1] = b;
        tile[4 * blockIdx.x + 2] = lo;
        tile[4 * blockIdx.x + 3] = hi;
    }
}

// row totals -> row starts, deposit work items, active ring range; one
// block per tile of ROW_TILE rows, the carry-in from the tile sums
__global__ void __launch_bounds__(ROW_TILE) k_row_scan(int nrow, int ngz, int nr, int quad,
                                                       const uint32_t* __restrict__ rowcnt,
                                                       const int32_t* __restrict__ tile,
                                                       int32_t* __restrict__ rowstart,
                                                       int32_t* __restrict__ rowitem,
                                                       int32_t* __restrict__ items,
                                                       int32_t* __restrict__ nitems,
                                                       int32_t* __restrict__ jrk) {
    __shared__ int ws_a[ROW_TILE / 32], ws_b[ROW_TILE / 32];
    __shared__ int carry_a, carry_b;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int b = blockIdx.x;
    if (warp == 0) {
        int ca = 0, cb = 0;
        for (int t = lane; t < b; t += 32) {
            ca += tile[4 * t];
            cb += tile[4 * t + 1];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ca += __shfl_xor_sync(0xffffffffu, ca, o);
            cb += __shfl_xor_sync(0xffffffffu, cb, o);
        }
        if (lane == 0) {
            carry_a = ca;
            carry_b = cb;
        }
    }
    const int r = b * ROW_TILE + threadIdx.x;
    const int cnt = (r <= nrow) ? (int)rowcnt[r] : 0;
    const int nit = (r < nrow) ? (cnt + DEP_CH - 1) / DEP_CH : 0;
    int xa = cnt, xb = nit;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int ya = __shfl_up_sync(0xffffffffu, xa, o), yb = __shfl_up_sync(0xffffffffu, xb, o);
        if (lane >= o) {
            xa += ya;
            xb += yb;
        }
    }
    if (lane == 31) {
        ws_a[warp] = xa;
        ws_b[warp] = xb;
    }
    __syncthreads();
    int pa = carry_a, pb = carry_b;
    for (int w = 0; w < warp; w++) {
        pa += ws_a[w];
        pb += ws_b[w];
    }
    const int ea = pa + xa - cnt, eb = pb + xb - nit;
    if (r <= nrow) rowstart[r] = ea;
    if (r <= nrow) rowitem[r] = eb;
    if (r < nrow) {
        for (int q = 0; q < nit; q++) {
            const int it = eb + q;
            items[3 * it + 0] = r;
            items[3 * it + 1] = ea + q * DEP_CH;
            items[3 * it + 2] = min(ea + (q + 1) * DEP_CH, ea + cnt);
        }
    }
    if (r == nrow) {
        // the off-grid row closes the arrays
        rowstart[nrow + 1] = ea + cnt;
        *nitems = eb;
    }
    if (b == nrow / ROW_TILE && warp == 0) {
        // the active ring range over all tiles, one warp
        const int ntile = nrow / ROW_TILE + 1;
        int rmin = 0x7fffffff, rmax = -1;
        for (int t = lane; t < ntile; t += 32) {
            rmin = min(rmin, tile[4 * t + 2]);
            rmax = max(rmax, tile[4 * t + 3]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
            rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        }
        // 1-based ring range as massgn tracks it (jrad = j + 1, krad = j + 2;
        // quadratic: jrad = ju, the ring below the central one, massgn.f:180)
        if (lane == 0) {
            if (rmax >= 0) {
                jrk[0] = rmin / ngz + (quad ? 0 : 1);
                jrk[1] = min(rmax / ngz + 2, nr);
            } else {
                jrk[0] = nr;
                jrk[1] = 0;
            }
        }
    }
    (void)nw;
}

// slot of every particle in the row-ordered permutation: perm[slot] = t.
// A thread places PLACE_U particles, one from each of PLACE_U consecutive
// 256-particle blocks of the counting pass (whose block index chose the
// counter copy), with their loads and atomics issued together.
#define PLACE_U 4
__global__ void __launch_bounds__(256) k_place(DevGeo g, const int32_t* __restrict__ keys, int64_t n,
                                               const int32_t* __restrict__ rowstart,
                                               const uint32_t* __restrict__ rowbase,
                                               uint32_t* __restrict__ rowfill,
                                               int32_t* __restrict__ perm,
                                               const int32_t* __restrict__ zone, int zsel) {
    const int nrow = g.nrow;
    const unsigned lane = threadIdx.x & 31;
    int64_t t[PLACE_U];
    uint32_t row[PLACE_U], peers[PLACE_U], base[PLACE_U];
    size_t co[PLACE_U];
#pragma unroll
    for (int u = 0; u < PLACE_U; u++) {
        const int64_t blk = (int64_t)blockIdx.x * PLACE_U + u;
        t[u] = blk * 256 + threadIdx.x;
        co[u] = (size_t)(blk & (NCOPY - 1)) * (nrow + 1);
        row[u] = 0xffffffffu;
        if (t[u] < n) {
            const int32_t key = __ldg(keys + t[u]);
            int r;
            row[u] = (key >= 0 && (!zone || __ldg(zone + t[u]) == zsel)) ? (uint32_t)gx_div_na(g, key, r)
                                                                         : (uint32_t)nrow;
        }
    }
#pragma unroll
    for (int u = 0; u < PLACE_U; u++) {
        const bool act = t[u] < n;
        const uint32_t am = __ballot_sync(0xffffffffu, act);
        peers[u] = __match_any_sync(0xffffffffu, row[u]) & am;
        const int leader = __ffs(peers[u]) - 1;
        base[u] = 0;
        if (act && (int)lane == leader) base[u] = atomicAdd(rowfill + co[u] + row[u], (uint32_t)__popc(peers[u]));
    }
#pragma unroll
    for (int u = 0; u < PLACE_U; u++) {
        const int leader = __ffs(peers[u]) - 1;
        const uint32_t b = __shfl_sync(0xffffffffu, base[u], leader < 0 ? 0 : leader);
        if (t[u] < n)
            perm[__ldg(rowstart + row[u]) + __ldg(rowbase + co[u] + row[u]) + b +
                 __popc(peers[u] & lanemask_lt())] = (int32_t)t[u];
    }
}

// owner-computes deposit of one work item per CTA iteration, from the cell
// keys and fractions the particle pass stored
template <int NW>
__global__ void __launch_bounds__(256) k_deposit(DevGeo g, const int32_t* __restrict__ items,
                                                 const int32_t* __restrict__ nitems,
                                                 const int32_t* __restrict__ keys,
                                                 const float* __restrict__ fr, int64_t cap,
                                                 const int32_t* __restrict__ perm,
                                                 int32_t* __restrict__ stage,
                                                 int32_t* __restrict__ errword) {
    extern __shared__ __align__(16) int32_t bins[];  // [NW][na]
    const int na = g.na;
    constexpr int NQ = (NW == 27) ? 9 : NW / 2;
    const int nit = *nitems;
    for (int item = blockIdx.x; item < nit; item += gridDim.x) {
        const int row = items[3 * item], s0 = items[3 * item + 1], s1 = items[3 * item + 2];
        for (int i = threadIdx.x; i < NW * na; i += blockDim.x) bins[i] = 0;
        __syncthreads();
        // an item holds at most DEP_CH < 8 x 256 particles: each thread loads
        // four together, adds them, then the next four
        static_assert(DEP_CH <= 8 * 256, "eight particles per thread");
        for (int s00 = s0; s00 < s1; s00 += 1024) {
            CellW cw[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int s = s00 + threadIdx.x + u * 256;
                cw[u].key = -2;
                if (s < s1) {
                    const int p = __ldg(perm + s);
                    cw[u].key = __ldg(keys + p);
                    cw[u].du = __ldg(fr + p);
                    cw[u].dt = __ldg(fr + cap + p);
                    cw[u].dz = (NW >= 8) ? __ldg(fr + 2 * cap + p) : 0.f;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (cw[u].key == -2) continue;
                int jt;
                if (cw[u].key < 0 || gx_div_na(g, cw[u].key, jt) != row) {
                    atomicExch(errword, 1);
                    continue;
                }
                float w[NW == 27 ? 27 : 8];
                if constexpr (NW == 27) gx_weights27(cw[u], w);
                else gx_weights<(NW == 8) ? 3 : 2>(g, cw[u], w);
#pragma unroll
                for (int k = 0; k < NW; k++) atomicAdd(&bins[k * na + jt], __float2int_rn(w[k] * FIXQ));
            }
        }
        __syncthreads();
        int32_t* dst = stage + (size_t)item * NQ * na;
        if constexpr (NW == 27) {
            // output row q = 3 (u offset + 1) + (z offset + 1) gets the theta
            // weight i of the particles whose central spoke is j + 1 - i
            for (int i = threadIdx.x; i < NQ * na; i += blockDim.x) {
                const int q = i / na, j = i - q * na;
                const int jp = (j == na - 1) ? 0 : j + 1, jm = (j == 0) ? na - 1 : j - 1;
                dst[i] = bins[(3 * q) * na + jp] + bins[(3 * q + 1) * na + j] +
                         bins[(3 * q + 2) * na + jm];
            }
        } else {
            // output row q gets the lo weight at j and the hi weight from j - 1
            for (int i = threadIdx.x; i < NQ * na; i += blockDim.x) {
                const int q = i / na, j = i - q * na;
                const int jm = (j == 0) ? na - 1 : j - 1;
                dst[i] = bins[(2 * q) * na + j] + bins[(2 * q + 1) * na + jm];
            }
        }
        __syncthreads();
    }
}

// mass[R][j] = pmass 2^-20 (sum over the base rows that feed row R: R,
// R-1, R-ngz, R-ngz-1 for the linear scheme, R + 1 .. R - 1 - ngz for the
// quadratic one).  The item ranges of all base rows are loaded first and
// the first item of each in one batch, so that a thread waits on two
// dependent loads rather than one chain per base row.
template <int NQ>
__global__ void __launch_bounds__(256) k_mass_combine(DevGeo g, const int32_t* __restrict__ stage,
                                                      const int32_t* __restrict__ rowitem,
                                                      float* __restrict__ mass, float pm) {
    const int na = g.na, nrow = g.nrow;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // mesh < 2^24
    if (i >= nrow * na) return;
    int j;
    const int R = gx_div_na(g, i, j);
    int b0[NQ], b1[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        // row offset of output row q from its base row: linear (same, plane
        // above, ring above, both); quadratic (u - 1 .. u + 1) x (z - 1 .. z + 1)
        const int off = (NQ == 9) ? (q / 3 - 1) * g.ngz + (q % 3 - 1)
                                  : ((q & 1) + ((q >> 1) ? g.ngz : 0));
        const int B = R - off;
        const bool ok = B >= 0 && B < nrow;
        b0[q] = ok ? __ldg(rowitem + B) : 0;
        b1[q] = ok ? __ldg(rowitem + B + 1) : 0;
    }
    int first[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++)
        first[q] = (b0[q] < b1[q]) ? __ldg(stage + ((size_t)b0[q] * NQ + q) * na + j) : 0;
    long long v = 0;
#pragma unroll
    for (int q = 0; q < NQ; q++) v += first[q];
    // rows with more than DEP_CH particles have several items: sixteen
    // loads in flight per thread (the densest rows of an evolved disc hold
    // 100+ items)
    for (int q = 0; q < NQ; q++) {
        const int32_t* sp = stage + (size_t)q * na + j;
        const size_t stride = (size_t)NQ * na;
        int it = b0[q] + 1;
        for (; it + 16 <= b1[q]; it += 16) {
            int32_t x[16];
#pragma unroll
            for (int u = 0; u < 16; u++) x[u] = __ldg(sp + (size_t)(it + u) * stride);
#pragma unroll
            for (int u = 0; u < 16; u++) v += x[u];
        }
        for (; it < b1[q]; it++) v += __ldg(sp + (size_t)it * stride);
    }
    mass[i] = (float)((double)v * (1.0 / (double)FIXQ)) * pm;
}

// cell keys and fractions of the stored particles, rows counted (masset)
__global__ void k_row_keys(DevGeo g, const float* __restrict__ P, int64_t cap, int64_t n,
                           int32_t* __restrict__ keys, float* __restrict__ fr,
                           uint32_t* __restrict__ rowcnt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool act = i < n;
    uint32_t row = 0;
    if (act) {
        const float z = (g.ndim == 3) ? P[2 * cap + i] : 0.f;
        const CellW c = gx_cell(g, P[i], P[cap + i], z, false);
        row = (c.key >= 0) ? (uint32_t)(c.key / g.na) : (uint32_t)g.nrow;
        keys[i] = c.key;
        fr[i] = c.du;
        fr[cap + i] = c.dt;
        if (g.ndim == 3) fr[2 * cap + i] = c.dz;
    }
    gx_row_count(row, act, rowcnt + (size_t)(blockIdx.x & (NCOPY - 1)) * (g.nrow + 1));
}

// rows counted by the caller's pass -> permutation, deposit, mass
int gx_deposit_rows(GxCtx* c, const int32_t* keys, const float* fr, int32_t* perm_out,
                    const int32_t* zone, int zsel, float* mass_out, float pm) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    int rc = gx_phase_mark(c, PH_SORT);
    if (rc) return rc;
    const int ntile = (g.nrow + 1 + ROW_TILE - 1) / ROW_TILE;
    k_row_reduce<<<ntile, ROW_TILE * RR_GROUPS, 0, c->stream>>>(g.nrow, c->rowcnt, c->rowfill, c->rowbase,
                                                                 c->rowtot, c->rowtile);
    GX_LAUNCHED(c);
    k_row_scan<<<ntile, ROW_TILE, 0, c->stream>>>(g.nrow, g.ngz, g.nr, g.quad, c->rowtot, c->rowtile, c->rowstart,
                                                   c->rowitem, c->items, c->nitems_d, c->jrk_d);
    GX_LAUNCHED(c);
    if (n > 0) {
        const int64_t nblk = (n + 255) / 256;
        k_place<<<(unsigned)((nblk + PLACE_U - 1) / PLACE_U), 256, 0, c->stream>>>(
            g, keys, n, c->rowstart, c->rowbase, c->rowfill, perm_out, zone, zsel);
        GX_LAUNCHED(c);
    }
    rc = gx_phase_mark(c, PH_DEPOSIT);
    if (rc) return rc;
    const int nw = g.quad ? 27 : (g.ndim == 3) ? 8 : 4;
    const size_t sm = sizeof(int32_t) * (size_t)nw * g.na;
    const int grid = std::min(c->maxitems, 148 * 32);  // ~4 items per CTA at 10M particles
    if (nw == 27) {
        // 27 rows of bins of up to 512 spokes exceed the default 48 KB (the
        // attribute belongs to the calling thread's current device)
        GX_CUDA(c, cudaFuncSetAttribute(k_deposit<27>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(sizeof(int32_t) * 27 * 512)));
        k_deposit<27><<<grid, 256, sm, c->stream>>>(g, c->items, c->nitems_d, keys, fr, c->cap,
                                                    perm_out, c->stage, c->errword);
    } else if (nw == 8)
        k_deposit<8><<<grid, 256, sm, c->stream>>>(g, c->items, c->nitems_d, keys, fr, c->cap,
                                                   perm_out, c->stage, c->errword);
    else
        k_deposit<4><<<grid, 256, sm, c->stream>>>(g, c->items, c->nitems_d, keys, fr, c->cap,
                                                   perm_out, c->stage, c->errword);
    GX_LAUNCHED(c);
    rc = gx_phase_mark(c, PH_COMBINE);
    if (rc) return rc;
    const int64_t tot = (int64_t)g.nrow * g.na;
    auto kc = g.quad ? k_mass_combine<9> : (g.ndim == 3) ? k_mass_combine<4> : k_mass_combine<2>;
    kc<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(
        g, c->stage, c->rowitem, mass_out ? mass_out : c->mass, pm < 0.f ? g.pmass : pm);
    GX_LAUNCHED(c);
    return GX_OK;
}

int gx_mixed_masset(GxCtx* c) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    if (n > 0) {
        k_row_keys<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
            g, c->pbuf[c->cur], c->cap, n, c->pkey[c->cur], c->pfr, c->rowcnt);
        GX_LAUNCHED(c);
    }
    int rc = gx_deposit_rows(c, c->pkey[c->cur], c->pfr, c->perm);
    if (rc) return rc;
    c->have_keys = true;
    return gx_phase_end(c);
}
