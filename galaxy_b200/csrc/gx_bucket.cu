// gx_bucket.cu -- the fused particle pass of the mixed-precision step on a
// bucketed particle store.
//
// One step of the reference (step.f:135-290) is, per particle, grdacc
// (grdacc.f:189-266: weights of the current cell, gather of the fields at
// its corners), stpgrp (stpgrp.f:26-32: v += a, x += v) and massgn
// (massgn.f:68-89, 140-172: the weights of the new cell scatter-added into
// the mesh), then scaled (scaled.f:89-92).  Here that is one kernel per
// step, k_push_bkt, over a store that keeps the particles grouped by the
// ring-plane row of their cell:
//
//   * pbuf[b] holds one segment of slots per row (row nrow: off the grid);
//     segment r starts at bk_base[b][r] and has bk_cap[b][r] slots, planned
//     from the previous step's row counts with 1/8 + 16 slots of slack, so
//     that a particle that changes row usually finds room in its new row's
//     segment.  A particle that does not is appended to an overflow area
//     after the segments (capacity: every particle), so no particle is ever
//     dropped, and the next plan gives its row the room.
//   * k_push_bkt walks work items (up to BK_ITEM particles of one row's
//     segment, or of the overflow area) in the input buffer, and for each
//     particle interpolates the field, moves it, computes its new cell
//     exactly as the reference does (bit-exact keys), writes it into the
//     segment of its new row in the output buffer (warp-aggregated slot
//     atomics), and adds its 4 / 8 CIC weights as 2^-20 fixed-point
//     integers: into int64 shared-memory bins over the window of rows around
//     the item's row (4 rings, and 4 planes in 3D: every cell a particle of
//     the row can reach moving less than a cell), or, for corners outside
//     it, straight into the int64 mesh accumulator.  The bins are flushed
//     into the accumulator (nonzero bins only) after each item.
//   * k_bk_plan (one CTA) turns the output buffer's row counts into its
//     work items, the next output buffer's segments and the active ring
//     range (jrad, krad); k_mass_convert turns the accumulator into the mass
//     array (x pmass) and clears it.
//
// Integer sums do not depend on their order, so the mass array is the same
// integers, converted the same way, as the sort-based deposit of
// gx_deposit.cu: the fused path is bitwise identical to it, whatever order
// the atomics resolve in.  Particles keep their load index (origin) next to
// them; gx_dense() compacts the store back to n contiguous particles for the
// entry points that walk it that way (unload, getacc, tmcent, icheck, the
// adjoint, masset).
#include <algorithm>

#include "gx_common.cuh"

#define BK_FIXQ 1048576.0f  // 2^20: the fixed-point quantum of gx_deposit.cu
#define BK_ITEM 8192        // particles per work item
#define BK_SPARSE 64        // items with fewer particles add straight into the mesh
#define BK_THREADS 256
#define PLAN_THREADS 1024
#define PLAN_ROWS 8         // rows per plan thread per pass

__device__ __forceinline__ void red_add_s64(unsigned long long* a, int v) {
    atomicAdd(a, (unsigned long long)(long long)v);  // two's complement sum
}

// ---------------------------------------------------------------------------
// block-wide exclusive scan of two ints (PLAN_THREADS threads)
__device__ __forceinline__ void plan_scan2(int a, int b, int& ea, int& eb, int& ta, int& tb) {
    __shared__ int wa[PLAN_THREADS / 32], wb[PLAN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int xa = a, xb = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int ya = __shfl_up_sync(0xffffffffu, xa, o), yb = __shfl_up_sync(0xffffffffu, xb, o);
        if (lane >= o) {
            xa += ya;
            xb += yb;
        }
    }
    if (lane == 31) {
        wa[warp] = xa;
        wb[warp] = xb;
    }
    __syncthreads();
    if (warp == 0) {
        int va = wa[lane], vb = wb[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int ya = __shfl_up_sync(0xffffffffu, va, o), yb = __shfl_up_sync(0xffffffffu, vb, o);
            if (lane >= o) {
                va += ya;
                vb += yb;
            }
        }
        wa[lane] = va;
        wb[lane] = vb;
    }
    __syncthreads();
    const int pa = warp ? wa[warp - 1] : 0, pb = warp ? wb[warp - 1] : 0;
    ea = pa + xa - a;
    eb = pb + xb - b;
    ta = wa[PLAN_THREADS / 32 - 1];
    tb = wb[PLAN_THREADS / 32 - 1];
    __syncthreads();
}

// The plan of one step, one CTA:
//  * with fill_o: the work items of the buffer just written (fill_o, cap_o,
//    base_o, overflow count *ovf_o at slot ovf_base), the active ring range
//    of its particles (jrad = first ring + 1, krad = min(last ring + 2, nr),
//    as massgn tracks them), and ctl[0] = items, ctl[1] = 0 (work counter);
//  * the segments of the buffer to be written next from the row counts
//    want: cap_n = want + want/8 + 16 (0 for empty rows), base_n their
//    exclusive sum; its fill counters and overflow count cleared.
__global__ void __launch_bounds__(PLAN_THREADS) k_bk_plan(
    int nrow1, int nr, int ngz, const int32_t* __restrict__ fill_o, const int32_t* __restrict__ cap_o,
    const int32_t* __restrict__ base_o, const int32_t* __restrict__ ovf_o, int64_t ovf_base,
    int4* __restrict__ items, int32_t* __restrict__ ctl, int32_t* __restrict__ jrk,
    const int32_t* __restrict__ want, int32_t* __restrict__ cap_n, int32_t* __restrict__ base_n,
    int32_t* __restrict__ fill_n, int32_t* __restrict__ ovf_n) {
    __shared__ int s_mn[PLAN_THREADS / 32], s_mx[PLAN_THREADS / 32];
    const int nrow = nrow1 - 1;
    int carry_cap = 0, carry_it = 0, rmin = 0x7fffffff, rmax = -1;
    for (int c0 = 0; c0 < nrow1; c0 += PLAN_THREADS * PLAN_ROWS) {
        const int r0 = c0 + threadIdx.x * PLAN_ROWS;
        int capv[PLAN_ROWS], nit[PLAN_ROWS], val[PLAN_ROWS];
        int scap = 0, snit = 0;
#pragma unroll
        for (int k = 0; k < PLAN_ROWS; k++) {
            const int r = r0 + k;
            capv[k] = nit[k] = val[k] = 0;
            if (r < nrow1) {
                const int w = want[r];
                capv[k] = w + (w >> 3) + (w > 0 ? 16 : 0);
                if (fill_o) {
                    const int f = fill_o[r];
                    val[k] = min(f, cap_o[r]);
                    nit[k] = (val[k] + BK_ITEM - 1) / BK_ITEM;
                    if (f > 0 && r < nrow) {
                        rmin = min(rmin, r);
                        rmax = max(rmax, r);
                    }
                }
            }
            scap += capv[k];
            snit += nit[k];
        }
        int ecap, eit, tcap, tit;
        plan_scan2(scap, snit, ecap, eit, tcap, tit);
        ecap += carry_cap;
        eit += carry_it;
#pragma unroll
        for (int k = 0; k < PLAN_ROWS; k++) {
            const int r = r0 + k;
            if (r >= nrow1) break;
            cap_n[r] = capv[k];
            base_n[r] = ecap;
            fill_n[r] = 0;
            ecap += capv[k];
            if (fill_o) {
                const int b = base_o[r];
                for (int q = 0; q < nit[k]; q++)
                    items[eit + q] = make_int4(r, b + q * BK_ITEM, b + min((q + 1) * BK_ITEM, val[k]), 0);
                eit += nit[k];
            }
        }
        carry_cap += tcap;
        carry_it += tit;
    }
    if (fill_o) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
            rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        }
        if (lane == 0) {
            s_mn[warp] = rmin;
            s_mx[warp] = rmax;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 0; w < PLAN_THREADS / 32; w++) {
                rmin = min(rmin, s_mn[w]);
                rmax = max(rmax, s_mx[w]);
            }
            if (rmax >= 0) {
                jrk[0] = rmin / ngz + 1;
                jrk[1] = min(rmax / ngz + 2, nr);
            } else {
                jrk[0] = nr;
                jrk[1] = 0;
            }
            const int ov = *ovf_o;
            int it = carry_it;
            for (int q = 0; q * BK_ITEM < ov; q++, it++)
                items[it] = make_int4(-1, (int)ovf_base + q * BK_ITEM,
                                      (int)ovf_base + min((q + 1) * BK_ITEM, ov), 0);
            ctl[0] = it;
            ctl[1] = 0;
        }
    }
    if (threadIdx.x == 0) *ovf_n = 0;
}

// ---------------------------------------------------------------------------
// slot of a particle bound for row rk in the output buffer: warp-aggregated
// atomics on the row's fill counter; past the segment's capacity, the
// overflow area (all 32 lanes call; act false lanes take no slot)
__device__ __forceinline__ int64_t bk_slot(bool act, uint32_t rk, const int32_t* __restrict__ cap_o,
                                           const int32_t* __restrict__ base_o, int32_t* __restrict__ fill_o,
                                           int32_t* __restrict__ ovf_o, int64_t ovf_base) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t am = __ballot_sync(0xffffffffu, act);
    const uint32_t peers = __match_any_sync(0xffffffffu, act ? rk : 0xffffffffu) & am;
    const int leader = __ffs(peers) - 1;
    int b = 0;
    if (act && (int)lane == leader) b = atomicAdd(fill_o + rk, __popc(peers));
    b = __shfl_sync(0xffffffffu, b, leader < 0 ? 0 : leader);
    const int slot = b + __popc(peers & lanemask_lt());
    int64_t dst = -1;
    bool ovf = false;
    if (act) {
        if (slot < __ldg(cap_o + rk)) dst = (int64_t)__ldg(base_o + rk) + slot;
        else ovf = true;
    }
    const uint32_t om = __ballot_sync(0xffffffffu, ovf);
    if (om) {
        const int ol = __ffs(om) - 1;
        int ob = 0;
        if ((int)lane == ol) ob = atomicAdd(ovf_o, __popc(om));
        ob = __shfl_sync(0xffffffffu, ob, ol);
        if (ovf) dst = ovf_base + ob + __popc(om & lanemask_lt());
    }
    return dst;
}

// The fused particle pass of one step.  Persistent CTAs take work items from
// a counter.  bins: int64 [WROWS][na] over the item's window, zero between
// items.  Window of an item of row (ir, iz): rings ir - 1 .. ir + 2 and, in
// 3D, planes iz - 1 .. iz + 2 (bin row 4 a + b for ring ir - 1 + a, plane
// iz - 1 + b); 2D: rows ir - 1 .. ir + 2.
template <int ND, bool COMP>
__global__ void __launch_bounds__(BK_THREADS) k_push_bkt(
    DevGeo g, const float* __restrict__ Pin, float* __restrict__ Pout, int64_t cap,
    const int32_t* __restrict__ oin, int32_t* __restrict__ oout, const float4* __restrict__ F,
    const int4* __restrict__ items, int32_t* __restrict__ ctl, const int32_t* __restrict__ cap_o,
    const int32_t* __restrict__ base_o, int32_t* __restrict__ fill_o, int32_t* __restrict__ ovf_o,
    int64_t ovf_base, unsigned long long* __restrict__ acc) {
    extern __shared__ __align__(16) unsigned long long bins[];
    __shared__ int s_item;
    constexpr bool d3 = ND == 3;
    constexpr int WROWS = d3 ? 16 : 4;
    constexpr int NW = 2 * ND;
    const int na = g.na, ngz = d3 ? g.ngz : 1, nrow = g.nrow;
    const int nit = ctl[0];
    for (int i = threadIdx.x; i < WROWS * na; i += BK_THREADS) bins[i] = 0ull;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(ctl + 1, 1);
        __syncthreads();  // also orders the previous item's flush before these deposits
        const int it = s_item;
        if (it >= nit) break;
        const int4 I = items[it];
        const int row = I.x, s0 = I.y, s1 = I.z;
        const bool win = row >= 0 && row < nrow && (s1 - s0) >= BK_SPARSE;
        // ring and plane of the item's row: the window's origin is one below
        const int wir = d3 ? row / ngz : row;
        const int wiz = d3 ? row - wir * ngz : 0;
        for (int b0 = s0; b0 < s1; b0 += BK_THREADS) {
            const int s = b0 + threadIdx.x;
            const bool act = s < s1;
            uint32_t rk = 0;
            float P[NW + (COMP ? ND : 0)];
            int32_t o = 0;
            if (act) {
#pragma unroll
                for (int k = 0; k < NW + (COMP ? ND : 0); k++) P[k] = Pin[(size_t)k * cap + s];
                o = oin[s];
                float &x = P[0], &y = P[1];
                float z = d3 ? P[2] : 0.f;
                const CellW cw = gx_cell_t<false, ND>(g, x, y, z, true);
                float ax, ay, az, ph;
                gx_accel_cell_t<false, ND>(g, F, cw, x, y, z, ax, ay, az, ph);
                float& vx = P[ND];
                float& vy = P[ND + 1];
                vx += ax;
                vy += ay;
                if (d3) P[ND + 2] += az;
                if (COMP) {
                    gx_comp_add(x, P[NW], vx);
                    gx_comp_add(y, P[NW + 1], vy);
                    if (d3) gx_comp_add(P[2], P[NW + 2], P[ND + 2]);
                } else {
                    x += vx;
                    y += vy;
                    if (d3) P[2] += P[ND + 2];
                }
                z = d3 ? P[2] : 0.f;
                const CellW cn = gx_cell_t<true, ND>(g, x, y, z, false);
                rk = (cn.key >= 0) ? (uint32_t)cn.row : (uint32_t)nrow;
                if (cn.key >= 0) {
                    float w[8];
                    gx_weights<ND>(g, cn, w);
                    const int jt0 = cn.jt, jt1 = (cn.jt == na - 1) ? 0 : cn.jt + 1;
                    // the corner rows: row, row + 1 (the next plane, or ring in
                    // 2D), and in 3D row + ngz, row + ngz + 1, with their
                    // window coordinates (a, b)
                    int fr[4], wa[4], wb[4];
                    fr[0] = cn.row;
                    fr[1] = cn.row + 1;
                    if (d3) {
                        int ju1 = cn.ju, iz1 = cn.iz + 1;
                        if (iz1 == ngz) {
                            iz1 = 0;
                            ju1 += 1;
                        }
                        wa[0] = cn.ju - wir + 1;
                        wb[0] = cn.iz - wiz + 1;
                        wa[1] = ju1 - wir + 1;
                        wb[1] = iz1 - wiz + 1;
                        fr[2] = cn.row + ngz;
                        fr[3] = cn.row + ngz + 1;
                        wa[2] = wa[0] + 1;
                        wb[2] = wb[0];
                        wa[3] = wa[1] + 1;
                        wb[3] = wb[1];
                    } else {
                        wa[0] = cn.row - row + 1;
                        wa[1] = wa[0] + 1;
                        wb[0] = wb[1] = 0;
                    }
                    constexpr int NQ = d3 ? 4 : 2;
#pragma unroll
                    for (int q = 0; q < NQ; q++) {
                        if (fr[q] >= nrow) continue;  // past the mesh end: dropped, as massgn does
                        const int v0 = __float2int_rn(w[2 * q] * BK_FIXQ);
                        const int v1 = __float2int_rn(w[2 * q + 1] * BK_FIXQ);
                        const bool inw = win && wa[q] >= 0 && wa[q] < 4 && wb[q] >= 0 && wb[q] < 4;
                        if (inw) {
                            unsigned long long* br = bins + (size_t)(d3 ? 4 * wa[q] + wb[q] : wa[q]) * na;
                            if (v0) atomicAdd(br + jt0, (unsigned long long)(long long)v0);
                            if (v1) atomicAdd(br + jt1, (unsigned long long)(long long)v1);
                        } else {
                            unsigned long long* ar = acc + (size_t)fr[q] * na;
                            if (v0) red_add_s64(ar + jt0, v0);
                            if (v1) red_add_s64(ar + jt1, v1);
                        }
                    }
                }
            }
            const int64_t dst = bk_slot(act, rk, cap_o, base_o, fill_o, ovf_o, ovf_base);
            if (act) {
#pragma unroll
                for (int k = 0; k < NW + (COMP ? ND : 0); k++) Pout[(size_t)k * cap + dst] = P[k];
                oout[dst] = o;
            }
        }
        if (win) {
            __syncthreads();
            for (int i = threadIdx.x; i < WROWS * na; i += BK_THREADS) {
                const unsigned long long v = bins[i];
                if (v) {
                    const int wr = i / na, j = i - wr * na;
                    const int R = d3 ? (wir - 1 + (wr >> 2)) * ngz + (wiz - 1 + (wr & 3)) : wir - 1 + wr;
                    atomicAdd(acc + (size_t)R * na + j, v);
                    bins[i] = 0ull;
                }
            }
        }
        __syncthreads();  // s_item is rewritten by thread 0 next
    }
}

// mass = pmass 2^-20 acc (as k_mass_combine forms it); acc cleared for the
// next step.  Two cells per thread (mesh is even: na is).
__global__ void k_mass_convert(unsigned long long* __restrict__ acc, float* __restrict__ mass, int mesh,
                               float pm) {
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= mesh) return;
    ulonglong2 v = *reinterpret_cast<const ulonglong2*>(acc + i);
    float2 m;
    m.x = (float)((double)(long long)v.x * (1.0 / (double)BK_FIXQ)) * pm;
    m.y = (float)((double)(long long)v.y * (1.0 / (double)BK_FIXQ)) * pm;
    *reinterpret_cast<float2*>(mass + i) = m;
    if (v.x | v.y) *reinterpret_cast<ulonglong2*>(acc + i) = make_ulonglong2(0ull, 0ull);
}

// ---------------------------------------------------------------------------
// dense store -> bucketed store: the row of every particle's cell (the
// deposit's exact cell), counted
template <int ND>
__global__ void k_bk_rows(DevGeo g, const float* __restrict__ P, int64_t cap, int64_t n,
                          int32_t* __restrict__ rows, int32_t* __restrict__ cnt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool act = i < n;
    uint32_t rk = 0;
    if (act) {
        const CellW c = gx_cell_t<true, ND>(g, P[i], P[cap + i], ND == 3 ? P[2 * cap + i] : 0.f, false);
        rk = (c.key >= 0) ? (uint32_t)c.row : (uint32_t)g.nrow;
        rows[i] = (int32_t)rk;
    }
    const uint32_t am = __ballot_sync(0xffffffffu, act);
    const uint32_t peers = __match_any_sync(0xffffffffu, act ? rk : 0xffffffffu) & am;
    if (act && (peers & lanemask_lt()) == 0) atomicAdd(cnt + rk, (int)__popc(peers));
}

__global__ void k_bk_scatter(const float* __restrict__ Pin, float* __restrict__ Pout, int64_t cap, int64_t n,
                             int nplanes, const int32_t* __restrict__ oin, int32_t* __restrict__ oout,
                             const int32_t* __restrict__ rows, const int32_t* __restrict__ cap_o,
                             const int32_t* __restrict__ base_o, int32_t* __restrict__ fill_o,
                             int32_t* __restrict__ ovf_o, int64_t ovf_base) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool act = i < n;
    const uint32_t rk = act ? (uint32_t)rows[i] : 0u;
    const int64_t dst = bk_slot(act, rk, cap_o, base_o, fill_o, ovf_o, ovf_base);
    if (!act) return;
    for (int k = 0; k < nplanes; k++) Pout[(size_t)k * cap + dst] = Pin[(size_t)k * cap + i];
    oout[dst] = oin[i];
}

// bucketed store -> n contiguous particles, item by item (CTA-reserved ranges)
__global__ void k_bk_densify(const float* __restrict__ Pin, float* __restrict__ Pout, int64_t cap,
                             int nplanes, const int32_t* __restrict__ oin, int32_t* __restrict__ oout,
                             const int4* __restrict__ items, const int32_t* __restrict__ ctl,
                             int32_t* __restrict__ dense_ctr) {
    __shared__ int s_d0;
    const int nit = ctl[0];
    for (int it = blockIdx.x; it < nit; it += gridDim.x) {
        const int4 I = items[it];
        if (threadIdx.x == 0) s_d0 = atomicAdd(dense_ctr, I.z - I.y);
        __syncthreads();
        const int d0 = s_d0;
        for (int s = I.y + threadIdx.x; s < I.z; s += blockDim.x) {
            const int64_t d = d0 + (s - I.y);
            for (int k = 0; k < nplanes; k++) Pout[(size_t)k * cap + d] = Pin[(size_t)k * cap + s];
            oout[d] = oin[s];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
bool gx_fast_ok(const GxCtx* c) {
    return !c->fp64 && c->nzones == 1 && !c->g.quad && !(c->cfg.flags & GX_FLAG_SORTED_DEPOSIT);
}

static inline int bk_nplanes(const GxCtx* c) { return 2 * c->g.ndim + (c->g.comp ? c->g.ndim : 0); }

template <typename T>
static int bk_alloc(GxCtx* c, T** p, size_t count) {
    if (*p) return GX_OK;
    if (cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) {
        *p = nullptr;
        c->err = "cudaMalloc of the bucketed store's tables failed";
        return GX_ERR_NOMEM;
    }
    return GX_OK;
}

// row tables and the mass accumulator (grid-sized, once per context)
int gx_bucket_alloc(GxCtx* c) {
    const size_t nrow1 = (size_t)c->g.nrow + 1;
    int rc = 0;
    for (int b = 0; b < 2 && !rc; b++) {
        rc = rc ? rc : bk_alloc(c, &c->bk_cap[b], nrow1);
        rc = rc ? rc : bk_alloc(c, &c->bk_base[b], nrow1);
        rc = rc ? rc : bk_alloc(c, &c->bk_fill[b], nrow1);
    }
    rc = rc ? rc : bk_alloc(c, &c->bk_ctl, 16);
    rc = rc ? rc : bk_alloc(c, &c->bk_cnt, nrow1);
    rc = rc ? rc : bk_alloc(c, &c->macc, (size_t)c->g.mesh);
    if (rc) return rc;
    GX_CUDA(c, cudaMemsetAsync(c->macc, 0, sizeof(unsigned long long) * c->g.mesh, c->stream));
    GX_CUDA(c, cudaMemsetAsync(c->bk_ctl, 0, sizeof(int32_t) * 16, c->stream));
    return GX_OK;
}

static int bk_plan(GxCtx* c, int out, bool with_items) {
    const DevGeo& g = c->g;
    const int nxt = out ^ 1;
    k_bk_plan<<<1, PLAN_THREADS, 0, c->stream>>>(
        g.nrow + 1, g.nr, g.ngz, with_items ? c->bk_fill[out] : nullptr, c->bk_cap[out], c->bk_base[out],
        c->bk_ctl + 4 * out, c->bk_main, c->bk_items, c->bk_ctl + 8, c->jrk_d,
        with_items ? c->bk_fill[out] : c->bk_cnt, c->bk_cap[nxt], c->bk_base[nxt], c->bk_fill[nxt],
        c->bk_ctl + 4 * nxt);
    GX_LAUNCHED(c);
    return GX_OK;
}

// dense pbuf[cur] -> bucketed pbuf[cur ^ 1] (becomes cur)
static int gx_bucketize(GxCtx* c) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    const int cur = c->cur, nxt = cur ^ 1;
    const unsigned nb = (unsigned)((std::max<int64_t>(n, 1) + 255) / 256);
    GX_CUDA(c, cudaMemsetAsync(c->bk_cnt, 0, sizeof(int32_t) * (g.nrow + 1), c->stream));
    if (n > 0) {
        auto kr = (g.ndim == 3) ? k_bk_rows<3> : k_bk_rows<2>;
        kr<<<nb, 256, 0, c->stream>>>(g, c->pbuf[cur], c->cap, n, c->pkey[0], c->bk_cnt);
        GX_LAUNCHED(c);
    }
    // segments of pbuf[nxt] from the exact counts (with_items = false plans
    // the layout of buffer "out ^ 1" = nxt from want = bk_cnt)
    int rc = bk_plan(c, cur, false);
    if (rc) return rc;
    if (n > 0) {
        k_bk_scatter<<<nb, 256, 0, c->stream>>>(c->pbuf[cur], c->pbuf[nxt], c->cap, n, bk_nplanes(c), c->origin,
                                                c->origin_tmp, c->pkey[0], c->bk_cap[nxt], c->bk_base[nxt],
                                                c->bk_fill[nxt], c->bk_ctl + 4 * nxt, c->bk_main);
        GX_LAUNCHED(c);
    }
    // items of pbuf[nxt]; segments of pbuf[cur] for the first fused pass
    rc = bk_plan(c, nxt, true);
    if (rc) return rc;
    std::swap(c->origin, c->origin_tmp);
    c->cur = nxt;
    c->bucketed = true;
    c->have_keys = false;
    return GX_OK;
}

__global__ void k_bk_iota(int32_t* p, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = (int32_t)i;
}

int gx_dense(GxCtx* c) {
    if (!c->bucketed) return GX_OK;
    const int cur = c->cur, nxt = cur ^ 1;
    int32_t* ctr = c->bk_ctl + 12;
    GX_CUDA(c, cudaMemsetAsync(ctr, 0, sizeof(int32_t), c->stream));
    k_bk_densify<<<148 * 8, 256, 0, c->stream>>>(c->pbuf[cur], c->pbuf[nxt], c->cap, bk_nplanes(c), c->origin,
                                                 c->origin_tmp, c->bk_items, c->bk_ctl + 8, ctr);
    GX_LAUNCHED(c);
    if (c->n > 0) {
        k_bk_iota<<<(unsigned)((c->n + 255) / 256), 256, 0, c->stream>>>(c->perm, c->n);
        GX_LAUNCHED(c);
    }
    std::swap(c->origin, c->origin_tmp);
    c->cur = nxt;
    c->bucketed = false;
    c->have_keys = false;
    return GX_OK;
}

template <int ND, bool COMP>
static int bk_launch_push(GxCtx* c, int cur, int nxt) {
    const DevGeo& g = c->g;
    const size_t sm = sizeof(unsigned long long) * (ND == 3 ? 16 : 4) * g.na;
    auto kp = k_push_bkt<ND, COMP>;
    GX_CUDA(c, cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    if (!c->bk_grid) {
        int per = 0, sms = 148;
        GX_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kp, BK_THREADS, sm));
        GX_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev));
        c->bk_grid = std::max(1, per) * sms;
    }
    kp<<<c->bk_grid, BK_THREADS, sm, c->stream>>>(g, c->pbuf[cur], c->pbuf[nxt], c->cap, c->origin,
                                                  c->origin_tmp, c->field, c->bk_items, c->bk_ctl + 8,
                                                  c->bk_cap[nxt], c->bk_base[nxt], c->bk_fill[nxt],
                                                  c->bk_ctl + 4 * nxt, c->bk_main, c->macc);
    GX_LAUNCHED(c);
    return GX_OK;
}

int gx_fast_step(GxCtx* c, int nsteps, int phys) {
    const DevGeo& g = c->g;
    int rc;
    if (!c->bucketed) {
        rc = gx_bucketize(c);
        if (rc) return rc;
    }
    for (int s = 0; s < nsteps; s++) {
        const bool last = (s == nsteps - 1);
        rc = gx_mixed_findf(c, phys && last, true);
        if (rc) return rc;
        const int cur = c->cur, nxt = cur ^ 1;
        rc = gx_phase_mark(c, PH_PUSH);
        if (rc) return rc;
        if (g.ndim == 3) rc = g.comp ? bk_launch_push<3, true>(c, cur, nxt) : bk_launch_push<3, false>(c, cur, nxt);
        else rc = g.comp ? bk_launch_push<2, true>(c, cur, nxt) : bk_launch_push<2, false>(c, cur, nxt);
        if (rc) return rc;
        rc = gx_phase_mark(c, PH_SORT);
        if (rc) return rc;
        rc = bk_plan(c, nxt, true);
        if (rc) return rc;
        rc = gx_phase_mark(c, PH_COMBINE);
        if (rc) return rc;
        k_mass_convert<<<(unsigned)((g.mesh / 2 + 255) / 256), 256, 0, c->stream>>>(c->macc, c->mass, g.mesh,
                                                                                   g.pmass);
        GX_LAUNCHED(c);
        std::swap(c->origin, c->origin_tmp);
        c->cur = nxt;
    }
    rc = gx_phase_end(c);
    if (rc) return rc;
    c->have_field = false;
    return GX_OK;
}
