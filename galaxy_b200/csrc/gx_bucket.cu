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
//   * bq[b] holds one segment of slots per row (row nrow: off the grid);
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
//     integers: into unsigned 32-bit shared-memory bins over the window of
//     rows around the item's row (4 rings, and 4 planes in 3D: every cell a
//     particle of the row can reach moving less than a cell), or, for
//     corners outside it (and the rare negative weight), straight into the
//     int64 mesh accumulator.  The bins are flushed into the accumulator
//     (nonzero bins only) after each item.  A bin cannot wrap: the linear
//     weights that reach it are >= 0 and <= 1 + 1e-4, each particle adds at
//     most one to a bin, and an item holds at most 4095 particles, so a bin
//     stays below 4095 (2^20 + 105) < 2^32.
//   * k_bk_plan (one CTA) turns the output buffer's row counts into its
//     work items, the next output buffer's segments and the active ring
//     range (jrad, krad); k_mass_convert turns the accumulator into the mass
//     array (x pmass) and clears it.
//
// Integer sums do not depend on their order, so the mass array is the same
// integers, converted the same way, as the sort-based deposit of
// gx_deposit.cu: the fused path is bitwise identical to it, whatever order
// the atomics resolve in.  A particle's record carries its load index;
// gx_dense() writes the store back to the n contiguous SoA particles of
// pbuf[cur] for the entry points that walk them that way (getacc, tmcent,
// icheck, the adjoint); unload writes the records straight from the store
// in load order, and masset deposits from the store with the same kernel
// run without the field and the move.
#include <algorithm>

#include "gx_common.cuh"

#define BK_FIXQ 1048576.0f  // 2^20: the fixed-point quantum of gx_deposit.cu
#define BK_SPARSE 256       // items with fewer particles add straight into the mesh
#define BK_THREADS 256
#define PLAN_THREADS 512
#define PLAN_ROWS 8         // rows per plan thread per pass
#ifndef BK_MINB
#define BK_MINB 5           // resident CTAs per SM the register budget is set for
#endif

__device__ __forceinline__ void red_add_s64(unsigned long long* a, int v) {
    atomicAdd(a, (unsigned long long)(long long)v);  // two's complement sum
}

// round(w 2^20) to the nearest integer, ties to even, for |w 2^20| < 2^22:
// adding 1.5 2^23 leaves the rounded integer in the low mantissa bits (the
// product by a power of two is exact, so one FMA rounds once, exactly as
// __float2int_rn(w * 2^20) does), on the FMA pipe instead of a conversion
__device__ __forceinline__ int bk_fix(float w) {
    return __float_as_int(fmaf(w, BK_FIXQ, 12582912.0f)) - 0x4B400000;
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
    constexpr int NWP = PLAN_THREADS / 32;  // warps (<= 32): lanes past them hold zeros
    static_assert(NWP <= 32, "one warp scans the warp totals");
    if (warp == 0) {
        int va = (lane < NWP) ? wa[lane] : 0, vb = (lane < NWP) ? wb[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int ya = __shfl_up_sync(0xffffffffu, va, o), yb = __shfl_up_sync(0xffffffffu, vb, o);
            if (lane >= o) {
                va += ya;
                vb += yb;
            }
        }
        if (lane < NWP) {
            wa[lane] = va;
            wb[lane] = vb;
        }
    }
    __syncthreads();
    const int pa = warp ? wa[warp - 1] : 0, pb = warp ? wb[warp - 1] : 0;
    ea = pa + xa - a;
    eb = pb + xb - b;
    ta = wa[NWP - 1];
    tb = wb[NWP - 1];
    __syncthreads();
}

// The plan of one step, one CTA:
//  * with fill_o: the work items of the buffer just written (fill_o, cap_o,
//    base_o, overflow count *ovf_o at slot ovf_base; each item: row, first
//    slot, end slot, ring of the row), and ctl[0] = items, ctl[1] = 0 (the
//    work counter);
//  * the segments of the buffer to be written next from the row counts
//    want: cap_n = want + want/8 + 16 (0 for empty rows), base_n their
//    exclusive sum; its fill counters and overflow count cleared.
// The row tables are padded with zeros to a multiple of PLAN_THREADS x
// PLAN_ROWS entries, so that every thread moves its eight consecutive rows
// with two 16-byte loads per table, all issued before they are used.
__device__ __forceinline__ void ld8(const int32_t* __restrict__ p, int r0, int* v) {
    const int4 a = __ldg(reinterpret_cast<const int4*>(p + r0));
    const int4 b = __ldg(reinterpret_cast<const int4*>(p + r0 + 4));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void st8(int32_t* __restrict__ p, int r0, const int* v) {
    reinterpret_cast<int4*>(p + r0)[0] = make_int4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<int4*>(p + r0)[1] = make_int4(v[4], v[5], v[6], v[7]);
}
static_assert(PLAN_ROWS == 8, "ld8 / st8 move eight rows");

__global__ void __launch_bounds__(PLAN_THREADS) k_bk_plan(
    int nrow1, int ngz, const int32_t* __restrict__ fill_o, const int32_t* __restrict__ cap_o,
    const int32_t* __restrict__ base_o, const int32_t* __restrict__ ovf_o, int64_t ovf_base,
    int4* __restrict__ items, int32_t* __restrict__ ctl,
    const int32_t* __restrict__ want, int32_t* __restrict__ cap_n, int32_t* __restrict__ base_n,
    int32_t* __restrict__ fill_n, int32_t* __restrict__ ovf_n, int item) {
    int carry_cap = 0, carry_it = 0;
    for (int c0 = 0; c0 < nrow1; c0 += PLAN_THREADS * PLAN_ROWS) {
        const int r0 = c0 + threadIdx.x * PLAN_ROWS;
        int wv[PLAN_ROWS], fv[PLAN_ROWS], cv[PLAN_ROWS], bv[PLAN_ROWS];
        ld8(want, r0, wv);
        if (fill_o) {
            ld8(fill_o, r0, fv);
            ld8(cap_o, r0, cv);
            ld8(base_o, r0, bv);
        }
        int capv[PLAN_ROWS], nit[PLAN_ROWS], val[PLAN_ROWS], zero[PLAN_ROWS];
        int scap = 0, snit = 0;
#pragma unroll
        for (int k = 0; k < PLAN_ROWS; k++) {
            const int w = wv[k];
            zero[k] = 0;
            capv[k] = w + (w >> 3) + (w > 0 ? 16 : 0);
            val[k] = nit[k] = 0;
            if (fill_o) {
                val[k] = min(fv[k], cv[k]);
                nit[k] = (val[k] + item - 1) / item;
            }
            scap += capv[k];
            snit += nit[k];
        }
        int ecap, eit, tcap, tit;
        plan_scan2(scap, snit, ecap, eit, tcap, tit);
        ecap += carry_cap;
        eit += carry_it;
        int basev[PLAN_ROWS];
#pragma unroll
        for (int k = 0; k < PLAN_ROWS; k++) {
            basev[k] = ecap;
            ecap += capv[k];
        }
        st8(cap_n, r0, capv);
        st8(base_n, r0, basev);
        st8(fill_n, r0, zero);
        if (fill_o) {
#pragma unroll
            for (int k = 0; k < PLAN_ROWS; k++) {
                const int ring = (r0 + k) / ngz;
                for (int q = 0; q < nit[k]; q++)
                    items[eit + q] = make_int4(r0 + k, bv[k] + q * item, bv[k] + min((q + 1) * item, val[k]), ring);
                eit += nit[k];
            }
        }
        carry_cap += tcap;
        carry_it += tit;
    }
    if (fill_o && threadIdx.x == 0) {
        const int ov = *ovf_o;
        int it = carry_it;
        for (int q = 0; q * item < ov; q++, it++)
            items[it] = make_int4(-1, (int)ovf_base + q * item, (int)ovf_base + min((q + 1) * item, ov), 0);
        ctl[0] = it;
        ctl[1] = 0;
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

// A particle of the bucketed store is one record: its NP floats (x, y[, z],
// vx, vy[, vz][, the compensated low parts]) then its load index as float
// bits, zero-padded to R float4 words.  The first two words of record s
// are bytes 32 s .. 32 s + 31 (moved with one 32-byte ld/st.v8 access, so a
// warp's loads of consecutive records are contiguous and each store writes
// a whole sector); a third word (the compensated 3D records, R = 3) sits in
// a plane of its own after them, at word 2 bcap + s.
template <int NP>
struct Rec {
    static constexpr int R = (NP + 1 + 3) / 4;
    static_assert(R >= 2 && R <= 3, "records of 5 to 12 floats");
};

__device__ __forceinline__ void ld8f(const float4* p, float* w) {
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(w[0]), "=f"(w[1]), "=f"(w[2]), "=f"(w[3]), "=f"(w[4]), "=f"(w[5]), "=f"(w[6]), "=f"(w[7])
                 : "l"(p));
}
__device__ __forceinline__ void st8f(float4* p, const float* w) {
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(w[0]), "f"(w[1]), "f"(w[2]),
                 "f"(w[3]), "f"(w[4]), "f"(w[5]), "f"(w[6]), "f"(w[7])
                 : "memory");
}

template <int NP>
__device__ __forceinline__ void rec_load(const float4* __restrict__ Q, int64_t bcap, int64_t s, float* P,
                                         int32_t& o) {
    constexpr int R = Rec<NP>::R;
    float w[4 * R];
    ld8f(Q + 2 * s, w);
    if (R == 3) {
        const float4 v = __ldg(Q + 2 * bcap + s);
        w[8] = v.x;
        w[9] = v.y;
        w[10] = v.z;
        w[11] = v.w;
    }
#pragma unroll
    for (int k = 0; k < NP; k++) P[k] = w[k];
    o = __float_as_int(w[NP]);
}

template <int NP>
__device__ __forceinline__ void rec_store(float4* __restrict__ Q, int64_t bcap, int64_t s, const float* P,
                                          int32_t o) {
    constexpr int R = Rec<NP>::R;
    float w[4 * R];
#pragma unroll
    for (int k = 0; k < 4 * R; k++) w[k] = (k < NP) ? P[k] : 0.f;
    w[NP] = __int_as_float(o);
    st8f(Q + 2 * s, w);
    if (R == 3) Q[2 * bcap + s] = make_float4(w[8], w[9], w[10], w[11]);
}

// The fused particle pass of one step.  Persistent CTAs take work items from
// a counter.  bins: int64 [WROWS][na] over the item's window, zero between
// items.  Window of an item of row (ir, iz): rings ir - 1 .. ir + 2 and, in
// 3D, planes iz - 1 .. iz + 2 (bin row 4 a + b for ring ir - 1 + a, plane
// iz - 1 + b); 2D: rows ir - 1 .. ir + 2.
// DEP: the deposit alone (masset on the bucketed store): the cell of each
// particle's current position, its weights into the bins and the mesh, the
// ring and plane range; no field, no move, the store is not rewritten
template <int ND, bool COMP, bool DEP = false>
__global__ void __launch_bounds__(BK_THREADS, BK_MINB) k_push_bkt(
    DevGeo g, const float4* __restrict__ Qin, float4* __restrict__ Qout, int64_t bcap,
    const float4* __restrict__ F,
    const int4* __restrict__ items, int32_t* __restrict__ ctl, const int32_t* __restrict__ cap_o,
    const int32_t* __restrict__ base_o, int32_t* __restrict__ fill_o, int32_t* __restrict__ ovf_o,
    int64_t ovf_base, unsigned long long* __restrict__ acc) {
    extern __shared__ __align__(16) uint32_t bins[];
    __shared__ int s_item;
    constexpr bool d3 = ND == 3;
    constexpr int WROWS = d3 ? 16 : 4;
    constexpr int NW = 2 * ND;
    const int na = g.na, ngz = d3 ? g.ngz : 1, nrow = g.nrow;
    const int nit = ctl[0];
    int rmin_l = 0x7fffffff, rmax_l = -1;  // ring range of this lane's new cells
    int zmin_l = 0x7fffffff, zmax_l = -1;  // and their plane range (3D)
    for (int i = threadIdx.x; i < WROWS * na; i += BK_THREADS) bins[i] = 0u;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(ctl + 1, 1);
        __syncthreads();  // also orders the previous item's flush before these deposits
        const int it = s_item;
        if (it >= nit) break;
        const int4 I = items[it];
        const int row = I.x, s0 = I.y, s1 = I.z;
        const bool win = row >= 0 && row < nrow && (s1 - s0) >= BK_SPARSE;
        // ring and plane of the item's row (the plan stores the ring): the
        // window's origin is one below
        const int wir = I.w;
        const int wiz = d3 ? row - wir * ngz : 0;
        constexpr int NP = NW + (COMP ? ND : 0);
        constexpr int NQC = d3 ? 4 : 2;  // corner rows of a cell
        for (int b0 = s0; b0 < s1; b0 += BK_THREADS) {
            const int s = b0 + threadIdx.x;
            const bool act = s < s1;
            float P[NP];
            int32_t o = 0;
            CellW cn;
            cn.key = -1;
            uint32_t rk = 0;
            if (act) {
                rec_load<NP>(Qin, bcap, s, P, o);
                float &x = P[0], &y = P[1];
                float z = d3 ? P[2] : 0.f;
                if (!DEP) {
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
                }
                cn = gx_cell_t<true, ND>(g, x, y, z, false);
                rk = (cn.key >= 0) ? (uint32_t)cn.row : (uint32_t)nrow;
                if (cn.key >= 0) {
                    rmin_l = min(rmin_l, cn.ju);
                    rmax_l = max(rmax_l, cn.ju);
                    if (d3) {
                        // a cell in the top plane (a spoke coordinate that
                        // rounded up to na moved it there) has its upper
                        // corners in plane 0 of the next ring
                        zmin_l = min(zmin_l, (cn.iz + 1 == ngz) ? 0 : cn.iz);
                        zmax_l = max(zmax_l, cn.iz);
                    }
                }
            }
            // the row's slot: warp-aggregated atomic on its fill counter,
            // issued before the deposit so that its latency overlaps it
            const unsigned lane = threadIdx.x & 31;
            uint32_t peers = 0;
            int leader = -1, bslot = 0, capr = 0, baser = 0;
            if (!DEP) {
                const uint32_t am = __ballot_sync(0xffffffffu, act);
                peers = __match_any_sync(0xffffffffu, act ? rk : 0xffffffffu) & am;
                leader = __ffs(peers) - 1;
                if (act && (int)lane == leader) bslot = atomicAdd(fill_o + rk, __popc(peers));
                if (act) {
                    capr = __ldg(cap_o + rk);
                    baser = __ldg(base_o + rk);
                }
            }
            // the common case: every corner inside the window (the new cell
            // in its inner 3 x 3 rows, or 3 rows in 2D, no plane wrap, inside
            // the mesh) and no negative weight: eight shared-memory adds
            int va[8];
            bool fast = false;
            if (act && cn.key >= 0) {
                float w[8];
                gx_weights<ND>(g, cn, w);
                int neg = 0;
#pragma unroll
                for (int k = 0; k < 2 * NQC; k++) {
                    va[k] = bk_fix(w[k]);
                    neg |= va[k];
                }
                const int a0 = d3 ? cn.ju - wir + 1 : cn.row - row + 1;
                const int b0 = d3 ? cn.iz - wiz + 1 : 0;
                fast = win && neg >= 0 && (unsigned)a0 <= 2u && (unsigned)b0 <= 2u &&
                       (d3 ? (cn.iz + 1 < ngz && cn.ju + 1 < g.nr) : cn.row + 1 < nrow);
                if (fast) {
                    const int jt0 = cn.jt, jt1 = (cn.jt == na - 1) ? 0 : cn.jt + 1;
                    uint32_t* b = bins + (d3 ? 4 * a0 + b0 : a0) * na;
#pragma unroll
                    for (int q = 0; q < NQC; q++) {
                        // corner row q: + 1 (next plane / ring), + ngz (next ring): bin rows + 1, + 4
                        uint32_t* br = b + (d3 ? (q & 1) + 4 * (q >> 1) : q) * na;
                        atomicAdd(br + jt0, (uint32_t)va[2 * q]);
                        atomicAdd(br + jt1, (uint32_t)va[2 * q + 1]);
                    }
                }
            }
            if (act && cn.key >= 0 && !fast) {
                const int jt0 = cn.jt, jt1 = (cn.jt == na - 1) ? 0 : cn.jt + 1;
                // the corner rows: row, row + 1 (the next plane, or ring in
                // 2D), and in 3D row + ngz, row + ngz + 1, with their window
                // coordinates (a, b)
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
                    const int v0 = va[2 * q];
                    const int v1 = va[2 * q + 1];
                    const bool inw = win && wa[q] >= 0 && wa[q] < 4 && wb[q] >= 0 && wb[q] < 4;
                    unsigned long long* ar = acc + (size_t)fr[q] * na;
                    uint32_t* br = bins + (inw ? (d3 ? 4 * wa[q] + wb[q] : wa[q]) * na : 0);
                    if (inw && v0 > 0) atomicAdd(br + jt0, (uint32_t)v0);
                    else if (v0) red_add_s64(ar + jt0, v0);
                    if (inw && v1 > 0) atomicAdd(br + jt1, (uint32_t)v1);
                    else if (v1) red_add_s64(ar + jt1, v1);
                }
            }
            if (!DEP) {
                bslot = __shfl_sync(0xffffffffu, bslot, leader < 0 ? 0 : leader);
                const int slot = bslot + __popc(peers & lanemask_lt());
                int64_t dst = (int64_t)baser + slot;
                const bool ovf = act && slot >= capr;
                const uint32_t om = __ballot_sync(0xffffffffu, ovf);
                if (om) {
                    const int ol = __ffs(om) - 1;
                    int ob = 0;
                    if ((int)lane == ol) ob = atomicAdd(ovf_o, __popc(om));
                    ob = __shfl_sync(0xffffffffu, ob, ol);
                    if (ovf) dst = ovf_base + ob + __popc(om & lanemask_lt());
                }
                if (act) rec_store<NP>(Qout, bcap, dst, P, o);
            }
        }
        if (win) {
            __syncthreads();
#pragma unroll 4
            for (int wr = 0; wr < WROWS; wr++) {
                const int R = d3 ? (wir - 1 + (wr >> 2)) * ngz + (wiz - 1 + (wr & 3)) : wir - 1 + wr;
                uint32_t* br = bins + wr * na;
                for (int j = threadIdx.x; j < na; j += BK_THREADS) {
                    const uint32_t v = br[j];
                    if (v) {
                        atomicAdd(acc + (size_t)R * na + j, (unsigned long long)v);
                        br[j] = 0u;
                    }
                }
            }
        }
        __syncthreads();  // s_item is rewritten by thread 0 next
    }
    // the ring range of the new cells (massgn's jrad / krad): one atomic
    // pair per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rmin_l = min(rmin_l, __shfl_xor_sync(0xffffffffu, rmin_l, o));
        rmax_l = max(rmax_l, __shfl_xor_sync(0xffffffffu, rmax_l, o));
        zmin_l = min(zmin_l, __shfl_xor_sync(0xffffffffu, zmin_l, o));
        zmax_l = max(zmax_l, __shfl_xor_sync(0xffffffffu, zmax_l, o));
    }
    if ((threadIdx.x & 31) == 0 && rmax_l >= 0) {
        atomicMin(ctl + 5, rmin_l);
        atomicMax(ctl + 6, rmax_l);
        if (d3) {
            atomicMin(ctl + 2, zmin_l);
            atomicMax(ctl + 3, zmax_l);
        }
    }
}

// mass = pmass 2^-20 acc (as k_mass_combine forms it); acc cleared for the
// next step.  Two cells per thread (mesh is even: na is).
__global__ void k_mass_convert(unsigned long long* __restrict__ acc, float* __restrict__ mass, int mesh,
                               float pm, int32_t* __restrict__ rng, int32_t* __restrict__ jrk, int nr,
                               int32_t* __restrict__ zrng, int32_t* __restrict__ zr, int ngz) {
    // the active ring range of the new mass, as massgn tracks it (jrad =
    // first ring + 1, krad = min(last ring + 2, nr), 1-based), from the ring
    // range the push gathered (rng[0], rng[1]); the planes holding mass
    // (the cells' planes and the next, clamped) from its plane range; both
    // reset for the next pass
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int mn = rng[0], mx = rng[1];
        jrk[0] = (mx >= 0) ? mn + 1 : nr;
        jrk[1] = (mx >= 0) ? min(mx + 2, nr) : 0;
        rng[0] = 0x7fffffff;
        rng[1] = -1;
        const int zn = zrng[0], zx = zrng[1];
        zr[0] = (zx >= 0) ? zn : ngz;
        zr[1] = (zx >= 0) ? min(zx + 1, ngz - 1) : -1;
        zrng[0] = 0x7fffffff;
        zrng[1] = -1;
    }
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

// The same two steps with the counts gathered per CTA first (grids whose row
// table fits in shared memory): a CTA takes a run of BK_RUN particles, counts
// their rows in shared memory, and touches each global counter once per
// nonzero row instead of once per warp group -- a disc's central rows get
// tens of thousands of particles, whose single-address atomics otherwise
// serialise.  The scatter reserves each row's slots for the CTA with one
// atomic on the row's fill counter and hands them out from shared memory.
#define BK_RUN 32768
template <int ND>
__global__ void __launch_bounds__(256) k_bk_rows_cta(DevGeo g, const float* __restrict__ P, int64_t cap,
                                                     int64_t n, int32_t* __restrict__ rows,
                                                     int32_t* __restrict__ cnt) {
    extern __shared__ int32_t hist[];  // [nrow + 1]
    const int nr1 = g.nrow + 1;
    for (int r = threadIdx.x; r < nr1; r += blockDim.x) hist[r] = 0;
    __syncthreads();
    const int64_t i0 = (int64_t)blockIdx.x * BK_RUN, i1 = min(n, i0 + BK_RUN);
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const CellW c = gx_cell_t<true, ND>(g, P[i], P[cap + i], ND == 3 ? P[2 * cap + i] : 0.f, false);
        const int rk = (c.key >= 0) ? c.row : g.nrow;
        rows[i] = rk;
        atomicAdd(hist + rk, 1);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nr1; r += blockDim.x)
        if (hist[r]) atomicAdd(cnt + r, hist[r]);
}

template <int NP>
__global__ void __launch_bounds__(256) k_bk_scatter_cta(const float* __restrict__ P, int64_t cap, int64_t n,
                                                        const int32_t* __restrict__ oin, float4* __restrict__ Qout,
                                                        int64_t bcap, const int32_t* __restrict__ rows, int nr1,
                                                        const int32_t* __restrict__ cap_o,
                                                        const int32_t* __restrict__ base_o,
                                                        int32_t* __restrict__ fill_o, int32_t* __restrict__ ovf_o,
                                                        int64_t ovf_base) {
    extern __shared__ int32_t slot[];  // [nrow + 1]: this CTA's count, then its next slot
    for (int r = threadIdx.x; r < nr1; r += blockDim.x) slot[r] = 0;
    __syncthreads();
    const int64_t i0 = (int64_t)blockIdx.x * BK_RUN, i1 = min(n, i0 + BK_RUN);
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) atomicAdd(slot + rows[i], 1);
    __syncthreads();
    for (int r = threadIdx.x; r < nr1; r += blockDim.x)
        if (slot[r]) slot[r] = atomicAdd(fill_o + r, slot[r]);
    __syncthreads();
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const int rk = rows[i];
        const int sl = atomicAdd(slot + rk, 1);
        int64_t dst;
        if (sl < __ldg(cap_o + rk)) dst = (int64_t)__ldg(base_o + rk) + sl;
        else dst = ovf_base + atomicAdd(ovf_o, 1);  // past the segment (rare): the overflow area
        float w[NP];
#pragma unroll
        for (int k = 0; k < NP; k++) w[k] = P[(size_t)k * cap + i];
        rec_store<NP>(Qout, bcap, dst, w, oin[i]);
    }
}

template <int NP>
__global__ void k_bk_scatter(const float* __restrict__ P, int64_t cap, int64_t n, const int32_t* __restrict__ oin,
                             float4* __restrict__ Qout, int64_t bcap, const int32_t* __restrict__ rows,
                             const int32_t* __restrict__ cap_o, const int32_t* __restrict__ base_o,
                             int32_t* __restrict__ fill_o, int32_t* __restrict__ ovf_o, int64_t ovf_base) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool act = i < n;
    const uint32_t rk = act ? (uint32_t)rows[i] : 0u;
    const int64_t dst = bk_slot(act, rk, cap_o, base_o, fill_o, ovf_o, ovf_base);
    if (!act) return;
    float w[NP];
#pragma unroll
    for (int k = 0; k < NP; k++) w[k] = P[(size_t)k * cap + i];
    rec_store<NP>(Qout, bcap, dst, w, oin[i]);
}

// bucketed store -> n contiguous particles (SoA planes and load index),
// item by item (CTA-reserved ranges)
template <int NP>
__global__ void k_bk_densify(const float4* __restrict__ Qin, int64_t bcap, float* __restrict__ P, int64_t cap,
                             int32_t* __restrict__ oout, const int4* __restrict__ items,
                             const int32_t* __restrict__ ctl, int32_t* __restrict__ dense_ctr) {
    __shared__ int s_d0;
    const int nit = ctl[0];
    for (int it = blockIdx.x; it < nit; it += gridDim.x) {
        const int4 I = items[it];
        if (threadIdx.x == 0) s_d0 = atomicAdd(dense_ctr, I.z - I.y);
        __syncthreads();
        const int d0 = s_d0;
        for (int s = I.y + threadIdx.x; s < I.z; s += blockDim.x) {
            const int64_t d = d0 + (s - I.y);
            float w[NP];
            int32_t o;
            rec_load<NP>(Qin, bcap, s, w, o);
#pragma unroll
            for (int k = 0; k < NP; k++) P[(size_t)k * cap + d] = w[k];
            oout[d] = o;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
bool gx_fast_ok(const GxCtx* c) {
    return !c->fp64 && c->nzones == 1 && !c->g.quad && !(c->cfg.flags & GX_FLAG_SORTED_DEPOSIT);
}

static inline int bk_nplanes(const GxCtx* c) { return 2 * c->g.ndim + (c->g.comp ? c->g.ndim : 0); }

// bucketed store -> the host records (x, y[, z], vx, vy[, vz]) in load
// order, in two passes: k_bk_inv writes each record's slot at its load
// index (4-byte scattered writes into an n-entry table that stays in L2),
// k_bk_gather walks the load indices in order, reads each record (one
// 32-byte access) and writes the host layout contiguously.  Writing the
// 16 / 24-byte records straight to their scattered load positions (one
// pass) made partial-sector writes over an output larger than L2.
template <int NP>
__global__ void k_bk_inv(const float4* __restrict__ Qin, int64_t bcap, int32_t* __restrict__ inv,
                         const int4* __restrict__ items, const int32_t* __restrict__ ctl) {
    const int nit = ctl[0];
    for (int it = blockIdx.x; it < nit; it += gridDim.x) {
        const int4 I = items[it];
        for (int s = I.y + threadIdx.x; s < I.z; s += blockDim.x) {
            float w[NP];
            int32_t o;
            rec_load<NP>(Qin, bcap, s, w, o);
            inv[o] = s;
        }
    }
}

template <int NP, int NW>
__global__ void k_bk_gather(const float4* __restrict__ Qin, int64_t bcap, const int32_t* __restrict__ inv,
                            float* __restrict__ aos, int64_t n) {
    static_assert(NW == 4 || NW == 6, "2D or 3D records");
    const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (o >= n) return;
    float w[NP];
    int32_t oo;
    rec_load<NP>(Qin, bcap, __ldg(inv + o), w, oo);
    if (NW == 4) {
        reinterpret_cast<float4*>(aos)[o] = make_float4(w[0], w[1], w[2], w[3]);
    } else {
        float2* d = reinterpret_cast<float2*>(aos + (size_t)o * 6);
        d[0] = make_float2(w[0], w[1]);
        d[1] = make_float2(w[2], w[3]);
        d[2] = make_float2(w[4], w[5]);
    }
}

template <int NP, int NW>
static void bk_unload_launch(GxCtx* c, float* aos) {
    int32_t* inv = c->pkey[0];  // free while the store is bucketed (the keys are recomputed after it)
    k_bk_inv<NP><<<148 * 8, 256, 0, c->stream>>>(c->bq[c->bcur], c->bcap, inv, c->bk_items, c->bk_ctl + 8);
    k_bk_gather<NP, NW><<<(unsigned)((c->n + 255) / 256), 256, 0, c->stream>>>(c->bq[c->bcur], c->bcap, inv,
                                                                                aos, c->n);
}

// float4 words of one record of the bucketed store
int gx_bucket_words(const GxCtx* c) { return (bk_nplanes(c) + 1 + 3) / 4; }

static inline size_t bk_npad(const GxCtx* c);
static int bk_plan(GxCtx* c, int out, bool with_items, cudaStream_t st);

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
static inline size_t bk_npad(const GxCtx* c) {
    const size_t per = (size_t)PLAN_THREADS * PLAN_ROWS;
    return ((size_t)c->g.nrow + 1 + per - 1) / per * per;
}

int gx_bucket_alloc(GxCtx* c) {
    const size_t nrow1 = bk_npad(c);
    int rc = 0;
    for (int b = 0; b < 2 && !rc; b++) {
        rc = rc ? rc : bk_alloc(c, &c->bk_cap[b], nrow1);
        rc = rc ? rc : bk_alloc(c, &c->bk_base[b], nrow1);
        rc = rc ? rc : bk_alloc(c, &c->bk_fill[b], nrow1);
    }
    rc = rc ? rc : bk_alloc(c, &c->bk_ctl, 16);
    rc = rc ? rc : bk_alloc(c, &c->bk_cnt, nrow1);
    rc = rc ? rc : bk_alloc(c, &c->macc, (size_t)c->g.mesh);
    rc = rc ? rc : bk_alloc(c, &c->zr_d, 4);
    if (rc) return rc;
    for (int b = 0; b < 2; b++) {
        GX_CUDA(c, cudaMemsetAsync(c->bk_fill[b], 0, sizeof(int32_t) * nrow1, c->stream));
        GX_CUDA(c, cudaMemsetAsync(c->bk_cap[b], 0, sizeof(int32_t) * nrow1, c->stream));
        GX_CUDA(c, cudaMemsetAsync(c->bk_base[b], 0, sizeof(int32_t) * nrow1, c->stream));
    }
    GX_CUDA(c, cudaMemsetAsync(c->macc, 0, sizeof(unsigned long long) * c->g.mesh, c->stream));
    const int32_t ctl0[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0x7fffffff, -1, 0, 0x7fffffff, -1, 0};
    GX_CUDA(c, cudaMemcpyAsync(c->bk_ctl, ctl0, sizeof ctl0, cudaMemcpyHostToDevice, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

static int bk_plan(GxCtx* c, int out, bool with_items, cudaStream_t st) {
    const DevGeo& g = c->g;
    const int nxt = out ^ 1;
    k_bk_plan<<<1, PLAN_THREADS, 0, st>>>(
        g.nrow + 1, g.ngz, with_items ? c->bk_fill[out] : nullptr, c->bk_cap[out], c->bk_base[out],
        c->bk_ctl + 4 * out, c->bk_main, c->bk_items, c->bk_ctl + 8,
        with_items ? c->bk_fill[out] : c->bk_cnt, c->bk_cap[nxt], c->bk_base[nxt], c->bk_fill[nxt],
        c->bk_ctl + 4 * nxt, c->bk_item);
    GX_LAUNCHED(c);
    return GX_OK;
}

template <int NP>
static void bk_scatter_cta_launch(GxCtx* c, int b) {
    const int nr1 = c->g.nrow + 1;
    const unsigned nruns = (unsigned)((c->n + BK_RUN - 1) / BK_RUN);
    cudaFuncSetAttribute(k_bk_scatter_cta<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(int32_t) * nr1));
    k_bk_scatter_cta<NP><<<nruns, 256, sizeof(int32_t) * nr1, c->stream>>>(
        c->pbuf[c->cur], c->cap, c->n, c->origin, c->bq[b], c->bcap, c->pkey[0], nr1, c->bk_cap[b], c->bk_base[b],
        c->bk_fill[b], c->bk_ctl + 4 * b, c->bk_main);
}

template <int NP>
static void bk_scatter_launch(GxCtx* c, unsigned nb, int b) {
    k_bk_scatter<NP><<<nb, 256, 0, c->stream>>>(c->pbuf[c->cur], c->cap, c->n, c->origin, c->bq[b], c->bcap,
                                                c->pkey[0], c->bk_cap[b], c->bk_base[b], c->bk_fill[b],
                                                c->bk_ctl + 4 * b, c->bk_main);
}

template <int NP>
static void bk_densify_launch(GxCtx* c, int32_t* ctr) {
    k_bk_densify<NP><<<148 * 8, 256, 0, c->stream>>>(c->bq[c->bcur], c->bcap, c->pbuf[c->cur], c->cap,
                                                     c->origin, c->bk_items, c->bk_ctl + 8, ctr);
}

// the dense store pbuf[cur] -> the bucketed store bq[b], b = bcur ^ 1
// (becomes bcur); the dense store is left as it was, and is stale from the
// first fused step on
static int gx_bucketize(GxCtx* c) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    const int b = c->bcur ^ 1;
    const unsigned nb = (unsigned)((std::max<int64_t>(n, 1) + 255) / 256);
    GX_CUDA(c, cudaMemsetAsync(c->bk_cnt, 0, sizeof(int32_t) * bk_npad(c), c->stream));
    // the row table in shared memory when it fits in 96 KB (two CTAs per SM)
    const size_t hbytes = sizeof(int32_t) * ((size_t)g.nrow + 1);
    const bool cta = hbytes <= 96 * 1024;
    if (n > 0) {
        if (cta) {
            auto kr = (g.ndim == 3) ? k_bk_rows_cta<3> : k_bk_rows_cta<2>;
            cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hbytes);
            kr<<<(unsigned)((n + BK_RUN - 1) / BK_RUN), 256, hbytes, c->stream>>>(g, c->pbuf[c->cur], c->cap, n,
                                                                                c->pkey[0], c->bk_cnt);
        } else {
            auto kr = (g.ndim == 3) ? k_bk_rows<3> : k_bk_rows<2>;
            kr<<<nb, 256, 0, c->stream>>>(g, c->pbuf[c->cur], c->cap, n, c->pkey[0], c->bk_cnt);
        }
        GX_LAUNCHED(c);
    }
    // segments of bq[b] from the exact counts (with_items = false plans the
    // layout of buffer "out ^ 1" = b from want = bk_cnt)
    int rc = bk_plan(c, b ^ 1, false, c->stream);
    if (rc) return rc;
    if (n > 0) {
        switch (bk_nplanes(c)) {
            case 4: cta ? bk_scatter_cta_launch<4>(c, b) : bk_scatter_launch<4>(c, nb, b); break;
            case 6: cta ? bk_scatter_cta_launch<6>(c, b) : bk_scatter_launch<6>(c, nb, b); break;
            default: cta ? bk_scatter_cta_launch<9>(c, b) : bk_scatter_launch<9>(c, nb, b); break;
        }
        GX_LAUNCHED(c);
    }
    // items of bq[b]; segments of bq[b ^ 1] for the first fused pass
    rc = bk_plan(c, b, true, c->stream);
    if (rc) return rc;
    c->bcur = b;
    c->bucketed = true;
    c->have_keys = false;
    return GX_OK;
}

__global__ void k_bk_iota(int32_t* p, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = (int32_t)i;
}

// bucketed store -> the dense store pbuf[cur] (its SoA planes and load
// index), in the store's row order; the processing order becomes the
// identity
int gx_dense(GxCtx* c) {
    if (!c->bucketed) return GX_OK;
    int32_t* ctr = c->bk_ctl + 12;
    GX_CUDA(c, cudaMemsetAsync(ctr, 0, sizeof(int32_t), c->stream));
    switch (bk_nplanes(c)) {
        case 4: bk_densify_launch<4>(c, ctr); break;
        case 6: bk_densify_launch<6>(c, ctr); break;
        default: bk_densify_launch<9>(c, ctr); break;
    }
    GX_LAUNCHED(c);
    if (c->n > 0) {
        k_bk_iota<<<(unsigned)((c->n + 255) / 256), 256, 0, c->stream>>>(c->perm, c->n);
        GX_LAUNCHED(c);
    }
    c->bucketed = false;
    c->have_keys = false;
    return GX_OK;
}

// gx_unload's records from the bucketed store (the store stays as it is)
int gx_bucket_unload(GxCtx* c, float* aos) {
    if (c->n <= 0) return GX_OK;
    // record planes: the phase space (2D: 4, 3D: 6) and the compensated
    // update's low parts of the positions
    if (c->g.ndim == 3) {
        if (c->g.comp) bk_unload_launch<9, 6>(c, aos);
        else bk_unload_launch<6, 6>(c, aos);
    } else {
        if (c->g.comp) bk_unload_launch<6, 4>(c, aos);
        else bk_unload_launch<4, 4>(c, aos);
    }
    c->launches++;  // two kernels: the inversion and the gather
    GX_LAUNCHED(c);
    return GX_OK;
}

template <int ND, bool COMP, bool DEP = false>
static int bk_launch_push(GxCtx* c, int cur, int nxt) {
    const DevGeo& g = c->g;
    const size_t sm = sizeof(uint32_t) * (ND == 3 ? 16 : 4) * g.na;
    auto kp = k_push_bkt<ND, COMP, DEP>;
    GX_CUDA(c, cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    if (!c->bk_grid) {
        int per = 0, sms = 148;
        GX_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_push_bkt<ND, COMP>, BK_THREADS, sm));
        GX_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev));
        c->bk_grid = std::max(1, per) * sms;
    }
    kp<<<c->bk_grid, BK_THREADS, sm, c->stream>>>(g, c->bq[cur], c->bq[nxt], c->bcap, c->field, c->bk_items,
                                                  c->bk_ctl + 8, c->bk_cap[nxt], c->bk_base[nxt],
                                                  c->bk_fill[nxt], c->bk_ctl + 4 * nxt, c->bk_main, c->macc);
    GX_LAUNCHED(c);
    return GX_OK;
}

// the main stream waits for the plan queued on the side stream
static int bk_join(GxCtx* c) {
    if (!c->bk_pending) return GX_OK;
    GX_CUDA(c, cudaStreamWaitEvent(c->stream, c->bk_ev[1], 0));
    c->bk_pending = false;
    return GX_OK;
}

// masset on the fused path: the deposit-only pass over the bucketed store
// (bucketized first when the particles are dense), then the conversion.
// The mass is the same integers, converted the same way, as the sorted
// deposit's (massgn.f:140-172), and the ring and plane ranges of the mass
// are known to the next solve.
int gx_fast_masset(GxCtx* c) {
    const DevGeo& g = c->g;
    int rc = c->bucketed ? bk_join(c) : gx_bucketize(c);
    if (rc) return rc;
    const int cur = c->bcur, nxt = cur ^ 1;
    if (g.ndim == 3)
        rc = g.comp ? bk_launch_push<3, true, true>(c, cur, nxt) : bk_launch_push<3, false, true>(c, cur, nxt);
    else
        rc = g.comp ? bk_launch_push<2, true, true>(c, cur, nxt) : bk_launch_push<2, false, true>(c, cur, nxt);
    if (rc) return rc;
    // the pass took the items through the work counter: the next pass starts it afresh
    GX_CUDA(c, cudaMemsetAsync(c->bk_ctl + 9, 0, sizeof(int32_t), c->stream));
    k_mass_convert<<<(unsigned)((g.mesh / 2 + 255) / 256), 256, 0, c->stream>>>(
        c->macc, c->mass, g.mesh, g.pmass, c->bk_ctl + 13, c->jrk_d, g.nr, c->bk_ctl + 10, c->zr_d, g.ngz);
    GX_LAUNCHED(c);
    c->zr_valid = true;
    return GX_OK;
}

// one fused step: the solve of the current mass (only the planes that hold
// it once they are known), the pass, its plan on the side stream, the mass
static int fast_one_step(GxCtx* c, bool lpot) {
    const DevGeo& g = c->g;
    // once the mass is a fused pass's, the solve knows the planes that
    // hold it, and the field is needed only where the particles are
    int rc = gx_mixed_findf(c, lpot ? 1 : 0, true, nullptr, (c->zr_valid && g.ndim == 3) ? c->zr_d : nullptr);
    if (rc) return rc;
    const int cur = c->bcur, nxt = cur ^ 1;
    rc = bk_join(c);
    if (rc) return rc;
    rc = gx_phase_mark(c, PH_PUSH);
    if (rc) return rc;
    if (g.ndim == 3) rc = g.comp ? bk_launch_push<3, true>(c, cur, nxt) : bk_launch_push<3, false>(c, cur, nxt);
    else rc = g.comp ? bk_launch_push<2, true>(c, cur, nxt) : bk_launch_push<2, false>(c, cur, nxt);
    if (rc) return rc;
    if (c->prof) {
        // profile mode: the plan in line, so that it has a phase time
        rc = gx_phase_mark(c, PH_SORT);
        if (rc) return rc;
        rc = bk_plan(c, nxt, true, c->stream);
        if (rc) return rc;
    } else {
        // the plan needs only the push: it runs on the side stream while
        // the next field solve runs, and the next push waits for it
        GX_CUDA(c, cudaEventRecord(c->bk_ev[0], c->stream));
        GX_CUDA(c, cudaStreamWaitEvent(c->bk_side, c->bk_ev[0], 0));
        rc = bk_plan(c, nxt, true, c->bk_side);
        if (rc) return rc;
        GX_CUDA(c, cudaEventRecord(c->bk_ev[1], c->bk_side));
        c->bk_pending = true;
    }
    rc = gx_phase_mark(c, PH_COMBINE);
    if (rc) return rc;
    k_mass_convert<<<(unsigned)((g.mesh / 2 + 255) / 256), 256, 0, c->stream>>>(
        c->macc, c->mass, g.mesh, g.pmass, c->bk_ctl + 13, c->jrk_d, g.nr, c->bk_ctl + 10, c->zr_d, g.ngz);
    GX_LAUNCHED(c);
    c->zr_valid = true;
    c->bcur = nxt;
    return GX_OK;
}

// two fused steps from the current store captured into a CUDA graph (the
// plans forked to the side stream and joined inside it): the graph, and the
// kernels of one replay in *per; null when the capture is refused, and the
// steps then run as plain launches.  Capturing runs nothing: the host state
// the two steps would change is put back.
static cudaGraphExec_t fast_capture(GxCtx* c, int64_t* per) {
    const int b = c->bcur;
    if (bk_join(c) != GX_OK) return nullptr;
    const int64_t l0 = c->launches;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // a stream the caller is capturing already is left alone
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return nullptr;
    }
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    bool ok = fast_one_step(c, false) == GX_OK && fast_one_step(c, false) == GX_OK && bk_join(c) == GX_OK;
    const cudaError_t ec = cudaStreamEndCapture(c->stream, &graph);
    ok = ok && ec == cudaSuccess && graph;
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    *per = c->launches - l0;
    c->bcur = b;
    c->bk_pending = false;
    c->launches = l0;
    c->err.clear();
    return ok ? exec : nullptr;
}

int gx_fast_step(GxCtx* c, int nsteps, int phys) {
    int rc;
    if (!c->bk_side) {
        int lo = 0, hi = 0;
        GX_CUDA(c, cudaDeviceGetStreamPriorityRange(&lo, &hi));
        GX_CUDA(c, cudaStreamCreateWithPriority(&c->bk_side, cudaStreamNonBlocking, hi));
        GX_CUDA(c, cudaEventCreateWithFlags(&c->bk_ev[0], cudaEventDisableTiming));
        GX_CUDA(c, cudaEventCreateWithFlags(&c->bk_ev[1], cudaEventDisableTiming));
    }
    if (!c->bucketed) {
        rc = gx_bucketize(c);
        if (rc) return rc;
    }
    // 2D contexts (small grids: their steps take tens of microseconds, so the
    // gaps between launches count) replay pairs of steps from a CUDA graph,
    // captured in this call once the state is steady (the mass a fused
    // pass's, every buffer allocated) and released at its end
    const bool graphs = c->g.ndim == 2 && !c->prof && c->nranks <= 1;
    cudaGraphExec_t exec = nullptr;
    int64_t per = 0;
    bool tried = false;
    int s = 0;
    while (s < nsteps) {
        const bool last = (s == nsteps - 1);
        const int pairs = (nsteps - s - 1) / 2;  // the last step runs as plain launches (phys)
        if (graphs && c->zr_valid && pairs >= 4 && !tried) {
            tried = true;
            exec = fast_capture(c, &per);
        }
        if (exec && pairs > 0) {
            rc = bk_join(c);
            if (rc) break;
            for (int p = 0; p < pairs && !rc; p++) {
                if (cudaGraphLaunch(exec, c->stream) != cudaSuccess) rc = (c->err = "cudaGraphLaunch failed", GX_ERR_CUDA);
                c->launches += per;
            }
            if (rc) break;
            s += 2 * pairs;
            continue;
        }
        rc = fast_one_step(c, phys && last);
        if (rc) break;
        s++;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (rc) return rc;
    rc = bk_join(c);
    if (rc) return rc;
    rc = gx_phase_end(c);
    if (rc) return rc;
    c->have_field = false;
    return GX_OK;
}
