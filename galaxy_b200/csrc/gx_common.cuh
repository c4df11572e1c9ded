// gx_common.cuh -- shared device/host definitions of the B200 polar-grid
// particle-mesh library (context, geometry constants, cell-key arithmetic).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/galaxy_gpu.h"

#define GX_PI 3.141592653589793238462643

// ---------------------------------------------------------------------------
// particles per deposit work item (bounds the fixed-point bin sums)
#define DEP_CH 2047  // particles per deposit item (int32 bins: see gx_deposit.cu)
#define BK_ITEM 4095 // particles per work item of the fused pass (u32 bins: see gx_bucket.cu)
// striped copies of the row counters (copy = block index mod NCOPY); spreads
// the integer atomics of row-sorted particles over NCOPY addresses per row
#define NCOPY 32

// Phases of a step timed in profile mode
#define GX_NPHASE 8
enum { PH_FWD = 0, PH_CONV, PH_SYN, PH_PUSH, PH_SORT, PH_DEPOSIT, PH_COMBINE, PH_OTHER };

// Geometry constants passed by value to kernels.
struct DevGeo {
    int ndim, nr, na, ngz, nkz, ng, mmax, nsect, mesh, nrow;  // nrow = nr*ngz
    int rmap, tsoft, halo;
    float alpha, ua, inv_ua, uoffs, rinh, rgrid, zm, thmax, dzg, inv_dzg;
    float t_scale;  // na / (2 pi) in FP32
    float inv_na;   // 1 / na (fast division of cell keys, gx_div_na)
    float fna;      // na, as a float
    float eps_t, eps_z;  // guard bands of the spoke and plane coordinates (gx_cell)
    int comp;       // compensated positions: planes 2 ndim .. 3 ndim - 1 hold the low parts
    int quad;       // 27-point quadratic interpolation (p3d jmass = 3)
    float halo_v2, halo_rc2;
    float pmass;
    const int* act;  // [nact] m of each active harmonic (device, per context)
    // FP64 copies for the plain FP64 path
    double ua_d, uoffs_d, rinh_d, rgrid_d, zm_d, thmax_d, dzg_d, halo_v2_d, halo_rc2_d;
};

// Time-step zones (gx_zones.cu): zone i (1-based) steps every nstep[i-1]
// base steps and holds the particles at radius >= zbr[i-1]; code nz + 1
// marks a particle off the grid.
struct ZoneTab {
    int nz;
    int nstep[GX_MAX_ZONES];
    float zbr[GX_MAX_ZONES];
};

// Spectral bookkeeping: active harmonics (lg false, m < ng).
struct Spec {
    int nact;        // number of active harmonics
    int m[260];      // their m values, ascending
};

struct GxCtx {
    GxConfig cfg;
    GxGeometry geo;
    DevGeo g;
    Spec spec;
    std::string err;
    int dev = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    int64_t launches = 0;
    bool fp64 = false;

    // Green table (device): [4][ng][nkz][is][ir]
    float* green32 = nullptr;
    double* green64 = nullptr;
    bool have_green = false;

    // particles
    int64_t n = 0;
    int64_t cap = 0;
    float* pbuf[2] = {nullptr, nullptr};   // SoA [2*ndim][cap] (mixed path)
    int cur = 0;
    int32_t* perm = nullptr;               // processing order of pbuf[cur]
    int32_t* perm_next = nullptr;          // permutation being built by the deposit
    int32_t* origin = nullptr;             // original load index of pbuf[cur][i]
    int32_t* origin_tmp = nullptr;
    int32_t* pkey[2] = {nullptr, nullptr}; // cell key (ncl - 1, -1 off the grid) of the particles of pbuf[i]
    float* pfr = nullptr;                  // cell fractions du, dt, dz of pkey[cur], SoA [3][cap],
                                           // written by the pass that keyed them for its deposit
    bool have_keys = false;                // pkey[cur] matches pbuf[cur]
    double* p64 = nullptr;                 // SoA [2*ndim][cap] (FP64 path)
    int32_t* key64 = nullptr;
    double* w64 = nullptr;                 // [8][cap]
    double* acc64 = nullptr;               // [3][cap]
    float* ppot = nullptr;                 // per-particle potential (analysis)
    float* stagebuf = nullptr;             // [2 ndim][cap] host record staging (loadup, unload)
    float* pacc = nullptr;                 // per-particle acceleration (getacc)

    // grids
    float* mass = nullptr;                 // [mesh] scaled mass (mixed)
    int* act_d = nullptr;                  // [260] active harmonics (DevGeo::act)
    double* mass64 = nullptr;              // [mesh] (FP64 path)
    float4* field = nullptr;               // [mesh] (fx, fy, fz, pot) mixed
    float* polar = nullptr;                // [4][mesh] polar fields (fr, ft, fz, pot)
    double* field64 = nullptr;             // [4][mesh] (FP64 path: fx, fy, fz, pot)
    double* polar64 = nullptr;             // [4][mesh]
    float4* specS = nullptr;               // forward spectrum [nact][nkz][nr]
    float4* specO = nullptr;               // convolved [4][nact][nkz][nr]
    float* syntab = nullptr;               // synthesis twiddle tables (gx_synth.cu)
    float* synR = nullptr;                 // vertically synthesised rows [4][nr][ngz][ncp]
    float* fwdtab = nullptr;               // forward twiddles: azimuthal [na][ncp], vertical [ru4(2nkz)][ngz]
    float* fwdC1 = nullptr;                // azimuthal spectra of every ring-plane row [nrow][ncp]
    double* spec64 = nullptr;
    double* out64 = nullptr;
    double* az64 = nullptr;                // FP64 path: azimuthal spectra [2][nr*ngz*nact]
    double* rows64 = nullptr;              // FP64 path: vertically synthesised rows [4][...]
    double* pot64 = nullptr;               // FP64 path: per-particle potential [cap]
    bool have_mass = false;
    bool have_field = false;
    bool field_pot = false;
    int jrs = 1, krs = 0;                  // active source ring range (1-based)

    // deposit
    int32_t* rowstart = nullptr;           // [nrow + 1]
    int32_t* items = nullptr;              // work items [maxitems][3]: row, start, end
    int32_t* nitems_d = nullptr;
    int32_t* rowitem = nullptr;            // [nrow + 1] first work item of each row
    int32_t* stage = nullptr;              // [maxitems][NQ][na] fixed-point rows
    uint32_t* rowcnt = nullptr;            // [NCOPY][nrow + 1] particles per row (zeroed after use)
    uint32_t* rowfill = nullptr;           // [NCOPY][nrow + 1] slots handed out per row
    uint32_t* rowbase = nullptr;           // [NCOPY][nrow + 1] offset of each copy in its row
    uint32_t* rowtot = nullptr;            // [nrow + 1] particles per row
    int32_t* rowtile = nullptr;            // [tiles of ROW_TILE rows][4]: particles, items, first and last occupied row
    int maxitems = 0;
    int32_t* jrk_d = nullptr;              // device min/max ring
    int32_t* errword = nullptr;            // device error word

    // diagnostics scratch
    double* dsum = nullptr;

    // phase timing (gx_set_profile): an event at every phase mark, recorded
    // without waiting, read back at gx_phase_end (so the kernels still run
    // back to back and a phase's time holds no host launch gap)
    bool prof = false;
    std::vector<cudaEvent_t> pev;          // event pool
    std::vector<int> pev_ph;               // phase opened by each recorded mark (-1: end)
    int nmarks = 0;
    float phase_ms[GX_NPHASE] = {};
    int64_t phase_n[GX_NPHASE] = {};

    // time-step zones (gx_zones.cu); nzones = 1 is the single-zone step
    int nzones = 1;
    ZoneTab zt = {};
    int32_t* pzone[2] = {nullptr, nullptr};  // zone code of the particles of pbuf[i]
    float* zbuf = nullptr;                   // [2][nzones][mesh] mass arrays of zones 2..nzones
    float* znew[GX_MAX_ZONES] = {};          // newest array of each zone (index >= 1)
    float* zold[GX_MAX_ZONES] = {};          // the one before it
    int32_t* zjrk_d = nullptr;               // [GX_MAX_ZONES][2] ring range of each zone's mass,
                                             // then [2] the field rings of the next partial solve
    int istep = 0;                           // step counter of the zone schedule
    int lstep[GX_MAX_ZONES][2] = {};         // step numbers of zold, znew
    bool zones_ready = false;                // zone arrays deposited (gx_masset)

    // bucketed particle store of the fused step (gx_bucket.cu): bq[b] holds
    // one segment of slots per ring-plane row (row nrow: off the grid),
    // [bk_base[b][r], + bk_cap[b][r]), of which the first
    // min(bk_fill[b][r], bk_cap[b][r]) are particles, then an overflow area
    // of bk_ctl[b][0] particles from slot bk_main on
    bool bucketed = false;
    float4* bq[2] = {nullptr, nullptr};       // records of R float4 words, R planes of bcap each
    int64_t bcap = 0;                         // records per plane: bk_main + an overflow area of n
    int bcur = 0;                             // the bucketed store's current buffer
    int64_t bk_main = 0;
    int32_t* bk_cap[2] = {nullptr, nullptr};
    int32_t* bk_base[2] = {nullptr, nullptr};
    int32_t* bk_fill[2] = {nullptr, nullptr};
    int32_t* bk_ctl = nullptr;               // [2][4]: overflow count of each buffer; [8] items, [9] work
                                             // counter, [10..11] plane range, [12] compaction counter,
                                             // [13..14] ring range (of the pass's new cells)
    int4* bk_items = nullptr;                // work items of pbuf[cur]: row (-1: overflow), first, end slot
    int64_t bk_maxitems = 0;
    int bk_item = BK_ITEM;                   // particles per work item of the fused pass
    int32_t* bk_cnt = nullptr;               // [nrow + 1] row counts of the dense store (bucketing)
    unsigned long long* macc = nullptr;      // [mesh] fixed-point mass (2^-20 of a particle), zero between steps
    int32_t* zr_d = nullptr;                 // [2] first, last plane holding the fused pass's mass
                                             // (ngz, -1 when empty)
    bool zr_valid = false;                   // the mass array is the fused pass's (zr_d describes it)
    int bk_grid = 0;                         // CTAs of the fused pass
    cudaStream_t bk_side = nullptr;          // the plan's stream (overlaps the field solve)
    cudaEvent_t bk_ev[2] = {nullptr, nullptr};  // push done (main), plan done (side)
    bool bk_pending = false;                 // a plan on bk_side the main stream has not joined

    // multi-GPU (gx_comm.cu): NCCL communicator of the particle decomposition
    void* comm = nullptr;
    int nranks = 1, rank = 0;
    gx_host_reduce_fn host_fn = nullptr;     // exchanges through the host (gx_comm_host)
    void* host_user = nullptr;
    std::vector<char> host_buf;
};

// record the start of phase ph (prof mode) and close the previous one
int gx_phase_mark(GxCtx* c, int ph);
int gx_phase_end(GxCtx* c);

// ---------------------------------------------------------------------------
// error helpers (host)
#define GX_CUDA(ctx, call)                                                  \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) {                                            \
            (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e_);\
            return GX_ERR_CUDA;                                             \
        }                                                                   \
    } while (0)

#define GX_LAUNCHED(ctx)                                                    \
    do {                                                                    \
        (ctx)->launches++;                                                  \
        cudaError_t e_ = cudaGetLastError();                                \
        if (e_ != cudaSuccess) {                                            \
            (ctx)->err = std::string("launch: ") + cudaGetErrorString(e_);  \
            return GX_ERR_CUDA;                                             \
        }                                                                   \
    } while (0)

// ---------------------------------------------------------------------------
// cell-key arithmetic (device).  The reference (SRC/lib15/weight.f:61-101,
// 196-250) forms r = sqrt(x*x + y*y) in FP32, u = uofgr(r) in FP32, the
// spoke coordinate t from an FP64 atan2 rounded to FP32, z = (z + zm)/dzg in
// FP32, and truncates.  The fast path below evaluates u and t with FP32
// library functions; when either lies within a guard band of an integer
// boundary it is recomputed with the reference's exact operation sequence
// (correctly rounded log, FP64 atan2), so the integer cell indices agree
// with the reference's wherever its own libm calls are correctly rounded.

// ND = 2 or 3 fixes the dimension at compile time (the particle pass is
// instantiated per dimension, so that its corner loop unrolls and its
// eight gathers are issued together); ND = 0 reads it from the geometry
template <int ND>
__device__ __forceinline__ bool gx_is3(const DevGeo& g) {
    return ND == 0 ? g.ndim == 3 : ND == 3;
}

struct CellW {
    int key;      // ncl - 1, or -1 when off the grid / in the hole
    float du, dt, dz;  // fractions in the cell; quadratic: coord + 1/2 - index
    int row, jt;  // ring-plane row and spoke of key (set by gx_cell)
    int ju, iz;   // ring and plane of row (linear scheme; row = ju * ngz + iz)
};

// floor of a float in [0, 2^23) and the exact fraction v - floor(v), on the
// FMA and integer pipes: v + 2^23 rounded toward zero holds floor(v) in its
// low mantissa bits (negative v count as 0: the fraction is then v itself,
// as v - (int)v gives for the reference's truncation of -0 < v < 0)
__device__ __forceinline__ int gx_trunc(float v, float& frac) {
    const float t = __fadd_rz(fmaxf(v, 0.f), 8388608.0f);
    frac = v - (t - 8388608.0f);
    return __float_as_int(t) - 0x4B000000;
}

// (float)i for 0 <= i < 2^23, exact, without a conversion instruction
__device__ __forceinline__ float gx_i2f(int i) {
    return __int_as_float(0x4B000000 | i) - 8388608.0f;
}

__device__ __forceinline__ float gx_u_exact(const DevGeo& g, float rr) {
    if (g.rmap == GX_RMAP_STDPOL) {
        float v = __fadd_rn(1.0f, rr);
        float lf = (float)log((double)v);
        return __fdiv_rn(lf, g.ua);
    }
    float lf = (float)log((double)rr);
    return __fadd_rn(__fdiv_rn(lf, g.ua), g.uoffs);
}

__device__ __forceinline__ float gx_t_exact(const DevGeo& g, float x, float y) {
    double t = atan2((double)y, (double)x) * (double)g.na / (2.0 * GX_PI);
    float tf = (float)t;
    if (tf < 0.f) tf = __fadd_rn(tf, (float)g.na);
    return tf;
}

// atan2 for the fast cell estimate: octant reduction to q = min/max in
// [0, 1], atan(q) = q P(q^2) with an 8-term odd minimax polynomial (own
// Remez-exchange fit on [0, 1], 3.7e-8 absolute), then atan(y/x) =
// pi/2 - atan(x/y) above the diagonal and the quadrant from the signs.
// Absolute error about 4e-7 over the plane in FP32 (the final rounding near
// pi and the approximate reciprocal dominate), the same class as the
// library atan2f; gx_cell's guard band (4e-6 (na + 1) spokes, 2.5e-5 rad)
// covers it with a margin of 60.
__device__ __forceinline__ float gx_atan2_fast(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    float rc;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rc) : "f"(fmaxf(mx, 1e-30f)));
    const float q = mn * rc;
    const float s = q * q;
    float p = -4.054567311e-03f;
    p = fmaf(p, s, 2.186295763e-02f);
    p = fmaf(p, s, -5.591232702e-02f);
    p = fmaf(p, s, 9.642197192e-02f);
    p = fmaf(p, s, -1.390862912e-01f);
    p = fmaf(p, s, 1.994656622e-01f);
    p = fmaf(p, s, -3.332985938e-01f);
    p = fmaf(p, s, 9.999993443e-01f);
    p *= q;
    float r = (ay > ax) ? 1.570796327f - p : p;
    r = (x < 0.f) ? 3.141592654f - r : r;
    return (y < 0.f) ? -r : r;
}

__device__ __forceinline__ bool gx_near_int(float v, float eps) {
    float f;
    gx_trunc(v, f);
    return (f < eps) || (f > 1.f - eps);
}

// quadratic (27-point) cell of p3d, jmass = 3 (weight.f:280-298): the
// nearest node (ju, jz, jt) = int(coord + 1/2), ju in [1, nr - 2], jz in
// [0, ngz - 2], jt = na wrapping to spoke 0 in the key; the fractions are
// coord + 1/2 - index (outside [0, 1) where an index was clamped)
template <bool EXACT = true>
__device__ __forceinline__ CellW gx_cell27(const DevGeo& g, float u, float t, float z, CellW c) {
    const float uh = __fadd_rn(u, 0.5f), th = __fadd_rn(t, 0.5f);
    float f;
    int ju = gx_trunc(uh, f);
    ju = min(max(ju, 1), g.nr - 2);
    const int jt = gx_trunc(th, c.dt);
    float zz = (z + g.zm) * g.inv_dzg;
    if (EXACT && gx_near_int(zz + 0.5f, g.eps_z)) zz = __fdiv_rn(__fadd_rn(z, g.zm), g.dzg);
    const float zh = __fadd_rn(zz, 0.5f);
    int jz = gx_trunc(zh, f);
    jz = min(max(jz, 0), g.ngz - 2);
    c.du = uh - gx_i2f(ju);
    c.dz = zh - gx_i2f(jz);
    c.row = ju * g.ngz + jz;
    c.jt = (jt == g.na) ? 0 : jt;
    c.key = c.row * g.na + c.jt;
    return c;
}

// Cell of a particle; old != 0 for interpolation (no sector folding).
// EXACT = false drops the guard bands: the cell may then differ from the
// reference's for a coordinate within a few ulp of a cell boundary, where
// the interpolated field is continuous (the particle pass's interpolation
// cell); keys that are deposited or reported use the exact form.
template <bool EXACT, int ND = 0>
__device__ __forceinline__ CellW gx_cell_t(const DevGeo& g, float x, float y, float z, bool old) {
    CellW c;
    c.key = -1;
    c.du = c.dt = c.dz = 0.f;
    c.row = c.jt = 0;
    c.ju = c.iz = 0;
    const float r2 = __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y));
    float rr;
    if (EXACT) {
        rr = __fsqrt_rn(r2);
    } else {
        // the interpolation cell needs no correctly rounded radius
        asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(rr) : "f"(r2));
    }
    if (rr > g.rgrid) return c;
    if (gx_is3<ND>(g) && fabsf(z) > g.zm) return c;
    if (rr < g.rinh) return c;
    // u (fast path + guard)
    float u;
    if (g.rmap == GX_RMAP_STDPOL) u = __logf(1.0f + rr) * g.inv_ua;
    else u = __logf(rr) * g.inv_ua + g.uoffs;
    // the quadratic scheme truncates coord + 1/2: its boundaries sit at half-integers
    const float sh = g.quad ? 0.5f : 0.f;
    if (EXACT) {
        // __logf: 2^-21.41 absolute error on [0.5, 2], 3 ulp elsewhere
        float eps = 5.0e-7f * g.inv_ua + 2.0e-6f * (fabsf(u) + fabsf(g.uoffs) + 1.0f);
        if (gx_near_int(u + sh, eps) || u < eps) u = gx_u_exact(g, rr);
    }
    // t
    float t;
    if (!gx_is3<ND>(g) || rr > 0.f) {
        t = gx_atan2_fast(y, x) * g.t_scale;
        if (t < 0.f) t += g.fna;
        const float eps = g.eps_t;
        if (EXACT && (gx_near_int(t + sh, eps) || t < eps || t > g.fna - eps)) t = gx_t_exact(g, x, y);
    } else {
        t = 0.f;
    }
    if (!old && g.nsect > 1) t = fmodf(t, g.thmax);
    if (g.quad) return gx_cell27<EXACT>(g, u, t, z, c);
    int ju = gx_trunc(u, c.du);
    if (ju > g.nr - 2) {
        ju = g.nr - 2;
        c.du = u - gx_i2f(ju);
    }
    const int jt = gx_trunc(t, c.dt);
    c.ju = ju;
    if (!gx_is3<ND>(g)) {
        c.row = ju;
    } else {
        float zz = (z + g.zm) * g.inv_dzg;
        if (EXACT && gx_near_int(zz, g.eps_z)) zz = __fdiv_rn(__fadd_rn(z, g.zm), g.dzg);
        int jz = gx_trunc(zz, c.dz);
        if (jz > g.ngz - 2) {
            jz = g.ngz - 2;
            c.dz = zz - gx_i2f(jz);
        }
        c.row = ju * g.ngz + jz;
        c.iz = jz;
    }
    c.key = c.row * g.na + jt;
    // a spoke coordinate that rounded up to na keys the next row's spoke 0,
    // as the reference's flat cell number does; row and jt follow the key
    c.jt = jt;
    if (jt >= g.na) {
        c.jt = jt - g.na;
        c.row += 1;
        if (!gx_is3<ND>(g)) {
            c.ju += 1;
        } else if (++c.iz == g.ngz) {
            c.iz = 0;
            c.ju += 1;
        }
    }
    return c;
}

__device__ __forceinline__ CellW gx_cell(const DevGeo& g, float x, float y, float z, bool old) {
    return gx_cell_t<true>(g, x, y, z, old);
}

// x + v with the rounding error of the sum carried in a low part (the
// compensated drift): Knuth's two-sum of hi and v, then the error folded
// into lo and (hi, lo) renormalised so that |lo| <= ulp(hi) / 2
__device__ __forceinline__ void gx_comp_add(float& hi, float& lo, float v) {
    const float s = __fadd_rn(hi, v);
    const float bp = __fsub_rn(s, hi);
    const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(v, bp));
    const float l = __fadd_rn(lo, err);
    const float t = __fadd_rn(s, l);
    lo = __fsub_rn(l, __fsub_rn(t, s));
    hi = t;
}

// 8 (3D) or 4 (2D) weights in the reference order (weight.f:92-99, 241-248)
template <int ND = 0>
__device__ __forceinline__ void gx_weights(const DevGeo& g, const CellW& c, float* w) {
    if (!gx_is3<ND>(g)) {
        float dd = c.du * c.dt;
        w[0] = 1.f - c.du - c.dt + dd;
        w[1] = c.dt - dd;
        w[2] = c.du - dd;
        w[3] = dd;
    } else {
        float a0 = (1.f - c.dt) * (1.f - c.dz), a1 = c.dt * (1.f - c.dz);
        float a2 = (1.f - c.dt) * c.dz, a3 = c.dt * c.dz;
        float bu = 1.f - c.du;
        w[0] = a0 * bu;
        w[1] = a1 * bu;
        w[2] = a2 * bu;
        w[3] = a3 * bu;
        w[4] = a0 * c.du;
        w[5] = a1 * c.du;
        w[6] = a2 * c.du;
        w[7] = a3 * c.du;
    }
}

// q = v / na and r = v % na for 0 <= v < 2^24 (every cell key: the mesh is
// checked against 2^24 at set-up): the float reciprocal is off by at most
// one, fixed by one correction
__device__ __forceinline__ int gx_div_na(const DevGeo& g, int v, int& r) {
    int q = __float2int_rz((float)v * g.inv_na);
    r = v - q * g.na;
    if (r < 0) {
        q--;
        r += g.na;
    } else if (r >= g.na) {
        q++;
        r -= g.na;
    }
    return q;
}

// corner cells of a key (grdacc.f:193-202); -1 for cells past the mesh end
// 27 quadratic weights (weight.f:299-311): per axis (1 - 2dd + dd^2,
// 1 + 2dd - 2dd^2, dd^2); weight l = 9 k + 3 j + i (theta i fastest, then z
// j, then u k) = 1/8 f_theta(i) f_z(j) f_u(k)
__device__ __forceinline__ void gx_weights27(const CellW& c, float* w) {
    float f[3][3];
    const float d[3] = {c.dt, c.dz, c.du};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float dd = d[a], d2 = dd * dd;
        f[a][0] = (1.f - 2.f * dd) + d2;
        f[a][1] = (1.f + 2.f * dd) - 2.f * d2;
        f[a][2] = d2;
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int j = 0; j < 3; j++)
#pragma unroll
            for (int i = 0; i < 3; i++) w[9 * k + 3 * j + i] = 0.125f * f[0][i] * f[1][j] * f[2][k];
}

// the 27 nodes of a quadratic cell in weight order (massgn.f:180-193,
// grdacc.f:271-283): theta wraps, planes and rings are flat offsets of
// na and ngz na; nodes outside the mesh are -1
__device__ __forceinline__ void gx_corners27(const DevGeo& g, int row, int r, int* ic) {
    const int na = g.na, pl = g.ngz * na;
    const int base = row * na, key = base + r;
    const int mid[3] = {base + ((r == 0) ? na - 1 : r - 1), key, base + ((r == na - 1) ? 0 : r + 1)};
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int j = 0; j < 3; j++)
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const int v = mid[i] + (j - 1) * na + (k - 1) * pl;
                ic[9 * k + 3 * j + i] = (v < 0 || v >= g.mesh) ? -1 : v;
            }
}

template <int ND = 0>
__device__ __forceinline__ int gx_corners_rt(const DevGeo& g, int key, int jt, int* ic) {
    const int na = g.na;
    const int end = (jt == na - 1);
    ic[0] = key;
    ic[1] = key + 1 - (end ? na : 0);
    ic[2] = key + na;
    ic[3] = ic[1] + na;
    if (!gx_is3<ND>(g)) {
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (ic[k] >= g.mesh) ic[k] = -1;
        return 4;
    }
    const int pl = g.ngz * na;
    ic[4] = key + pl;
    ic[5] = ic[1] + pl;
    ic[6] = ic[4] + na;
    ic[7] = ic[5] + na;
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (ic[k] >= g.mesh) ic[k] = -1;
    return 8;
}

// the same from a key alone
__device__ __forceinline__ int gx_corners(const DevGeo& g, int key, int* ic) {
    int jt;
    gx_div_na(g, key, jt);
    return gx_corners_rt(g, key, jt, ic);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

#define ROW_TILE 256  // rows per block of the row reduce / scan

// warp-aggregated count of row (all 32 lanes must call)
__device__ __forceinline__ void gx_row_count(uint32_t row, bool act, uint32_t* __restrict__ cnt) {
    const uint32_t am = __ballot_sync(0xffffffffu, act);
    const uint32_t peers = __match_any_sync(0xffffffffu, act ? row : 0xffffffffu) & am;
    if (act && (peers & lanemask_lt()) == 0) atomicAdd(&cnt[row], (uint32_t)__popc(peers));
}

// fixed axisymmetric force of a softened Kuz'min-Toomre disc, applied to
// every particle on the grid when the m = 0 harmonic is filtered out
// (filset.f:3-5, getacc.f:118-121, axifrc.f, frdisc.f:27-29 'SOFT'):
// F(r) = -K r / (r^2 + Rs^2)^1.5 with K = halo_v2 (the disc mass in
// internal units, M lscale^3 ts^2) and Rs = halo_rc (grid units,
// (1 + epsilon) rscale lscale, inimod.f:74); potential -K / sqrt(r^2 + Rs^2)
// (phidsc.f:38).  Spherical radius in 3D, as getacc measures it.
__device__ __forceinline__ void gx_disc_force(const DevGeo& g, float x, float y, float z, float& ax,
                                              float& ay, float& az, float& ph) {
    const float r2 = x * x + y * y + ((g.ndim == 3) ? z * z : 0.f);
    const float d = r2 + g.halo_rc2;
    const float sd = sqrtf(d);
    const float f = -g.halo_v2 / (d * sd);
    ax += f * x;
    ay += f * y;
    if (g.ndim == 3) az += f * z;
    ph -= g.halo_v2 / sd;
}

// interpolated acceleration and potential of a particle at (x, y, z) whose
// interpolation cell is cw: grdacc + halfrc (or the fixed disc force)
template <bool Q, int ND = 0>
__device__ __forceinline__ void gx_accel_cell_t(const DevGeo& g, const float4* __restrict__ F,
                                                const CellW& cw, float x, float y, float z,
                                                float& ax, float& ay, float& az, float& ph) {
    ax = ay = az = ph = 0.f;
    // particles off the grid feel no force (getacc.f:103-122 acts on the
    // particles inside the grid)
    if (cw.key < 0) return;
    if constexpr (Q) {
        // grdacc.f:267-299
        float w[27];
        int ic[27];
        gx_weights27(cw, w);
        gx_corners27(g, cw.row, cw.jt, ic);
#pragma unroll
        for (int k = 0; k < 27; k++) {
            if (ic[k] < 0) continue;
            const float4 f = __ldg(F + ic[k]);
            ax += f.x * w[k];
            ay += f.y * w[k];
            az += f.z * w[k];
            ph += f.w * w[k];
        }
    } else if constexpr (ND != 0) {
        constexpr int NC = (ND == 3) ? 8 : 4;
        float w[8];
        int ic[8];
        gx_weights<ND>(g, cw, w);
        gx_corners_rt<ND>(g, cw.key, cw.jt, ic);
        float4 f[NC];
#pragma unroll
        for (int k = 0; k < NC; k++) f[k] = (ic[k] >= 0) ? __ldg(F + ic[k]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < NC; k++) {
            ax += f[k].x * w[k];
            ay += f[k].y * w[k];
            az += f[k].z * w[k];
            ph += f[k].w * w[k];
        }
    } else {
        float w[8];
        int ic[8];
        gx_weights(g, cw, w);
        const int nc = gx_corners_rt(g, cw.key, cw.jt, ic);
        for (int k = 0; k < nc; k++) {
            if (ic[k] < 0) continue;
            const float4 f = __ldg(F + ic[k]);
            ax += f.x * w[k];
            ay += f.y * w[k];
            az += f.z * w[k];
            ph += f.w * w[k];
        }
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
    } else if (g.halo == 2) {
        gx_disc_force(g, x, y, z, ax, ay, az, ph);
    }
}

__device__ __forceinline__ void gx_accel_cell(const DevGeo& g, const float4* __restrict__ F,
                                              const CellW& cw, float x, float y, float z, float& ax,
                                              float& ay, float& az, float& ph) {
    if (g.quad) gx_accel_cell_t<true>(g, F, cw, x, y, z, ax, ay, az, ph);
    else gx_accel_cell_t<false>(g, F, cw, x, y, z, ax, ay, az, ph);
}

// ---------------------------------------------------------------------------
// host-side entry points implemented in the .cu files
int setgrd(const GxConfig* c, GxGeometry* g, std::string& err);
void fill_devgeo(GxCtx* c);
int gx_green_build_dev(GxCtx* c);
int gx_mixed_masset(GxCtx* c);
// frk: device [2] 1-based field ring range of a partial-grid solve, or null
// zr: device [2] first and last plane holding mass (the step's own solve:
// the forward transforms skip the planes outside, the azimuthal synthesis
// covers them one plane wider, the planes the next particle pass reads), or
// null for the whole grid
int gx_mixed_findf(GxCtx* c, int lpot, bool polcat, const int32_t* frk = nullptr,
                   const int32_t* zr = nullptr);
int gx_mixed_getacc(GxCtx* c, float* acc, float* pot);
int gx_mixed_step(GxCtx* c, int nsteps, int phys);
int gx_mixed_sort_deposit(GxCtx* c);
int gx_mixed_keys_initial(GxCtx* c);
int gx_fp64_masset(GxCtx* c);
int gx_fp64_findf(GxCtx* c, int lpot, bool polcat);
int gx_fp64_getacc(GxCtx* c, float* acc, float* pot);
int gx_fp64_step(GxCtx* c, int nsteps, int phys);
// rows counted by the caller's pass -> permutation, deposit (from the
// keys and fractions the pass stored), mass.  With
// zone set, only particles whose zone code is zsel are deposited (the
// counting pass filtered the same way); the mass goes to mass_out
// (default c->mass), scaled by pm (default pmass).
int gx_deposit_rows(GxCtx* c, const int32_t* keys, const float* fr, int32_t* perm_out,
                    const int32_t* zone = nullptr, int zsel = 0, float* mass_out = nullptr,
                    float pm = -1.f);
int gx_zone_loadup(GxCtx* c);
int gx_zone_unload(GxCtx* c, float* staging);
int gx_zone_masset(GxCtx* c);
int gx_zone_step(GxCtx* c, int nsteps, int phys);
int gx_comm_reduce_range(GxCtx* c);
// fused step on the bucketed store (gx_bucket.cu)
bool gx_fast_ok(const GxCtx* c);  // single zone, linear scheme, mixed, not GX_FLAG_SORTED_DEPOSIT
int gx_fast_step(GxCtx* c, int nsteps, int phys);
int gx_dense(GxCtx* c);  // bucketed store -> dense store (no-op when dense)
int gx_bucket_unload(GxCtx* c, float* aos);  // unload from the bucketed store
int gx_fast_masset(GxCtx* c);  // masset by the deposit-only fused pass
int gx_bucket_alloc(GxCtx* c);
int gx_bucket_words(const GxCtx* c);  // float4 words per record of the bucketed store
int gx_synthesis(GxCtx* c, int tmask, float* polar, const int32_t* frk = nullptr,
                 const int32_t* zr = nullptr);
int gx_comm_reduce_spectrum(GxCtx* c);
int gx_comm_reduce_conv(GxCtx* c);    // sum of the contracted spectra (plane split)
int gx_comm_reduce_planes(GxCtx* c, int32_t* zr);  // MIN/MAX of the plane range of the mass
bool gx_plane_split(const GxCtx* c);
void gx_comm_destroy(GxCtx* c);
