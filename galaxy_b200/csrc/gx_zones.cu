// gx_zones.cu -- multiple time-step zones of the mixed path.
//
// The reference steps the particles of zone i (radius >= zbr(i)) every
// nstep(i) base steps with a step nstep(i) times longer, keeping velocities
// in units of each zone's own step:
//
//   zoneno.f, tsfac.f      zone of a position, its step factor
//   loadup.f:177-181, adjvls.f   zones at load time, velocity scaling
//   step.f:135-292         mzone = the largest i with istep mod nstep(i) = 0;
//                          zones 1..mzone move, the off-grid list moves with
//                          the outermost zone (mzone = nzones)
//   getacc.f:141-150       accelerations x tsfac^2
//   stpgrp.f:26-57, addoff.f:44-52   leaving the grid: the outermost zone's
//                          step; returning: zone nzones
//   rezgrp.f, chstep.f     zone changes after the step redo the step from
//                          the old coordinates with the new step
//   masscl.f:31-96         each zone keeps the mass array of its newest and
//                          its previous positions, with their step numbers
//   zoncmb.f:46-129, scaled.f:89-92   the solve's mass: zone 1's array plus
//                          the linear interpolation in time of the others,
//                          times pmass
//   p2fndf.f:25-33         the source ring range over all zones
//
// Here the particle pass of a step (k_push_zone) moves the particles of the
// active zones in one launch and copies the others through; the deposit
// runs once per active zone through the deterministic counting-sort
// deposit (gx_deposit.cu) filtered by zone code, into that zone's array;
// k_zone_combine forms the solve's mass.  The solve always covers the
// whole grid (findf.f:41-54 allows the reference a partial grid when only
// inner zones move; the forces at the moving particles are the same).
#include <algorithm>

#include "gx_common.cuh"

__device__ __forceinline__ int zt_zoneno(const ZoneTab& zt, int nd, float x, float y, float z) {
    float r2 = x * x + y * y;
    if (nd == 3) r2 += z * z;  // spherical boundaries in 3D (setrun.f:810)
    const float rad = sqrtf(r2);
    int k = 1;
    for (int i = 1; i < zt.nz; i++)
        if (rad >= zt.zbr[i]) k = i + 1;
    return k;
}

__device__ __forceinline__ float zt_tsfac(const ZoneTab& zt, int iz) {
    return (float)zt.nstep[min(iz, zt.nz) - 1];
}

// chstep (RVLF): redo the step from the old coordinates with the step
// changed by tfac; a is the step's acceleration, updated to the new step
__device__ __forceinline__ void zt_chstep(int nd, const float* qo, float* q, float* a,
                                          float tfac) {
    for (int i = 0; i < nd; i++) {
        const float vo = tfac * (qo[nd + i] + 0.5f * a[i] * (1.f - tfac));
        a[i] = a[i] * tfac * tfac;
        q[nd + i] = vo + a[i];
        q[i] = qo[i] + q[nd + i];
    }
}

// loadup: zone of every particle, velocities in units of its zone's step
__global__ void k_zone_setup(DevGeo g, ZoneTab zt, float* __restrict__ P, int64_t cap, int64_t n,
                             int32_t* __restrict__ zone) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nd = g.ndim;
    const float x = P[i], y = P[cap + i], z = (nd == 3) ? P[2 * cap + i] : 0.f;
    const CellW cw = gx_cell(g, x, y, z, true);
    if (cw.key < 0) {
        zone[i] = zt.nz + 1;
        return;
    }
    const int iz = zt_zoneno(zt, nd, x, y, z);
    zone[i] = iz;
    const float t = zt_tsfac(zt, iz);
    for (int d = 0; d < nd; d++) P[(nd + d) * cap + i] *= t;
}

// unload: records (AoS, load order) back to base-step velocities
__global__ void k_zone_unscale_aos(ZoneTab zt, int nd, float* __restrict__ aos,
                                   const int32_t* __restrict__ zone,
                                   const int32_t* __restrict__ origin, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int iz = zone[i];
    if (iz > zt.nz) return;
    const float r = 1.f / zt_tsfac(zt, iz);
    float* q = aos + (int64_t)origin[i] * 2 * nd;
    for (int d = 0; d < nd; d++) q[nd + d] *= r;
}

// zone codes in load order
__global__ void k_zone_gather(const int32_t* __restrict__ zone, const int32_t* __restrict__ origin,
                              int64_t n, int32_t* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[origin[i]] = zone[i];
}

// cell keys and fractions of the stored particles (masset)
__global__ void k_zone_keys(DevGeo g, const float* __restrict__ P, int64_t cap, int64_t n,
                            int32_t* __restrict__ keys, float* __restrict__ fr) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float z = (g.ndim == 3) ? P[2 * cap + i] : 0.f;
    const CellW cw = gx_cell(g, P[i], P[cap + i], z, false);
    keys[i] = cw.key;
    fr[i] = cw.du;
    fr[cap + i] = cw.dt;
    if (g.ndim == 3) fr[2 * cap + i] = cw.dz;
}

// rows of the particles of zone zsel for the deposit's counting sort (the
// others count in the off-grid row); same block geometry as k_place
__global__ void k_zone_rows(DevGeo g, const int32_t* __restrict__ keys,
                            const int32_t* __restrict__ zone, int64_t n, int zsel,
                            uint32_t* __restrict__ rowcnt) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool act = t < n;
    uint32_t row = (uint32_t)g.nrow;
    if (act) {
        const int32_t key = keys[t];
        int r;
        if (key >= 0 && zone[t] == zsel) row = (uint32_t)gx_div_na(g, key, r);
    }
    gx_row_count(row, act, rowcnt + (size_t)(blockIdx.x & (NCOPY - 1)) * (g.nrow + 1));
}

// the particle pass of a zoned step: the particles of zones 1..mzone (and,
// when mzone = nz, those off the grid) move; the others are copied through
__global__ void __launch_bounds__(256) k_push_zone(
    DevGeo g, ZoneTab zt, int mzone, const float* __restrict__ Pin, float* __restrict__ Pout,
    int64_t cap, int64_t n, const int32_t* __restrict__ perm, const int32_t* __restrict__ orig_in,
    int32_t* __restrict__ orig_out, const float4* __restrict__ F, const int32_t* __restrict__ key_in,
    int32_t* __restrict__ key_out, float* __restrict__ fr_out, const int32_t* __restrict__ zone_in,
    int32_t* __restrict__ zone_out, float* __restrict__ pot) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = perm[s];
    const int nd = g.ndim, nw = 2 * nd, nz = zt.nz, off = nz + 1;
    float q[6], qo[6];
    for (int k = 0; k < nw; k++) q[k] = qo[k] = Pin[k * cap + p];
    const float z = (nd == 3) ? q[2] : 0.f;
    const int z0 = zone_in[p];
    orig_out[s] = orig_in[p];
    const bool moves = z0 <= mzone || (z0 == off && mzone == nz);
    float a[3] = {0.f, 0.f, 0.f}, ph = 0.f;
    if (z0 != off && (moves || pot)) {
        const CellW cw = gx_cell(g, q[0], q[1], z, true);
        gx_accel_cell(g, F, cw, q[0], q[1], z, a[0], a[1], a[2], ph);
    }
    if (pot) pot[s] = ph;
    if (!moves) {
        for (int k = 0; k < nw; k++) Pout[k * cap + s] = q[k];
        key_out[s] = key_in[p];
        zone_out[s] = z0;
        return;
    }
    if (z0 > 1) {
        const float t = zt_tsfac(zt, z0);
        for (int d = 0; d < nd; d++) a[d] *= t * t;
    }
    for (int d = 0; d < nd; d++) {
        q[nd + d] += a[d];
        q[d] += q[nd + d];
    }
    CellW cn = gx_cell(g, q[0], q[1], (nd == 3) ? q[2] : 0.f, false);
    int iz = z0;
    if (z0 != off) {
        if (cn.key < 0) {
            iz = off;
            if (z0 < nz) {
                zt_chstep(nd, qo, q, a, zt_tsfac(zt, nz) / zt_tsfac(zt, z0));
                cn = gx_cell(g, q[0], q[1], (nd == 3) ? q[2] : 0.f, false);
            }
        }
    } else if (cn.key >= 0) {
        iz = nz;
    }
    if (z0 != off && mzone > 1 && iz <= mzone) {
        int kz = min(zt_zoneno(zt, nd, q[0], q[1], (nd == 3) ? q[2] : 0.f), mzone);
        if (kz > iz) kz = zt_zoneno(zt, nd, qo[0], qo[1], (nd == 3) ? qo[2] : 0.f);
        if (kz != iz) {
            zt_chstep(nd, qo, q, a, zt_tsfac(zt, kz) / zt_tsfac(zt, iz));
            iz = kz;
            cn = gx_cell(g, q[0], q[1], (nd == 3) ? q[2] : 0.f, false);
        }
    }
    for (int k = 0; k < nw; k++) Pout[k * cap + s] = q[k];
    // fractions for this step's deposit, which takes only particles that moved
    key_out[s] = cn.key;
    fr_out[s] = cn.du;
    fr_out[cap + s] = cn.dt;
    if (nd == 3) fr_out[2 * cap + s] = cn.dz;
    zone_out[s] = iz;
}

// the arrays added into zone 1's array and their time fractions
struct ZoneSrc {
    const float* p[2 * GX_MAX_ZONES];
    float fr[2 * GX_MAX_ZONES];
    int n;
};

// zoncmb + scaled: mass = (mass + sum fr_k src_k) pmass, in the reference's
// order; block 0 also forms the source ring range over the zones and the
// field rings of a partial-grid solve in which zones 1..mz move
__global__ void k_zone_combine(int64_t mesh, float* __restrict__ mass, ZoneSrc src, float pm,
                               int nz, int nr, int mz, int32_t* __restrict__ zjrk,
                               int32_t* __restrict__ jrk) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < mesh) {
        float v = mass[i];
        for (int k = 0; k < src.n; k++) v = __fadd_rn(v, __fmul_rn(src.fr[k], src.p[k][i]));
        mass[i] = v * pm;
    }
    if (i == 0) {
        int jrs = nr, krs = 0;
        for (int k = 0; k < nz; k++) {
            jrs = min(jrs, zjrk[2 * k]);
            krs = max(krs, zjrk[2 * k + 1]);
            if (k > 0 && krs > zjrk[2 * k + 1]) zjrk[2 * k + 1] = krs;
        }
        jrk[0] = jrs;
        jrk[1] = krs;
        // p3fndf.f:66-80, p2fndf.f:41-55: from jrad(1) to krad(mz), the
        // outer edge moved out while it lies inside jrad(1)
        int jrf = zjrk[0] < nr ? zjrk[0] : 1;
        int kz = mz - 1, krf = zjrk[2 * kz + 1];
        while (krf < jrf && kz + 1 < nz) krf = zjrk[2 * (++kz) + 1];
        int32_t* frk = zjrk + 2 * GX_MAX_ZONES;
        frk[0] = krf < jrf ? 1 : jrf;
        frk[1] = krf < jrf ? nr : min(krf, nr);
    }
}

// ---------------------------------------------------------------------------
static int zone_mzone(const GxCtx* c, int istep) {
    int m = 1;
    for (int i = 0; i < c->nzones; i++)
        if (istep % c->zt.nstep[i] == 0) m = i + 1;
    return m;
}

// masscl: the step numbers of the arrays about to be deposited; the newest
// arrays of zones 2..mzone become the previous ones
static void zone_masscl(GxCtx* c, int mzone, bool normal) {
    for (int k = 1; k < mzone; k++) {
        const int ns = c->zt.nstep[k];
        int mstep;
        if (normal) mstep = c->istep + ns;
        else mstep = c->istep > 0 ? ((c->istep - 1) / ns + 1) * ns : 0;
        std::swap(c->znew[k], c->zold[k]);
        c->lstep[k][0] = c->lstep[k][1];
        c->lstep[k][1] = mstep;
    }
}

// deposit the particles of zones 1..mzone into their arrays (zone 1: c->mass)
static int zone_deposit(GxCtx* c, int mzone, int32_t* perm_out) {
    const int64_t n = c->n;
    const int32_t* keys = c->pkey[c->cur];
    const int32_t* zone = c->pzone[c->cur];
    for (int k = 0; k < mzone; k++) {
        if (n > 0) {
            k_zone_rows<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, keys, zone, n, k + 1,
                                                                           c->rowcnt);
            GX_LAUNCHED(c);
        }
        int rc = gx_deposit_rows(c, keys, c->pfr, perm_out, zone, k + 1,
                                 k == 0 ? c->mass : c->znew[k], 1.f);
        if (rc) return rc;
        GX_CUDA(c, cudaMemcpyAsync(c->zjrk_d + 2 * k, c->jrk_d, 2 * sizeof(int32_t),
                                   cudaMemcpyDeviceToDevice, c->stream));
    }
    return GX_OK;
}

// zoncmb at the current step number
static int zone_combine(GxCtx* c) {
    ZoneSrc src = {};
    for (int k = 1; k < c->nzones; k++) {
        const int ns = c->zt.nstep[k];
        int i = c->lstep[k][1] - c->istep;
        if (i < 0 || i > ns) return c->err = "zone mass array at a useless time", GX_ERR_STATE;
        if (i != ns) {
            src.p[src.n] = c->znew[k];
            src.fr[src.n++] = 1.f - (float)i / (float)ns;
        }
        if (c->lstep[k][1] != c->istep) {
            i = c->istep - c->lstep[k][0];
            if (c->lstep[k][0] < 0 || i < 0 || i > ns)
                return c->err = "older zone mass array at a useless time", GX_ERR_STATE;
            src.p[src.n] = c->zold[k];
            src.fr[src.n++] = 1.f - (float)i / (float)ns;
        }
    }
    const int64_t mesh = c->g.mesh;
    k_zone_combine<<<(unsigned)((mesh + 255) / 256), 256, 0, c->stream>>>(
        mesh, c->mass, src, c->g.pmass, c->nzones, c->g.nr, zone_mzone(c, c->istep), c->zjrk_d,
        c->jrk_d);
    GX_LAUNCHED(c);
    return GX_OK;
}

int gx_zone_loadup(GxCtx* c) {
    const int64_t n = c->n;
    for (int b = 0; b < 2; b++)
        if (!c->pzone[b] && cudaMalloc((void**)&c->pzone[b], sizeof(int32_t) * c->cap) != cudaSuccess) {
            c->pzone[b] = nullptr;
            return c->err = "cudaMalloc of the zone codes failed", GX_ERR_NOMEM;
        }
    c->istep = 0;
    for (int k = 0; k < GX_MAX_ZONES; k++) c->lstep[k][0] = c->lstep[k][1] = -1;
    c->zones_ready = false;
    if (n == 0) return GX_OK;
    k_zone_setup<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, c->zt, c->pbuf[c->cur],
                                                                    c->cap, n, c->pzone[c->cur]);
    GX_LAUNCHED(c);
    return GX_OK;
}

int gx_zone_unload(GxCtx* c, float* staging) {
    const int64_t n = c->n;
    if (n == 0) return GX_OK;
    k_zone_unscale_aos<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        c->zt, c->g.ndim, staging, c->pzone[c->cur], c->origin, n);
    GX_LAUNCHED(c);
    return GX_OK;
}

int gx_zone_masset(GxCtx* c) {
    const int64_t n = c->n;
    if (n > 0) {
        k_zone_keys<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
            c->g, c->pbuf[c->cur], c->cap, n, c->pkey[c->cur], c->pfr);
        GX_LAUNCHED(c);
    }
    zone_masscl(c, c->nzones, false);
    int rc = zone_deposit(c, c->nzones, c->perm);
    if (rc) return rc;
    rc = zone_combine(c);
    if (rc) return rc;
    c->have_keys = true;
    c->zones_ready = true;
    return gx_phase_end(c);
}

int gx_zone_step(GxCtx* c, int nsteps, int phys) {
    if (!c->zones_ready) return c->err = "zone mass arrays not assigned (call gx_masset)", GX_ERR_STATE;
    const int64_t n = c->n;
    for (int s = 0; s < nsteps; s++) {
        const bool last = (s == nsteps - 1);
        const int mzone = zone_mzone(c, c->istep);
        // findf.f:41-54: the field over the rings of zones 1..mzone only, when
        // the outer zones stay and no potential is wanted
        const bool lpot = phys && last;
        const bool partial = !lpot && mzone < c->nzones && !(c->cfg.flags & GX_FLAG_WHOLE_GRID);
        int rc = gx_mixed_findf(c, lpot, true, partial ? c->zjrk_d + 2 * GX_MAX_ZONES : nullptr);
        if (rc) return rc;
        zone_masscl(c, mzone, true);
        const int nxt = c->cur ^ 1;
        rc = gx_phase_mark(c, PH_PUSH);
        if (rc) return rc;
        if (n > 0) {
            k_push_zone<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
                c->g, c->zt, mzone, c->pbuf[c->cur], c->pbuf[nxt], c->cap, n, c->perm, c->origin,
                c->origin_tmp, c->field, c->pkey[c->cur], c->pkey[nxt], c->pfr, c->pzone[c->cur],
                c->pzone[nxt], (phys && last) ? c->ppot : nullptr);
            GX_LAUNCHED(c);
        }
        std::swap(c->origin, c->origin_tmp);
        c->cur = nxt;
        rc = zone_deposit(c, mzone, c->perm_next);
        if (rc) return rc;
        std::swap(c->perm, c->perm_next);
        c->istep += 1;
        rc = zone_combine(c);
        if (rc) return rc;
    }
    int rc = gx_phase_end(c);
    if (rc) return rc;
    c->have_field = false;
    return GX_OK;
}

extern "C" {

int gx_set_zones(GxCtx* c, int32_t nzones, const int32_t* nstep, const float* zbr) {
    if (!c || nzones < 1 || nzones > GX_MAX_ZONES) return GX_ERR_ARG;
    if (nzones > 1 && (!nstep || !zbr)) return GX_ERR_ARG;
    if (c->n > 0) return c->err = "set the zones before gx_loadup", GX_ERR_STATE;
    if (nzones > 1) {
        if (c->fp64) return c->err = "time-step zones run on the mixed path", GX_ERR_ARG;
        if (c->g.comp) return c->err = "time-step zones exclude compensated positions", GX_ERR_ARG;
        if (nstep[0] != 1) return c->err = "nstep[0] must be 1", GX_ERR_ARG;
        for (int i = 1; i < nzones; i++) {
            if (nstep[i] < 1) return c->err = "zone step factors must be >= 1", GX_ERR_ARG;
            // setrun.f:774-790
            if (i > 1 && zbr[i] < zbr[i - 1]) return c->err = "zone boundaries in illogical order", GX_ERR_ARG;
            if (zbr[i] < c->geo.rinh) return c->err = "zone boundary inside the hole", GX_ERR_ARG;
            if (zbr[i] > c->geo.rgrid) return c->err = "zone boundary outside the grid", GX_ERR_ARG;
        }
    }
    cudaSetDevice(c->dev);
    if (c->zbuf) cudaFree(c->zbuf);
    if (c->zjrk_d) cudaFree(c->zjrk_d);
    c->zbuf = nullptr;
    c->zjrk_d = nullptr;
    c->zt = ZoneTab{};
    c->zt.nz = nzones;
    c->zt.nstep[0] = 1;
    for (int i = 1; i < nzones; i++) {
        c->zt.nstep[i] = nstep[i];
        c->zt.zbr[i] = zbr[i];
    }
    for (int k = 0; k < GX_MAX_ZONES; k++) c->znew[k] = c->zold[k] = nullptr;
    c->nzones = nzones;
    c->zones_ready = false;
    if (nzones == 1) return GX_OK;
    const size_t mesh = c->g.mesh;
    if (cudaMalloc((void**)&c->zbuf, sizeof(float) * 2 * (nzones - 1) * mesh) != cudaSuccess ||
        cudaMalloc((void**)&c->zjrk_d, sizeof(int32_t) * (2 * GX_MAX_ZONES + 2)) != cudaSuccess) {
        c->nzones = 1;
        return c->err = "cudaMalloc of the zone mass arrays failed", GX_ERR_NOMEM;
    }
    for (int k = 1; k < nzones; k++) {
        c->znew[k] = c->zbuf + (size_t)(2 * (k - 1)) * mesh;
        c->zold[k] = c->zbuf + (size_t)(2 * (k - 1) + 1) * mesh;
    }
    GX_CUDA(c, cudaMemset(c->zbuf, 0, sizeof(float) * 2 * (nzones - 1) * mesh));
    return GX_OK;
}

int gx_zone_rings(GxCtx* c, int32_t* rings) {
    if (!c || !rings) return GX_ERR_ARG;
    if (c->nzones < 2) return c->err = "no time-step zones (gx_set_zones)", GX_ERR_STATE;
    if (!c->zones_ready) return c->err = "zone mass arrays not assigned (call gx_masset)", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    GX_CUDA(c, cudaMemcpyAsync(rings, c->jrk_d, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaMemcpyAsync(rings + 2, c->zjrk_d + 2 * GX_MAX_ZONES, 2 * sizeof(int32_t),
                               cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    const int mz = zone_mzone(c, c->istep);
    if (mz == c->nzones || (c->cfg.flags & GX_FLAG_WHOLE_GRID)) {
        rings[2] = 1;
        rings[3] = c->g.nr;
    }
    return GX_OK;
}

int gx_zone_info(GxCtx* c, int32_t* zone, int32_t* istep) {
    if (!c) return GX_ERR_ARG;
    if (c->nzones < 2) return c->err = "no time-step zones (gx_set_zones)", GX_ERR_STATE;
    if (istep) *istep = c->istep;
    const int64_t n = c->n;
    if (!zone || n == 0) return GX_OK;
    cudaSetDevice(c->dev);
    int32_t* d = nullptr;
    GX_CUDA(c, cudaMallocAsync((void**)&d, sizeof(int32_t) * n, c->stream));
    k_zone_gather<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->pzone[c->cur], c->origin, n, d);
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaMemcpyAsync(zone, d, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaFreeAsync(d, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

}  // extern "C"
