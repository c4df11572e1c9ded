// gx_api.cu -- C ABI entry points (include/galaxy_gpu.h): context creation
// (grdset/setgrd), particle load/unload, grid access, and dispatch to the
// mixed-precision path (gx_step.cu, gx_solve.cu, gx_deposit.cu) or the plain
// FP64 path (gx_fp64.cu).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>

#include "gx_common.cuh"

static std::string g_last_err;  // errors of gx_grdset before a context exists

// ---------------------------------------------------------------------------
// setgrd for p2d/p3d (SRC/lib15/setgrd.f:52-200), filset's harmonic filter
// (SRC/lib15/filset.f:116-141) and p3dset's softening check
// (SRC/lib15/p3dset.f:99-100).  Reals are formed in FP32 as the reference
// forms them (alpha = 2.*pi/real(na), pi real*8, stored as real).
int setgrd(const GxConfig* c, GxGeometry* g, std::string& err) {
    memset(g, 0, sizeof *g);
    if (c->ndim != 2 && c->ndim != 3) return err = "ndim must be 2 or 3", GX_ERR_ARG;
    int na = 2 * (c->na / 2);
    if (na < 4 || na > 512) return err = "na must be an even number in [4, 512]", GX_ERR_ARG;
    if (c->nr < 3) return err = "nr must be >= 3", GX_ERR_ARG;
    int ngz = 1;
    if (c->ndim == 3) {
        int q = c->ngz;
        if (q < 3) return err = "ngz must be >= 3", GX_ERR_ARG;
        while (q % 3 == 0) q /= 3;
        while (q % 5 == 0) q /= 5;
        if (q != 1) return err = "ngz must be a multiple of 3 & 5", GX_ERR_ARG;
        ngz = c->ngz;
        if (!(c->dzg > 0.f)) return err = "dzg must be positive", GX_ERR_ARG;
    }
    if (c->nsect < 1) return err = "nsect not set", GX_ERR_ARG;
    if (c->tsoft != GX_SOFT_PLUMMER && c->tsoft != GX_SOFT_SPLINE)
        return err = "Unrecognized softening rule", GX_ERR_ARG;
    if (!(c->softl > 0.f)) return err = "Softening length must be greater than 0", GX_ERR_ARG;
    if (c->rmap != GX_RMAP_STDPOL && c->rmap != GX_RMAP_LOG) return err = "unknown radial map", GX_ERR_ARG;
    if (c->rmap == GX_RMAP_LOG && !(c->rmap_r0 > 0.f)) return err = "log map needs rmap_r0 > 0", GX_ERR_ARG;
    if (c->halo < 0 || c->halo > 2) return err = "unknown rigid force (halo)", GX_ERR_ARG;
    if (c->halo > 0 && !(c->halo_rc > 0.f)) return err = "halo_rc must be positive", GX_ERR_ARG;
    if (c->precision != GX_PREC_MIXED && c->precision != GX_PREC_FP64)
        return err = "unknown precision", GX_ERR_ARG;
    if ((c->flags & GX_FLAG_QUADRATIC) && c->ndim != 3)
        return err = "quadratic interpolation is a p3d scheme", GX_ERR_ARG;
    if ((c->flags & GX_FLAG_QUADRATIC) && c->precision == GX_PREC_FP64)
        return err = "quadratic interpolation runs on the mixed path", GX_ERR_ARG;
    g->nr = c->nr;
    g->na = na;
    g->ngz = ngz;
    g->mmax = na / 2 + 1;
    g->ng = std::min(std::max(c->ng, 1), g->mmax);
    g->nsect = c->nsect;
    int64_t mesh = (int64_t)c->nr * na * ngz;
    // cell keys are divided by na in single precision (gx_div_na): below 2^24
    if (mesh >= (int64_t)1 << 24) return err = "mesh too large (2^24 cells at most)", GX_ERR_RANGE;
    g->mesh = (int)mesh;
    g->alpha = (float)(2.0 * GX_PI / (double)(float)na);
    g->ua = (c->rmap_a > 0.f) ? c->rmap_a : g->alpha;
    g->uoffs = (c->rmap == GX_RMAP_LOG) ? -logf(c->rmap_r0) / g->ua : 0.f;
    auto grofu = [&](float u) {
        return (c->rmap == GX_RMAP_STDPOL) ? expf(g->ua * u) - 1.f : expf(g->ua * (u - g->uoffs));
    };
    g->rinh = grofu(0.f);
    g->rgrid = grofu((float)c->nr - 1.f);
    g->zm = (c->ndim == 3) ? 0.5f * c->dzg * (float)(ngz + 1 - 2) : 0.f;
    g->thmax = (float)na / (float)c->nsect;
    for (int m = 0; m < 260; m++) g->lg[m] = 1;
    g->lg[0] = 0;
    for (int m = 1; m < g->ng; m++) g->lg[m] = (c->nsect == 1) ? 0 : (m % c->nsect != 0);
    for (int k = 0; k < c->nskip && k < GX_MAX_SKIP; k++)
        if (c->skip[k] >= 0 && c->skip[k] < 260) g->lg[c->skip[k]] = 1;
    g->nact = 0;
    for (int m = 0; m < g->ng; m++) g->nact += !g->lg[m];
    {
        float a = g->rgrid - grofu((float)(c->nr - 2));
        if (a / c->softl > 5.f) return err = "Unsuitable choice of grid parameters", GX_ERR_ARG;
    }
    if (c->ndim == 3 && c->softl < c->dzg)
        return err = "Softening length cannot be less than z-spacing of grid planes", GX_ERR_ARG;
    return GX_OK;
}

void fill_devgeo(GxCtx* c) {
    const GxGeometry& G = c->geo;
    DevGeo& d = c->g;
    memset(&d, 0, sizeof d);
    d.ndim = c->cfg.ndim;
    d.nr = G.nr;
    d.na = G.na;
    d.ngz = G.ngz;
    d.nkz = (d.ndim == 3) ? G.ngz + 1 : 1;
    d.ng = G.ng;
    d.mmax = G.mmax;
    d.nsect = G.nsect;
    d.mesh = G.mesh;
    d.nrow = G.nr * G.ngz;
    d.rmap = c->cfg.rmap;
    d.tsoft = c->cfg.tsoft;
    d.halo = c->cfg.halo;
    d.alpha = G.alpha;
    d.ua = G.ua;
    d.inv_ua = 1.0f / G.ua;
    d.uoffs = G.uoffs;
    d.rinh = G.rinh;
    d.rgrid = G.rgrid;
    d.zm = G.zm;
    d.thmax = G.thmax;
    d.dzg = c->cfg.dzg;
    d.inv_dzg = (d.ndim == 3) ? 1.0f / c->cfg.dzg : 0.f;
    d.t_scale = (float)((double)G.na / (2.0 * GX_PI));
    d.inv_na = 1.0f / (float)G.na;
    d.fna = (float)G.na;
    d.eps_t = 4.0e-6f * (float)(G.na + 1);
    d.eps_z = 4.0e-6f * ((float)G.ngz + 1.f);
    d.comp = (c->cfg.flags & GX_FLAG_COMPENSATED) ? 1 : 0;
    d.quad = (c->cfg.ndim == 3 && (c->cfg.flags & GX_FLAG_QUADRATIC)) ? 1 : 0;
    d.halo_v2 = c->cfg.halo_v2;
    d.halo_rc2 = c->cfg.halo_rc * c->cfg.halo_rc;
    d.pmass = c->cfg.pmass;
    // FP64 geometry of the plain path
    d.ua_d = (c->cfg.rmap_a > 0.f) ? (double)c->cfg.rmap_a : 2.0 * GX_PI / (double)G.na;
    d.uoffs_d = (d.rmap == GX_RMAP_LOG) ? -log((double)c->cfg.rmap_r0) / d.ua_d : 0.0;
    if (d.rmap == GX_RMAP_STDPOL) {
        d.rinh_d = 0.0;
        d.rgrid_d = exp(d.ua_d * (double)(G.nr - 1)) - 1.0;
    } else {
        d.rinh_d = exp(d.ua_d * (0.0 - d.uoffs_d));
        d.rgrid_d = exp(d.ua_d * ((double)(G.nr - 1) - d.uoffs_d));
    }
    d.zm_d = 0.5 * (double)c->cfg.dzg * (double)(G.ngz - 1);
    d.thmax_d = (double)G.na / (double)G.nsect;
    d.dzg_d = (double)c->cfg.dzg;
    d.halo_v2_d = (double)c->cfg.halo_v2;
    d.halo_rc2_d = (double)c->cfg.halo_rc * (double)c->cfg.halo_rc;
    Spec& s = c->spec;
    s.nact = 0;
    for (int m = 0; m < G.ng; m++)
        if (!G.lg[m]) s.m[s.nact++] = m;
}

template <typename T>
static int dalloc(GxCtx* c, T** p, size_t count) {
    if (*p) return GX_OK;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
    if (e != cudaSuccess) {
        c->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        *p = nullptr;
        return GX_ERR_NOMEM;
    }
    return GX_OK;
}
#define DALLOC(c, p, n)                      \
    do {                                     \
        int rc_ = dalloc((c), &(p), (n));    \
        if (rc_) return rc_;                 \
    } while (0)

// grid-sized arrays, allocated once per context
static int alloc_grids(GxCtx* c) {
    const DevGeo& g = c->g;
    const size_t mesh = g.mesh;
    const size_t nspec = (size_t)c->spec.nact * g.nkz * g.nr;
    if (c->fp64) {
        DALLOC(c, c->mass64, mesh);
        DALLOC(c, c->field64, 4 * mesh);
        DALLOC(c, c->polar64, 4 * mesh);
        DALLOC(c, c->spec64, 4 * nspec);
        DALLOC(c, c->out64, 16 * nspec);
        // solve scratch, once per context (a solve allocates nothing)
        const size_t naz = (size_t)g.nr * g.ngz * c->spec.nact * 2;
        DALLOC(c, c->az64, naz);
        DALLOC(c, c->rows64, 4 * naz);
    } else {
        DALLOC(c, c->mass, mesh);
        DALLOC(c, c->field, mesh);
        DALLOC(c, c->specS, nspec);
        DALLOC(c, c->specO, 4 * nspec);
        DALLOC(c, c->rowstart, (size_t)g.nrow + 2);
        DALLOC(c, c->rowitem, (size_t)g.nrow + 2);
        DALLOC(c, c->rowcnt, (size_t)NCOPY * (g.nrow + 1));
        DALLOC(c, c->rowfill, (size_t)NCOPY * (g.nrow + 1));
        DALLOC(c, c->rowbase, (size_t)NCOPY * (g.nrow + 1));
        DALLOC(c, c->rowtot, (size_t)g.nrow + 1);
        DALLOC(c, c->rowtile, (size_t)4 * ((g.nrow + 1 + ROW_TILE - 1) / ROW_TILE));
        DALLOC(c, c->nitems_d, 4);
        GX_CUDA(c, cudaMemsetAsync(c->rowcnt, 0, sizeof(uint32_t) * NCOPY * (g.nrow + 1), c->stream));
        int rc = gx_bucket_alloc(c);
        if (rc) return rc;
    }
    DALLOC(c, c->jrk_d, 4);
    DALLOC(c, c->errword, 4);
    DALLOC(c, c->dsum, 64);
    GX_CUDA(c, cudaMemsetAsync(c->errword, 0, 4 * sizeof(int32_t), c->stream));
    return GX_OK;
}

extern "C" {

int gx_grdset(const GxConfig* cfg, GxCtx** out) {
    if (!cfg || !out) {
        g_last_err = "null argument";
        return GX_ERR_ARG;
    }
    *out = nullptr;
    GxGeometry geo;
    std::string err;
    int rc = setgrd(cfg, &geo, err);
    if (rc) {
        g_last_err = err;
        return rc;
    }
    GxCtx* c = new GxCtx();
    c->cfg = *cfg;
    c->geo = geo;
    c->fp64 = (cfg->precision == GX_PREC_FP64);
    fill_devgeo(c);
    c->dev = cfg->device;
    cudaError_t e = cudaSetDevice(c->dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e != cudaSuccess) {
        g_last_err = std::string("CUDA initialisation: ") + cudaGetErrorString(e);
        delete c;
        return GX_ERR_CUDA;
    }
    rc = alloc_grids(c);
    if (rc == GX_OK) {
        // the active harmonics, once per context (the kernels read them through DevGeo)
        if (cudaMalloc((void**)&c->act_d, sizeof(int) * 260) != cudaSuccess ||
            cudaMemcpy(c->act_d, c->spec.m, sizeof(int) * 260, cudaMemcpyHostToDevice) != cudaSuccess) {
            c->err = "cudaMalloc of the harmonic list failed";
            rc = GX_ERR_NOMEM;
        }
        c->g.act = c->act_d;
    }
    if (rc) {
        g_last_err = c->err;
        gx_destroy(c);
        return rc;
    }
    *out = c;
    return GX_OK;
}

void gx_destroy(GxCtx* c) {
    if (!c) return;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    gx_comm_destroy(c);
    void* ptrs[] = {c->green32, c->green64, c->pbuf[0], c->pbuf[1], c->perm, c->origin,
                    c->origin_tmp, c->pkey[0], c->pkey[1], c->pfr, c->p64, c->key64, c->w64, c->acc64, c->ppot,
                    c->pacc, c->mass, c->mass64, c->field, c->polar, c->field64, c->polar64,
                    c->specS, c->specO, c->syntab, c->synR, c->fwdtab, c->fwdC1, c->spec64, c->out64, c->az64, c->rows64, c->pot64, c->stagebuf, c->perm_next, c->rowstart,
                    c->items, c->nitems_d, c->rowitem, c->rowcnt, c->rowfill, c->rowbase, c->rowtot, c->rowtile, c->stage, c->jrk_d,
                    c->errword, c->dsum, c->pzone[0], c->pzone[1], c->zbuf, c->zjrk_d, c->act_d,
                    c->bk_cap[0], c->bk_cap[1], c->bk_base[0], c->bk_base[1], c->bk_fill[0], c->bk_fill[1],
                    c->bk_ctl, c->bk_items, c->bk_cnt, c->macc, c->bq[0], c->bq[1], c->zr_d};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (cudaEvent_t e : c->pev) cudaEventDestroy(e);
    if (c->bk_side) cudaStreamSynchronize(c->bk_side);
    for (cudaEvent_t e : c->bk_ev)
        if (e) cudaEventDestroy(e);
    if (c->bk_side) cudaStreamDestroy(c->bk_side);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* gx_last_error(const GxCtx* c) {
    if (!c) return g_last_err.c_str();
    return c->err.c_str();
}

int gx_geometry(const GxCtx* c, GxGeometry* geo) {
    if (!c || !geo) return GX_ERR_ARG;
    *geo = c->geo;
    return GX_OK;
}

int gx_greenm(GxCtx* c) {
    if (!c) return GX_ERR_ARG;
    cudaSetDevice(c->dev);
    return gx_green_build_dev(c);
}

int gx_green_get(GxCtx* c, int type, double* out, int64_t n) {
    if (!c || !out || type < 0 || type > 3) return GX_ERR_ARG;
    if (!c->have_green) return c->err = "no Green table (call gx_greenm)", GX_ERR_STATE;
    const DevGeo& g = c->g;
    int64_t per = (int64_t)g.ng * g.nkz * g.nr * g.nr;
    if (n != per) return c->err = "element count mismatch", GX_ERR_ARG;
    cudaSetDevice(c->dev);
    if (c->fp64) {
        GX_CUDA(c, cudaMemcpyAsync(out, c->green64 + type * per, per * sizeof(double),
                                   cudaMemcpyDeviceToHost, c->stream));
        GX_CUDA(c, cudaStreamSynchronize(c->stream));
    } else {
        std::vector<float> tmp(per);
        GX_CUDA(c, cudaMemcpyAsync(tmp.data(), c->green32 + type * per, per * sizeof(float),
                                   cudaMemcpyDeviceToHost, c->stream));
        GX_CUDA(c, cudaStreamSynchronize(c->stream));
        for (int64_t i = 0; i < per; i++) out[i] = tmp[i];
    }
    return GX_OK;
}

}  // extern "C"

// phase marks: a phase runs from its mark to the next mark (or the end).
// Marks only record events; gx_phase_end waits for the last one and adds
// up the elapsed times.  Only done in profile mode.
static int phase_record(GxCtx* c, int ph) {
    if (c->nmarks == (int)c->pev.size()) {
        cudaEvent_t e;
        GX_CUDA(c, cudaEventCreate(&e));
        c->pev.push_back(e);
        c->pev_ph.push_back(-1);
    }
    GX_CUDA(c, cudaEventRecord(c->pev[c->nmarks], c->stream));
    c->pev_ph[c->nmarks++] = ph;
    return GX_OK;
}

int gx_phase_mark(GxCtx* c, int ph) {
    if (!c->prof) return GX_OK;
    return phase_record(c, ph);
}

int gx_phase_end(GxCtx* c) {
    if (!c->prof || c->nmarks == 0) return GX_OK;
    int rc = phase_record(c, -1);
    if (rc) return rc;
    GX_CUDA(c, cudaEventSynchronize(c->pev[c->nmarks - 1]));
    for (int k = 0; k + 1 < c->nmarks; k++) {
        const int ph = c->pev_ph[k];
        if (ph < 0) continue;
        float ms = 0.f;
        GX_CUDA(c, cudaEventElapsedTime(&ms, c->pev[k], c->pev[k + 1]));
        c->phase_ms[ph] += ms;
        c->phase_n[ph] += 1;
    }
    c->nmarks = 0;
    return GX_OK;
}

// ---------------------------------------------------------------------------
// AoS <-> SoA transposes
__global__ void k_aos_to_soa(const float* __restrict__ aos, float* __restrict__ soa, int64_t n,
                             int64_t cap, int nw) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < nw; k++) soa[k * cap + i] = aos[i * nw + k];
}

__global__ void k_aos_to_soa64(const float* __restrict__ aos, double* __restrict__ soa, int64_t n,
                               int64_t cap, int nw) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < nw; k++) soa[k * cap + i] = (double)aos[i * nw + k];
}

// unload in load order: soa index i holds original particle origin[i]
__global__ void k_soa_to_aos(const float* __restrict__ soa, const int32_t* __restrict__ origin,
                             float* __restrict__ aos, int64_t n, int64_t cap, int nw) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t o = origin ? origin[i] : i;
    for (int k = 0; k < nw; k++) aos[o * nw + k] = soa[k * cap + i];
}

__global__ void k_soa64_to_aos(const double* __restrict__ soa, float* __restrict__ aos, int64_t n,
                               int64_t cap, int nw) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < nw; k++) aos[i * nw + k] = (float)soa[k * cap + i];
}

__global__ void k_iota(int32_t* p, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = (int32_t)i;
}

static int alloc_particles(GxCtx* c, int64_t n) {
    const int nw = 2 * c->g.ndim;
    if (n <= c->cap && c->cap > 0) return GX_OK;
    // grow: free old
    void* old[] = {c->pbuf[0], c->pbuf[1], c->perm, c->origin, c->origin_tmp, c->pkey[0], c->pkey[1],
                   c->pfr, c->p64,
                   c->key64, c->w64, c->acc64, c->pot64, c->ppot, c->pacc, c->perm_next, c->items,
                   c->stage, c->pzone[0], c->pzone[1], c->bk_items};
    for (void* p : old)
        if (p) cudaFree(p);
    c->pbuf[0] = c->pbuf[1] = nullptr;
    c->perm = c->origin = c->origin_tmp = nullptr;
    c->pkey[0] = c->pkey[1] = nullptr;
    c->pfr = nullptr;
    c->pzone[0] = c->pzone[1] = nullptr;
    c->p64 = nullptr;
    c->key64 = nullptr;
    c->w64 = c->acc64 = c->pot64 = nullptr;
    c->ppot = c->pacc = nullptr;
    if (c->stagebuf) cudaFree(c->stagebuf);
    c->stagebuf = nullptr;
    c->perm_next = nullptr;
    c->items = nullptr;
    c->stage = nullptr;
    c->bk_items = nullptr;
    for (int b = 0; b < 2; b++) {
        if (c->bq[b]) cudaFree(c->bq[b]);
        c->bq[b] = nullptr;
    }
    c->bucketed = false;
    int64_t cap = std::max<int64_t>(n, 1);
    c->cap = cap;
    DALLOC(c, c->ppot, cap);
    DALLOC(c, c->pacc, 3 * cap);
    // staging of the host records (AoS) for loadup and unload, once per
    // capacity: a per-call allocation would map and unmap it every time
    DALLOC(c, c->stagebuf, (size_t)nw * cap);
    if (c->fp64) {
        DALLOC(c, c->p64, nw * cap);
        DALLOC(c, c->key64, cap);
        DALLOC(c, c->w64, 8 * cap);
        DALLOC(c, c->acc64, 3 * cap);
        DALLOC(c, c->pot64, cap);
        return GX_OK;
    }
    // compensated positions keep a low part of every coordinate after the
    // 2 ndim planes of the records
    const int planes = nw + (c->g.comp ? c->g.ndim : 0);
    DALLOC(c, c->pbuf[0], planes * cap);
    DALLOC(c, c->pbuf[1], planes * cap);
    DALLOC(c, c->perm, cap);
    DALLOC(c, c->origin, cap);
    DALLOC(c, c->origin_tmp, cap);
    DALLOC(c, c->pkey[0], cap);
    DALLOC(c, c->pkey[1], cap);
    DALLOC(c, c->pfr, 3 * cap);
    DALLOC(c, c->perm_next, cap);
    // deposit work items: every row once plus one per DEP_CH particles
    c->maxitems = c->g.nrow + 1 + (int)((cap + DEP_CH - 1) / DEP_CH);
    DALLOC(c, c->items, (size_t)3 * c->maxitems);
    int nq = c->g.quad ? 9 : (c->g.ndim == 3) ? 4 : 2;
    DALLOC(c, c->stage, (size_t)c->maxitems * nq * c->g.na);
    // fused-pass work items: every row's segment in chunks of bk_item
    // particles, and the overflow area's.  bk_item: at most BK_ITEM, at
    // least half a deposit window of particles (the bins each item
    // flushes), and otherwise small enough that a B200's resident CTAs
    // (148 SMs x 5) get two items each when the particles are few
    {
        const int64_t wrows = (c->g.ndim == 3) ? 16 : 4;
        const int64_t wmin = std::min<int64_t>(BK_ITEM, std::max<int64_t>(256, wrows * c->g.na / 2));
        c->bk_item = (int)std::min<int64_t>(BK_ITEM, std::max<int64_t>(wmin, n / (2 * 148 * 5)));
    }
    c->bk_maxitems = (int64_t)c->g.nrow + 1 + 2 * (n / c->bk_item + 2);
    DALLOC(c, c->bk_items, (size_t)c->bk_maxitems);
    // the bucketed store: row segments with 1/8 + 16 slots of slack per row,
    // then an overflow area that can take every particle
    c->bk_main = cap + cap / 8 + 16 * ((int64_t)c->g.nrow + 1);
    c->bcap = c->bk_main + cap + 64;
    if (c->bcap > (int64_t)INT32_MAX) return c->err = "too many particles for the bucketed store", GX_ERR_RANGE;
    for (int b = 0; b < 2; b++) DALLOC(c, c->bq[b], (size_t)gx_bucket_words(c) * c->bcap);
    return GX_OK;
}

extern "C" {

int gx_loadup(GxCtx* c, const float* coords, int64_t n) {
    if (!c || n < 0 || (n > 0 && !coords)) return GX_ERR_ARG;
    if (n > (int64_t)INT32_MAX - 1) return c->err = "too many particles", GX_ERR_RANGE;
    cudaSetDevice(c->dev);
    int rc = alloc_particles(c, n);
    if (rc) return rc;
    c->n = n;
    c->have_mass = c->have_field = c->have_keys = false;
    c->bucketed = false;
    c->zr_valid = false;
    const int nw = 2 * c->g.ndim;
    if (n == 0) return (c->nzones > 1 && !c->fp64) ? gx_zone_loadup(c) : GX_OK;
    float* staging = c->stagebuf;
    GX_CUDA(c, cudaMemcpyAsync(staging, coords, sizeof(float) * nw * n, cudaMemcpyHostToDevice,
                               c->stream));
    int bs = 256;
    int64_t nb = (n + bs - 1) / bs;
    if (c->fp64) {
        k_aos_to_soa64<<<nb, bs, 0, c->stream>>>(staging, c->p64, n, c->cap, nw);
        GX_LAUNCHED(c);
    } else {
        c->cur = 0;
        k_aos_to_soa<<<nb, bs, 0, c->stream>>>(staging, c->pbuf[0], n, c->cap, nw);
        GX_LAUNCHED(c);
        if (c->g.comp)
            GX_CUDA(c, cudaMemsetAsync(c->pbuf[0] + (size_t)nw * c->cap, 0,
                                       sizeof(float) * c->g.ndim * c->cap, c->stream));
        k_iota<<<nb, bs, 0, c->stream>>>(c->origin, n);
        GX_LAUNCHED(c);
        k_iota<<<nb, bs, 0, c->stream>>>(c->perm, n);
        GX_LAUNCHED(c);
        if (c->nzones > 1) {
            rc = gx_zone_loadup(c);
            if (rc) return rc;
        }
    }
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

int gx_unload(GxCtx* c, float* coords) {
    if (!c || (!coords && c->n > 0)) return GX_ERR_ARG;
    if (c->n == 0) return GX_OK;
    cudaSetDevice(c->dev);
    if (c->bucketed && !c->fp64 && c->nzones <= 1) {
        // the step's bucketed store straight into the records, in load order
        int rc = gx_bucket_unload(c, c->stagebuf);
        if (rc) return rc;
        GX_CUDA(c, cudaMemcpyAsync(coords, c->stagebuf, sizeof(float) * 2 * c->g.ndim * c->n,
                                   cudaMemcpyDeviceToHost, c->stream));
        GX_CUDA(c, cudaStreamSynchronize(c->stream));
        return GX_OK;
    }
    int rc = gx_dense(c);
    if (rc) return rc;
    const int nw = 2 * c->g.ndim;
    const int64_t n = c->n;
    float* staging = c->stagebuf;
    int bs = 256;
    int64_t nb = (n + bs - 1) / bs;
    if (c->fp64) k_soa64_to_aos<<<nb, bs, 0, c->stream>>>(c->p64, staging, n, c->cap, nw);
    else k_soa_to_aos<<<nb, bs, 0, c->stream>>>(c->pbuf[c->cur], c->origin, staging, n, c->cap, nw);
    GX_LAUNCHED(c);
    if (c->nzones > 1) {
        rc = gx_zone_unload(c, staging);
        if (rc) return rc;
    }
    GX_CUDA(c, cudaMemcpyAsync(coords, staging, sizeof(float) * nw * n, cudaMemcpyDeviceToHost,
                               c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

int gx_masset(GxCtx* c) {
    if (!c) return GX_ERR_ARG;
    cudaSetDevice(c->dev);
    if (gx_fast_ok(c)) {
        int rc = gx_fast_masset(c);
        if (rc) return rc;
        GX_CUDA(c, cudaStreamSynchronize(c->stream));
        c->have_mass = true;
        c->have_field = false;
        return GX_OK;
    }
    int rc = gx_dense(c);
    if (rc) return rc;
    c->zr_valid = false;
    rc = c->fp64 ? gx_fp64_masset(c) : (c->nzones > 1 ? gx_zone_masset(c) : gx_mixed_masset(c));
    if (rc) return rc;
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_mass = true;
    c->have_field = false;
    return GX_OK;
}

int gx_findf(GxCtx* c, int lpot) {
    if (!c) return GX_ERR_ARG;
    if (!c->have_green) return c->err = "no Green table (call gx_greenm)", GX_ERR_STATE;
    if (!c->have_mass) return c->err = "no mass array (call gx_masset)", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    int rc = c->fp64 ? gx_fp64_findf(c, lpot, true) : gx_mixed_findf(c, lpot, true);
    if (rc) return rc;
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

int gx_findf_polar(GxCtx* c, int lpot) {
    if (!c) return GX_ERR_ARG;
    if (!c->have_green) return c->err = "no Green table (call gx_greenm)", GX_ERR_STATE;
    if (!c->have_mass) return c->err = "no mass array (call gx_masset)", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    int rc = c->fp64 ? gx_fp64_findf(c, lpot, false) : gx_mixed_findf(c, lpot, false);
    if (rc) return rc;
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

int gx_getacc(GxCtx* c, float* acc, float* pot) {
    if (!c || (!acc && c->n > 0)) return GX_ERR_ARG;
    if (!c->have_field) return c->err = "no fields (call gx_findf)", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    int rc = gx_dense(c);
    if (rc) return rc;
    rc = c->fp64 ? gx_fp64_getacc(c, acc, pot) : gx_mixed_getacc(c, acc, pot);
    if (rc) return rc;
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

int gx_step(GxCtx* c, int nsteps, int phys) {
    if (!c || nsteps < 0) return GX_ERR_ARG;
    if (!c->have_green) return c->err = "no Green table (call gx_greenm)", GX_ERR_STATE;
    if (!c->have_mass) return c->err = "no mass array (call gx_masset)", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    c->launches = 0;
    GX_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    int rc;
    if (c->fp64) rc = gx_fp64_step(c, nsteps, phys);
    else if (gx_fast_ok(c)) rc = gx_fast_step(c, nsteps, phys);
    else if ((rc = gx_dense(c)) == GX_OK) {
        c->zr_valid = false;
        rc = (c->nzones > 1) ? gx_zone_step(c, nsteps, phys) : gx_mixed_step(c, nsteps, phys);
    }
    if (rc) return rc;
    GX_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    GX_CUDA(c, cudaEventSynchronize(c->ev1));
    GX_CUDA(c, cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
    int32_t ew = 0;
    GX_CUDA(c, cudaMemcpy(&ew, c->errword, sizeof ew, cudaMemcpyDeviceToHost));
    if (ew) {
        char b[96];
        snprintf(b, sizeof b, "device check raised error word %d", ew);
        c->err = b;
        return GX_ERR_DEVICE;
    }
    return GX_OK;
}

int gx_host_alloc(int64_t bytes, void** ptr) {
    if (!ptr || bytes < 0) return GX_ERR_ARG;
    *ptr = nullptr;
    if (cudaMallocHost(ptr, (size_t)std::max<int64_t>(bytes, 1)) != cudaSuccess) {
        *ptr = nullptr;
        return GX_ERR_NOMEM;
    }
    return GX_OK;
}

int gx_host_free(void* ptr) {
    if (ptr && cudaFreeHost(ptr) != cudaSuccess) return GX_ERR_CUDA;
    return GX_OK;
}

int gx_set_profile(GxCtx* c, int on) {
    if (!c) return GX_ERR_ARG;
    cudaSetDevice(c->dev);
    c->prof = on != 0;
    c->nmarks = 0;
    for (int i = 0; i < GX_NPHASE; i++) {
        c->phase_ms[i] = 0.f;
        c->phase_n[i] = 0;
    }
    return GX_OK;
}

int gx_phase_ms(const GxCtx* c, float* ms, int64_t* count) {
    if (!c || !ms || !count) return GX_ERR_ARG;
    for (int i = 0; i < GX_NPHASE; i++) {
        ms[i] = c->phase_ms[i];
        count[i] = c->phase_n[i];
    }
    return GX_OK;
}

int gx_last_step_ms(const GxCtx* c, float* ms) {
    if (!c || !ms) return GX_ERR_ARG;
    *ms = c->last_ms;
    return GX_OK;
}

int gx_last_launch_count(const GxCtx* c, int64_t* n) {
    if (!c || !n) return GX_ERR_ARG;
    *n = c->launches;
    return GX_OK;
}

}  // extern "C"
