/*
 * gx_oracle.c -- CPU restatement of the GALAXY v15 polar-grid PM step.
 * TEST INFRASTRUCTURE ONLY (see gx_oracle.h): what the CUDA library's
 * results are checked against, never part of the product path.
 */
#include "gx_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OX_PI 3.141592653589793238462643

#ifdef _OPENMP
#include <omp.h>
#define OX_TID (ox_threads > 1 ? omp_get_thread_num() : 0)
#else
#define OX_TID 0
#endif

/* host threads used by the restated loops (1: sequential, deterministic) */
static int ox_threads = 1;
int ox_set_threads(int n) {
#ifdef _OPENMP
    ox_threads = n < 1 ? 1 : (n > 256 ? 256 : n);
#else
    (void)n;
    ox_threads = 1;
#endif
    return ox_threads;
}

/* setgrd (SRC/lib15/setgrd.f:52-200) for p2d/p3d, the harmonic filter of
 * filset (SRC/lib15/filset.f:116-141), and the grid-size checks of p3dset
 * (SRC/lib15/p3dset.f:99-100).  Reals are formed in FP32 as the reference
 * does (alpha = 2.*pi/real(na) with pi real*8, stored in a real). */
int ox_geometry(const GxConfig* c, GxGeometry* g, char* err, int errlen) {
    memset(g, 0, sizeof *g);
    if (c->ndim != 2 && c->ndim != 3) {
        snprintf(err, errlen, "ndim must be 2 or 3");
        return GX_ERR_ARG;
    }
    int na = 2 * (c->na / 2);
    int nr = c->nr;
    int ngz = 1;
    if (na < 4 || na > 512) {
        snprintf(err, errlen, "na must be an even number in [4, 512]");
        return GX_ERR_ARG;
    }
    if (nr < 3) {
        snprintf(err, errlen, "nr must be >= 3");
        return GX_ERR_ARG;
    }
    if (c->ndim == 3) {
        int q = c->ngz;
        if (q < 3) {
            snprintf(err, errlen, "ngz must be >= 3");
            return GX_ERR_ARG;
        }
        while (q % 3 == 0) q /= 3;
        while (q % 5 == 0) q /= 5;
        if (q != 1) {
            snprintf(err, errlen, "ngz must be a multiple of 3 & 5");
            return GX_ERR_ARG;
        }
        ngz = c->ngz;
        if (!(c->dzg > 0.f)) {
            snprintf(err, errlen, "dzg must be positive");
            return GX_ERR_ARG;
        }
    }
    if (c->nsect < 1) {
        snprintf(err, errlen, "nsect not set");
        return GX_ERR_ARG;
    }
    if (c->tsoft != GX_SOFT_PLUMMER && c->tsoft != GX_SOFT_SPLINE) {
        snprintf(err, errlen, "Unrecognized softening rule");
        return GX_ERR_ARG;
    }
    if (!(c->softl > 0.f)) {
        snprintf(err, errlen, "softl must be positive");
        return GX_ERR_ARG;
    }
    if (c->rmap != GX_RMAP_STDPOL && c->rmap != GX_RMAP_LOG) {
        snprintf(err, errlen, "unknown radial map");
        return GX_ERR_ARG;
    }
    if (c->rmap == GX_RMAP_LOG && !(c->rmap_r0 > 0.f)) {
        snprintf(err, errlen, "log map needs rmap_r0 > 0");
        return GX_ERR_ARG;
    }
    g->nr = nr;
    g->na = na;
    g->ngz = ngz;
    g->mmax = na / 2 + 1;
    g->ng = c->ng < 1 ? 1 : c->ng;
    if (g->ng > g->mmax) g->ng = g->mmax;
    g->nsect = c->nsect;
    g->mesh = nr * na * ngz;
    g->alpha = (float)(2.0 * OX_PI / (double)(float)na);
    g->ua = (c->rmap_a > 0.f) ? c->rmap_a : g->alpha;
    g->uoffs = (c->rmap == GX_RMAP_LOG) ? -logf(c->rmap_r0) / g->ua : 0.f;
    /* grofu in FP32 */
#define GROFU(u) ((c->rmap == GX_RMAP_STDPOL) ? expf(g->ua * (u)) - 1.f \
                                              : expf(g->ua * ((u) - g->uoffs)))
    g->rinh = GROFU(0.f);
    g->rgrid = GROFU((float)nr - 1.f);
    g->zm = (c->ndim == 3) ? 0.5f * c->dzg * (float)(ngz + 1 - 2) : 0.f;
    g->thmax = (float)na / (float)c->nsect;
    /* harmonic filter; lg[m] true means m is skipped */
    for (int m = 0; m < 260; m++) g->lg[m] = 1;
    g->lg[0] = 0;
    for (int m = 1; m < g->ng; m++) g->lg[m] = (c->nsect == 1) ? 0 : (m % c->nsect != 0);
    for (int k = 0; k < c->nskip && k < GX_MAX_SKIP; k++)
        if (c->skip[k] >= 0 && c->skip[k] < 260) g->lg[c->skip[k]] = 1;
    g->nact = 0;
    for (int m = 0; m < g->ng; m++) g->nact += !g->lg[m];
    /* outermost cell size against the softening (setgrd.f:150-171) */
    {
        float a = g->rgrid - GROFU((float)(nr - 2));
        if (a / c->softl > 5.f) {
            snprintf(err, errlen, "Unsuitable choice of grid parameters (outer cell %.4g softl)",
                     a / c->softl);
            return GX_ERR_ARG;
        }
    }
#undef GROFU
    if (c->ndim == 3 && c->softl < c->dzg) {
        /* p3dset.f:99-100 */
        snprintf(err, errlen, "softening length must be >= the plane spacing");
        return GX_ERR_ARG;
    }
    return GX_OK;
}

int64_t ox_green_size(const GxConfig* c) {
    GxGeometry g;
    char e[128];
    if (ox_geometry(c, &g, e, sizeof e)) return -1;
    int nkz = (c->ndim == 3) ? g.ngz + 1 : 1;
    return (int64_t)4 * g.ng * nkz * g.nr * g.nr;
}

int64_t ox_direct_size(const GxConfig* c) {
    GxGeometry g;
    char e[128];
    if (ox_geometry(c, &g, e, sizeof e)) return -1;
    int nkz = (c->ndim == 3) ? g.ngz + 1 : 1;
    return (int64_t)4 * g.nr * g.nr * nkz * (g.na / 2 + 1);
}

/* FP64 flavour */
#define R double
#define S f64
#define MIRROR 0
#define SQRT sqrt
#define LOG log
#define EXP exp
#define COS cos
#define SIN sin
#define FABS fabs
#define FMOD fmod
#define POW pow
#include "gx_oracle_tmpl.h"
#include "gx_oracle_adj.h"
#include "gx_oracle_zone.h"
#undef R
#undef S
#undef MIRROR
#undef SQRT
#undef LOG
#undef EXP
#undef COS
#undef SIN
#undef FABS
#undef FMOD
#undef POW

/* FP32 mirror flavour */
#define R float
#define S f32
#define MIRROR 1
#define SQRT sqrtf
#define LOG logf
#define EXP expf
#define COS cosf
#define SIN sinf
#define FABS fabsf
#define FMOD fmodf
#define POW powf
#include "gx_oracle_tmpl.h"

/* icheck (SRC/lib15/icheck.f:61-92) in FP64, plus the m = 2 amplitude of
 * the mass distribution (A2 = sum m e^{2 i phi} / sum m).  pos are
 * time-centred records; acc (optional) for the virial; pot (optional). */
int ox_icheck(const GxConfig* c, int64_t n, const double* pos, const double* acc,
              const double* pot, double pm, GxDiag* d) {
    const int nd = c->ndim, stride = 2 * nd;
    memset(d, 0, sizeof *d);
    double sre = 0, sim = 0, msum = 0;
    for (int64_t p = 0; p < n; p++) {
        const double* q = pos + p * stride;
        for (int i = 0; i < nd; i++) {
            d->ke += pm * q[nd + i] * q[nd + i];
            if (acc) d->virial += q[i] * pm * acc[p * nd + i];
        }
        if (pot) d->pe += 0.5 * pm * pot[p];
        d->lz += pm * (q[nd + 1] * q[0] - q[nd] * q[1]);
        double r2 = q[0] * q[0] + q[1] * q[1];
        if (r2 > 0) {
            double c2 = (q[0] * q[0] - q[1] * q[1]) / r2, s2 = 2 * q[0] * q[1] / r2;
            sre += pm * c2;
            sim += pm * s2;
        }
        msum += pm;
    }
    if (msum > 0) {
        d->a2_re = sre / msum;
        d->a2_im = sim / msum;
    }
    d->n_on_grid = n;
    return 0;
}

/* danl (SRC/lib15/densty.f:82-118, 190-250): surface density of the mass
 * projected onto one plane (ring areas from FP32 grofu as the reference
 * forms them), per ring the FFTPACK forward sums for m = 0 .. ng - 1
 * (a_m = sum x cos, the sine sum sum x sin = -b_m), m >= 1 divided by the
 * m = 0 term unless the ring is empty or that term is below 1e-6 of them.
 * w: real parts [nr][ng] then imaginary parts [nr][ng].                   */
int ox_danl(const GxConfig* c, const double* mass, double sigmaf, double* w) {
    GxGeometry geo;
    char err[256];
    if (ox_geometry(c, &geo, err, sizeof err)) return GX_ERR_ARG;
    const int nr = geo.nr, na = geo.na, ng = geo.ng, ngz = (c->ndim == 3) ? geo.ngz : 1;
#define GROFU(u) ((c->rmap == GX_RMAP_STDPOL) ? expf(geo.ua * (u)) - 1.f \
                                              : expf(geo.ua * ((u) - geo.uoffs)))
    float r1 = GROFU(0.f);
    double* sig = (double*)malloc(sizeof(double) * na);
    for (int i = 0; i < nr; i++) {
        const float r2 = GROFU((float)(i + 1) - 0.5f);
        const float area = 0.5f * geo.alpha * (r2 * r2 - r1 * r1);
        const double cf = (double)(float)(sigmaf / (double)area);
        r1 = r2;
        for (int j = 0; j < na; j++) {
            double s = 0;
            for (int iz = 0; iz < ngz; iz++) s += mass[((int64_t)i * ngz + iz) * na + j];
            sig[j] = cf * s;
        }
        double c0 = 0;
        for (int m = 0; m < ng; m++) {
            double a = 0, b = 0;
            for (int j = 0; j < na; j++) {
                const double ph = 2.0 * OX_PI * (double)((int64_t)m * j % na) / (double)na;
                a += sig[j] * cos(ph);
                b += sig[j] * sin(ph);
            }
            double re = 0, im = 0;
            if (m == 0) {
                c0 = a;
                re = a;
            } else if (c0 > 0 && c0 > 1e-6 * fmax(fabs(a), fabs(b))) {
                re = a / c0;
                im = b / c0;
            }
            w[(int64_t)i * ng + m] = re;
            w[(int64_t)ng * nr + (int64_t)i * ng + m] = im;
        }
    }
#undef GROFU
    free(sig);
    return 0;
}
