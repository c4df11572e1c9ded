/*
 * gx_oracle_sfp.c -- CPU restatement of the SFP (smooth-field-particle)
 * Abel-Jacobi coefficient sum and force evaluation, FP64.
 * TEST INFRASTRUCTURE ONLY (see gx_oracle.h): what the CUDA library's
 * gx_sfp_* entry points are checked against.
 *
 * Follows: ajfun.f:33-47 (basis function), ajder.f:38-101 (its radial
 * derivative), sfptab.f:43-78 (table at nrtab radii), sfpval.f:24-52 (5-point
 * Lagrange interpolation, A&S 25.2.15), sfpadd.f:37-93 (coefficient sums),
 * scaled.f:53-72 (x pmass / maxr^2), sfpacc.f:41-112, 249-259 (forces).
 * Coefficient layout: coeff[n * ngx + m + maxm], ngx = 2 maxm + 1, cosine
 * terms at +m and sine terms at -m (sfpadd.f:80-86).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gx_oracle.h"

#define OX_PI 3.141592653589793238462643

static const double* ox_roots(const GxSfpBasis* b, int m, int n) {
    return b->roots + ((size_t)m * (b->maxn + 1) + n) * b->maxn;
}
static const double* ox_xc(const GxSfpBasis* b, int m, int n) {
    return b->xcoeff + ((size_t)m * (b->maxn + 1) + n) * (b->k + 1);
}

/* pi / sqrt(2.) with sqrt taken in single precision as the reference writes it */
static double ox_ajnorm(void) { return OX_PI / (double)sqrtf(2.0f); }

double ox_ajfun(const GxSfpBasis* b, int m, int n, double r) {
    const double r2 = r * r, x = 1.0 - r2;
    const double* xc = ox_xc(b, m, n);
    const double* rt = ox_roots(b, m, n);
    double f = xc[0];
    for (int i = 1; i <= b->k; i++) f += xc[i] * pow(x, i);
    for (int i = 0; i < n; i++) f *= (r2 - rt[i] * rt[i]);
    if (m > 0) f = pow(r, m) * f;
    return ox_ajnorm() * f;
}

double ox_ajder(const GxSfpBasis* b, int m, int n, double r) {
    const double r2 = r * r, x = 1.0 - r2;
    const double* xc = ox_xc(b, m, n);
    const double* rt = ox_roots(b, m, n);
    double rm = 1.0, rmder = 0.0;
    if (m > 0) {
        rm = pow(r, m);
        rmder = (double)m * pow(r, m - 1);
    }
    double fac = 1.0;
    for (int j = 0; j < n; j++) fac *= (r2 - rt[j] * rt[j]);
    double facder = 0.0;
    for (int j = 0; j < n; j++) {
        double t = 2.0 * r;
        for (int jj = 0; jj < n; jj++)
            if (jj != j) t *= (r2 - rt[jj] * rt[jj]);
        facder += t;
    }
    double xp = xc[0];
    for (int i = 1; i <= b->k; i++) xp += xc[i] * pow(x, i);
    double xpd = 0.0;
    if (b->k > 0) {
        xpd = xc[1];
        for (int i = 2; i <= b->k; i++) xpd += (double)i * xc[i] * pow(x, i - 1);
        xpd = -2.0 * r * xpd;
    }
    return ox_ajnorm() * (rmder * fac * xp + rm * facder * xp + rm * fac * xpd);
}

typedef struct {
    int lastf, ngx, lsfpr;
    int msel[4096], nsel[4096];
    double* tab;   /* [lastf][lsfpr] values */
    double* dtab;  /* [lastf][lsfpr] derivatives */
} ox_sfp;

static void ox_sfp_init(const GxSfpBasis* b, ox_sfp* s) {
    s->lastf = 0;
    for (int m = b->minm; m <= b->maxm; m += b->nsect)
        for (int n = b->minn; n <= b->maxn; n++) {
            s->msel[s->lastf] = m;
            s->nsel[s->lastf] = n;
            s->lastf++;
        }
    s->ngx = 2 * b->maxm + 1;
    s->lsfpr = b->nrtab;
    s->tab = (double*)malloc(sizeof(double) * s->lastf * s->lsfpr);
    s->dtab = (double*)malloc(sizeof(double) * s->lastf * s->lsfpr);
    for (int j = 0; j < s->lastf; j++)
        for (int i = 0; i < s->lsfpr; i++) {
            double r = (double)i / (double)(s->lsfpr - 1);
            s->tab[(size_t)j * s->lsfpr + i] = ox_ajfun(b, s->msel[j], s->nsel[j], r);
            s->dtab[(size_t)j * s->lsfpr + i] = ox_ajder(b, s->msel[j], s->nsel[j], r);
        }
}

static void ox_sfp_free(ox_sfp* s) {
    free(s->tab);
    free(s->dtab);
}

/* sfpval / sfpvld: 5-point Lagrange interpolation in the table at p in [0,1] */
static void ox_sfp_interp(const ox_sfp* s, const double* tab, double p, double* out) {
    p = p * (double)(s->lsfpr - 1);
    int i = (int)p;
    if (i < 2) i = 2;
    if (i > s->lsfpr - 3) i = s->lsfpr - 3;
    p = p - (double)i;
    const double w1 = 1.0 / 24.0, w2 = 1.0 / 6.0, w3 = 0.25;
    const double pm1 = p - 1.0, pm2 = p - 2.0, pp1 = p + 1.0, pp2 = p + 2.0;
    const double ppm1 = p * p - 1.0, ppm4 = p * p - 4.0;
    /* 1-based sfplst(1, i-1 .. i+3) are 0-based entries i-2 .. i+2 */
    for (int j = 0; j < s->lastf; j++) {
        const double* t = tab + (size_t)j * s->lsfpr + (i - 2);
        out[j] = p * ppm1 * (pm2 * t[0] + pp2 * t[4]) * w1 - p * ppm4 * (pm1 * t[1] + pp1 * t[3]) * w2 +
                 ppm1 * ppm4 * t[2] * w3;
    }
}

int ox_sfp_coeffs(const GxSfpBasis* b, int64_t n, const double* pos, int stride, double maxr,
                  double pmass, double* coeff) {
    ox_sfp s;
    ox_sfp_init(b, &s);
    const int ngx = s.ngx, maxm = b->maxm;
    memset(coeff, 0, sizeof(double) * (size_t)(b->maxn + 1) * ngx);
    double* f = (double*)malloc(sizeof(double) * s.lastf);
    double cm[65], sm[65];
    for (int64_t p = 0; p < n; p++) {
        const double x = pos[p * stride], y = pos[p * stride + 1];
        const double r = sqrt(x * x + y * y);
        if (r > maxr) continue;  /* weight.f:425-429: outside the active region */
        if (maxm > 0) {
            cm[1] = r > 0 ? x / r : 1.0;
            sm[1] = r > 0 ? y / r : 0.0;
            for (int m = 2; m <= maxm; m++) {
                cm[m] = cm[m - 1] * cm[1] - sm[m - 1] * sm[1];
                sm[m] = cm[m - 1] * sm[1] + sm[m - 1] * cm[1];
            }
        }
        ox_sfp_interp(&s, s.tab, r / maxr, f);
        for (int j = 0; j < s.lastf; j++) {
            const int m = s.msel[j], nn = s.nsel[j];
            const int k = nn * ngx + maxm;
            if (m == 0) coeff[k] += f[j];
            else {
                coeff[k + m] += f[j] * cm[m];
                coeff[k - m] += f[j] * sm[m];
            }
        }
    }
    const double fac = pmass / (maxr * maxr);
    for (int i = 0; i < (b->maxn + 1) * ngx; i++) coeff[i] *= fac;
    free(f);
    ox_sfp_free(&s);
    return 0;
}

int ox_sfp_acc(const GxSfpBasis* b, const double* coeff, int64_t n, const double* pos, int stride,
               double maxr, double* acc, double* pot) {
    ox_sfp s;
    ox_sfp_init(b, &s);
    const int ngx = s.ngx, maxm = b->maxm;
    double* f = (double*)malloc(sizeof(double) * s.lastf);
    double* d = (double*)malloc(sizeof(double) * s.lastf);
    double cm[65], sm[65];
    for (int64_t p = 0; p < n; p++) {
        const double x = pos[p * stride], y = pos[p * stride + 1];
        double rr = sqrt(x * x + y * y);
        double ar = 0, at = 0, ph = 0;
        if (rr <= maxr) {
            const double r = rr > 1e-5 ? rr : 1e-5;
            cm[1] = x / r;
            sm[1] = y / r;
            for (int m = 2; m <= maxm; m++) {
                cm[m] = cm[m - 1] * cm[1] - sm[m - 1] * sm[1];
                sm[m] = cm[m - 1] * sm[1] + sm[m - 1] * cm[1];
            }
            ox_sfp_interp(&s, s.tab, rr / maxr, f);
            ox_sfp_interp(&s, s.dtab, rr / maxr, d);
            rr = r;
            for (int j = 0; j < s.lastf; j++) {
                const int m = s.msel[j], nn = s.nsel[j];
                const int l = nn * ngx + maxm;
                const double cr = coeff[l + m];
                if (m == 0) {
                    ar += d[j] * cr;
                    ph -= cr * f[j];
                } else {
                    const double ci = coeff[l - m];
                    ar += d[j] * (ci * sm[m] + cr * cm[m]);
                    at += (double)m * f[j] * (ci * cm[m] - cr * sm[m]);
                    ph -= f[j] * (ci * sm[m] + cr * cm[m]);
                }
            }
            at = at * maxr / rr;
            acc[p * 2] = ar * cm[1] - at * sm[1];
            acc[p * 2 + 1] = ar * sm[1] + at * cm[1];
        } else {
            acc[p * 2] = acc[p * 2 + 1] = 0;
        }
        if (pot) pot[p] = ph;
    }
    free(f);
    free(d);
    ox_sfp_free(&s);
    return 0;
}
