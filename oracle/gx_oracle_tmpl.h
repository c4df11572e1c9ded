/*
 * gx_oracle_tmpl.h -- one precision of the CPU restatement (TEST
 * INFRASTRUCTURE ONLY; see gx_oracle.h).  Included by gx_oracle.c with
 *   R   the real type (double or float)
 *   S   the name suffix (f64 or f32)
 *   MIRROR  1 when the reference's FP32 expressions are mirrored
 * Every function cites the reference routine (SRC/lib15/...) it restates.
 */

#define CAT_(a, b) a##_##b
#define CAT(a, b) CAT_(a, b)
#define F(name) CAT(name, S)

/* geometry in the working precision (SRC/lib15/setgrd.f:52-200) */
typedef struct {
    int ndim, nr, na, ngz, nkz, ng, mmax, nsect, mesh, tsoft, rmap, halo;
    int quad; /* 27-point quadratic interpolation (p3d jmass = 3) */
    R alpha, ua, uoffs, rinh, rgrid, zm, thmax, dzg, softl, softl2;
    R halo_v2, halo_rc;
    unsigned char lg[260];
} F(og);

static int F(og_init)(const GxConfig* c, F(og) * g) {
    GxGeometry geo;
    char err[256];
    if (ox_geometry(c, &geo, err, sizeof err)) return GX_ERR_ARG;
    g->ndim = c->ndim;
    g->nr = geo.nr;
    g->na = geo.na;
    g->ngz = geo.ngz;
    g->nkz = (c->ndim == 3) ? geo.ngz + 1 : 1;
    g->ng = geo.ng;
    g->mmax = geo.mmax;
    g->nsect = geo.nsect;
    g->mesh = geo.mesh;
    g->tsoft = c->tsoft;
    g->rmap = c->rmap;
    g->halo = c->halo;
    g->quad = (c->ndim == 3) && (c->flags & GX_FLAG_QUADRATIC);
    memcpy(g->lg, geo.lg, sizeof g->lg);
#if MIRROR
    g->alpha = geo.alpha;
    g->ua = geo.ua;
    g->uoffs = geo.uoffs;
    g->rinh = geo.rinh;
    g->rgrid = geo.rgrid;
    g->zm = geo.zm;
    g->thmax = geo.thmax;
#else
    g->alpha = 2.0 * OX_PI / (double)g->na;
    g->ua = (c->rmap_a > 0.f) ? (double)c->rmap_a : g->alpha;
    g->uoffs = (c->rmap == GX_RMAP_LOG) ? -log((double)c->rmap_r0) / g->ua : 0.0;
    g->thmax = (double)g->na / (double)g->nsect;
    g->zm = 0.5 * (double)c->dzg * (double)(g->ngz - 1);
#endif
    g->dzg = (R)c->dzg;
    g->softl = (R)c->softl;
    g->softl2 = g->softl * g->softl;
    g->halo_v2 = (R)c->halo_v2;
    g->halo_rc = (R)c->halo_rc;
#if !MIRROR
    /* grofu(0) and grofu(nr - 1) in FP64 */
    if (g->rmap == GX_RMAP_STDPOL) {
        g->rinh = 0.0;
        g->rgrid = exp(g->ua * (double)(g->nr - 1)) - 1.0;
    } else {
        g->rinh = exp(g->ua * (0.0 - g->uoffs));
        g->rgrid = exp(g->ua * ((double)(g->nr - 1) - g->uoffs));
    }
#endif
    return 0;
}

/* grofu (SRC/lib15/grofu.f:25-41): stdpol or log-with-hole rule */
static R F(grofu)(const F(og) * g, R u) {
    if (g->rmap == GX_RMAP_STDPOL) return EXP(g->ua * u) - (R)1;
    return EXP(g->ua * (u - g->uoffs));
}

/* uofgr (SRC/lib15/uofgr.f:22-36) */
static R F(uofgr)(const F(og) * g, R r) {
    if (g->rmap == GX_RMAP_STDPOL) return LOG((R)1 + r) / g->ua;
    return LOG(r) / g->ua + g->uoffs;
}

/* ------------------------------------------------------------------ */
/* softened kernels: radfor.f:25-38, azifor.f:25-37, vrtfor.f, grnfun.f,
 * sftpot.f:20-37, softm.f:15-27 (constants as written there)          */
static R F(softm)(R ds) {
    if (ds <= (R)0) return (R)0;
    if (ds < (R)1)
        return (R)4 * ds * ds * ds *
               ((R)0.333333333 - (R)0.3 * ds * ds + (R)0.125 * ds * ds * ds);
    if (ds < (R)2)
        return (R)(-1.0 / 15.0) +
               ds * ds * ds *
                   ((R)2.6666667 - (R)3 * ds + (R)1.2 * ds * ds - (R)0.166666667 * ds * ds * ds);
    return (R)1;
}

static R F(pow15)(R v) { return POW(v, (R)1.5); }

static R F(kernel)(const F(og) * g, int type, R rs, R rf, R th, R zf) {
    R cth = COS(th);
    R d2 = rs * rs + rf * rf - (R)2 * rs * rf * cth + zf * zf;
    if (type == 0) { /* radfor */
        if (g->tsoft == GX_SOFT_PLUMMER) return (rs * cth - rf) / F(pow15)(d2 + g->softl2);
        if (d2 > (R)0) return (rs * cth - rf) * F(softm)(SQRT(d2) / g->softl) / F(pow15)(d2);
        return (R)0;
    }
    if (type == 1) { /* azifor */
        if (g->tsoft == GX_SOFT_PLUMMER) return -rs * SIN(th) / F(pow15)(d2 + g->softl2);
        if (d2 > (R)0) return -rs * SIN(th) * F(softm)(SQRT(d2) / g->softl) / F(pow15)(d2);
        return (R)0;
    }
    if (type == 2) { /* vrtfor */
        if (g->tsoft == GX_SOFT_PLUMMER) return -zf / F(pow15)(d2 + g->softl2);
        if (zf != (R)0) return -zf * F(softm)(SQRT(d2) / g->softl) / F(pow15)(d2);
        return (R)0;
    }
    /* grnfun -> sftpot */
    if (g->tsoft == GX_SOFT_PLUMMER) return (R)-1 / SQRT(d2 + g->softl2);
    {
        R x = SQRT(d2) / g->softl, p;
        if (x <= (R)0) return (R)-1.4 / g->softl;
        if (x < (R)1) {
            p = (R)-1.4 + x * x * ((R)0.6666667 - (R)0.3 * x * x + (R)0.1 * x * x * x);
            return p / g->softl;
        }
        if (x < (R)2) {
            p = (R)-1.6 + (R)1 / ((R)15 * x) +
                x * x * ((R)1.33333333 - x + (R)0.3 * x * x - (R)0.033333333 * x * x * x);
            return p / g->softl;
        }
        return (R)-1 / SQRT(d2);
    }
}

/* ------------------------------------------------------------------ */
/* FFTPACK conventions restated as direct sums (SRC/utils/sfftpack):
 *   rcost(n): X_i = x_1 + (-1)^(i-1) x_n + 2 sum_{k=2}^{n-1} x_k cos((k-1)(i-1) pi/(n-1))
 *   rsint(n): X_i = 2 sum_{k=1}^{n} x_k sin(k i pi/(n+1))
 * twiddles are formed in FP64 and rounded to R.                        */
/* tab[i * n + k] holds the twiddle of output i, input k (rounded to R);
 * only the first nout outputs are formed.                              */
static R* F(cos_tab)(int n) {
    R* t = (R*)malloc(sizeof(R) * n * n);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < n; k++)
            t[i * n + k] = (R)cos((double)k * (double)i * OX_PI / (double)(n - 1));
    return t;
}

static R* F(sin_tab)(int n) {
    R* t = (R*)malloc(sizeof(R) * n * n);
    for (int i = 1; i <= n; i++)
        for (int k = 1; k <= n; k++)
            t[(i - 1) * n + (k - 1)] = (R)sin((double)k * (double)i * OX_PI / (double)(n + 1));
    return t;
}

static void F(rcost)(int n, const R* x, R* X, const R* tab, int nout) {
    for (int i = 0; i < nout; i++) {
        R s = x[0] + ((i & 1) ? -x[n - 1] : x[n - 1]);
        const R* tr = tab + (int64_t)i * n;
        for (int k = 1; k < n - 1; k++) s += (R)2 * x[k] * tr[k];
        X[i] = s;
    }
}

static void F(rsint)(int n, const R* x, R* X, const R* tab, int nout) {
    for (int i = 0; i < nout; i++) {
        R s = 0;
        const R* tr = tab + (int64_t)i * n;
        for (int k = 0; k < n; k++) s += (R)2 * x[k] * tr[k];
        X[i] = s;
    }
}

/* ------------------------------------------------------------------ */
/* Green table: p2grnm.f:99-203 / p2gwrt.f:34-52 (2D) and
 * p3grnm.f:94-263 / p3gwrt.f:47-64 (3D).  G is [4][ng][nkz][is][ir];
 * D (optional) is the direct, harmonic-filtered table used by the force
 * check, [4][is][ir][nkz][na/2 + 1].                                    */
int F(ox_green)(const GxConfig* c, R* G, R* D) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int nr = g.nr, na = g.na, ngz = g.ngz, nkz = g.nkz, ng = g.ng, mmax = g.mmax;
    const int nth = na / 2 + 1;
    const int64_t gsz = (int64_t)4 * ng * nkz * nr * nr;
    memset(G, 0, sizeof(R) * gsz);
    if (D) memset(D, 0, sizeof(R) * (int64_t)4 * nr * nr * nkz * nth);
    const int T = ox_threads;
    R* f_all = (R*)malloc(sizeof(R) * nth * (nkz + 1) * T);
    R* tr_all = (R*)malloc(sizeof(R) * nth * (nkz + 1) * T);
    R* zb_all = (R*)malloc(sizeof(R) * (nkz + 1) * T);
    R* zt_all = (R*)malloc(sizeof(R) * (nkz + 1) * T);
    R* back_all = (R*)malloc(sizeof(R) * nth * T);
    R* ctab = F(cos_tab)(na / 2 + 1);
    R* stab = F(sin_tab)(na / 2 - 1);
    R* zctab = (g.ndim == 3) ? F(cos_tab)(ngz + 1) : NULL;
    R* zstab = (g.ndim == 3) ? F(sin_tab)(ngz - 1) : NULL;
    for (int type = 0; type < 4; type++) {
        if (g.ndim == 2 && type == 2) continue;
        if (type == 1 && ng == 1) continue;
        const int azim = (type == 1), vert = (type == 2);
        const int it1 = azim ? 2 : 1, it2 = azim ? mmax - 1 : mmax;
        const int nt = it2 - it1 + 1;
        const int iz1 = vert ? 2 : 1, iz2 = (g.ndim == 3) ? (vert ? ngz : ngz + 1) : 1;
        const int nz = iz2 - iz1 + 1;
#pragma omp parallel for schedule(dynamic) num_threads(T) if (T > 1)
        for (int is = 0; is < nr; is++) {
            const int tid = OX_TID;
            R* f = f_all + (size_t)tid * nth * (nkz + 1);
            R* tr = tr_all + (size_t)tid * nth * (nkz + 1);
            R* zb = zb_all + (size_t)tid * (nkz + 1);
            R* zt = zt_all + (size_t)tid * (nkz + 1);
            R* back = back_all + (size_t)tid * nth;
            R rs = F(grofu)(&g, (R)is);
            for (int ir = 0; ir < nr; ir++) {
                R rf = F(grofu)(&g, (R)ir);
                for (int iz = iz1; iz <= iz2; iz++) {
                    R zf = (g.ndim == 3) ? g.dzg * (R)(iz - 1) : (R)0;
                    for (int it = it1; it <= it2; it++) {
                        R th;
#if MIRROR
                        if (g.ndim == 3) th = g.alpha * (R)(it - 1);
                        else th = (R)(2.0 * OX_PI * (double)(R)(it - 1) / (double)(R)na);
#else
                        th = 2.0 * OX_PI * (double)(it - 1) / (double)na;
#endif
                        f[(iz - iz1) * nt + (it - it1)] = F(kernel)(&g, type, rs, rf, th, zf);
                    }
                    /* angular transform, filter */
                    R* fr = f + (iz - iz1) * nt;
                    R* tt = tr + (iz - iz1) * nt;
                    /* harmonics m >= ng are filtered out: form only m < ng */
                    int nout = azim ? ((ng - 1 < nt) ? ng - 1 : nt) : ((ng < nt) ? ng : nt);
                    for (int it = it1; it <= it2; it++) tt[it - it1] = 0;
                    if (nout > 0) {
                        if (azim) F(rsint)(nt, fr, tt, stab, nout);
                        else F(rcost)(nt, fr, tt, ctab, nout);
                    }
                    for (int it = it1; it <= it2; it++) {
                        int m = it - 1;
                        int drop = (m >= ng);
                        if (g.ndim == 2) drop = drop || (m % g.nsect != 0);
                        else drop = drop || g.lg[m];
                        if (drop) tt[it - it1] = 0;
                    }
                    if (D) {
                        /* re-synthesised direct table (filtered), x 1/na */
                        if (azim) F(rsint)(nt, tt, back, stab, nt);
                        else F(rcost)(nt, tt, back, ctab, nt);
                        R* d = D + ((((int64_t)type * nr + is) * nr + ir) * nkz + (iz - 1)) * nth;
                        for (int it = it1; it <= it2; it++)
                            d[it - 1] = back[it - it1] * ((R)1 / (R)na);
                    }
                }
                /* vertical transform per harmonic (3D), store */
                for (int it = it1; it <= it2; it++) {
                    int m = it - 1;
                    if (m >= ng) continue;
                    if (g.ndim == 2) {
                        G[((((int64_t)type * ng + m) * nkz + 0) * nr + is) * nr + ir] = tr[it - it1];
                        continue;
                    }
                    for (int iz = iz1; iz <= iz2; iz++) zb[iz - iz1] = tr[(iz - iz1) * nt + (it - it1)];
                    if (vert) F(rsint)(nz, zb, zt, zstab, nz);
                    else F(rcost)(nz, zb, zt, zctab, nz);
                    for (int iz = iz1; iz <= iz2; iz++) {
                        int kz = iz - 1;
                        G[((((int64_t)type * ng + m) * nkz + kz) * nr + is) * nr + ir] = zt[iz - iz1];
                    }
                }
            }
        }
    }
    free(f_all);
    free(tr_all);
    free(zb_all);
    free(zt_all);
    free(back_all);
    free(ctab);
    free(stab);
    free(zctab);
    free(zstab);
    return 0;
}

/* ------------------------------------------------------------------ */
/* quadratic (27-point) weights of p3d, jmass = 3 (weight.f:280-311): the
 * central cell is the nearest node, (ju, jz, jt) = int(u + .5, z + .5,
 * t + .5), ju clamped to [1, nr - 2], jz to [0, ngz - 2], jt = na wrapping
 * to 0 in the key; per axis dd = coord + .5 - index and the factors
 * (1 - 2dd + dd^2, 1 + 2dd - 2dd^2, dd^2); weight l (theta fastest, then z,
 * then u) = .125 f_theta f_z f_u.                                        */
static int F(weight27)(const F(og) * gp, R u, R t, R z, int32_t* keyp, R* w) {
    R zz = (z + gp->zm) / gp->dzg;
    R uh = u + (R)0.5, th = t + (R)0.5, zh = zz + (R)0.5;
    int ju = (int)uh;
    if (ju > gp->nr - 2) ju = gp->nr - 2;
    if (ju < 1) ju = 1;
    int jt = (int)th;
    int jz = (int)zh;
    if (jz < 0) jz = 0;
    if (jz > gp->ngz - 2) jz = gp->ngz - 2;
    int ncl = (ju * gp->ngz + jz) * gp->na + jt;
    if (jt == gp->na) ncl -= gp->na;
    *keyp = ncl;
    R dp[3][3];
    for (int i = 0; i < 3; i++) {
        R dd = (i == 0) ? th - (R)jt : (i == 1) ? zh - (R)jz : uh - (R)ju;
        dp[i][0] = (R)1 - (R)2 * dd + dd * dd;
        dp[i][1] = (R)1 + (R)2 * dd - (R)2 * (dd * dd);
        dp[i][2] = dd * dd;
    }
    int l = 0;
    for (int k = 0; k < 3; k++)
        for (int j = 0; j < 3; j++)
            for (int i = 0; i < 3; i++) w[l++] = (R)0.125 * dp[0][i] * dp[1][j] * dp[2][k];
    return 1;
}

/* ------------------------------------------------------------------ */
/* weight (SRC/lib15/weight.f:61-101 p2d, 196-250 p3d linear) together
 * with the off-grid test of offgrd.f:51-77.  key = ncl - 1 or -1.      */
static int F(weight1)(const F(og) * gp, int old, const R* q, int32_t* keyp, R* w) {
    const int nd = gp->ndim;
    R x = q[0], y = q[1], z = (nd == 3) ? q[2] : (R)0;
    for (int k = 0; k < (gp->quad ? 27 : 8); k++) w[k] = 0;
    *keyp = -1;
    R rr = SQRT(x * x + y * y);
    if (rr > gp->rgrid) return 0;
    if (nd == 3 && FABS(z) > gp->zm) return 0;
    R u = F(uofgr)(gp, rr);
    R t;
    if (nd == 2 || rr > (R)0) {
#if MIRROR
        t = (R)(atan2((double)y, (double)x) * (double)gp->na / (2.0 * OX_PI));
#else
        t = atan2(y, x) * (double)gp->na / (2.0 * OX_PI);
#endif
        if (t < (R)0) t = t + (R)gp->na;
    } else {
        t = 0;
    }
    if (!old && gp->nsect > 1) t = FMOD(t, gp->thmax);
    if (rr < gp->rinh) return 0;
    if (gp->quad) return F(weight27)(gp, u, t, z, keyp, w);
    int ju = (int)u;
    if (ju > gp->nr - 2) ju = gp->nr - 2;
    int jt = (int)t;
    R du = u - (R)ju, dt = t - (R)jt;
    if (nd == 2) {
        *keyp = ju * gp->na + jt;
        R dd = du * dt;
        w[0] = (R)1 - du - dt + dd;
        w[1] = dt - dd;
        w[2] = du - dd;
        w[3] = dd;
    } else {
        R zz = z + gp->zm;
        zz = zz / gp->dzg;
        int jz = (int)zz;
        if (jz < 0) jz = 0;
        if (jz > gp->ngz - 2) jz = gp->ngz - 2;
        *keyp = (ju * gp->ngz + jz) * gp->na + jt;
        R dz = zz - (R)jz;
        w[0] = ((R)1 - dt) * ((R)1 - dz) * ((R)1 - du);
        w[1] = dt * ((R)1 - dz) * ((R)1 - du);
        w[2] = ((R)1 - dt) * dz * ((R)1 - du);
        w[3] = dt * dz * ((R)1 - du);
        w[4] = ((R)1 - dt) * ((R)1 - dz) * du;
        w[5] = dt * ((R)1 - dz) * du;
        w[6] = ((R)1 - dt) * dz * du;
        w[7] = dt * dz * du;
    }
    return 1;
}

int F(ox_weight)(const GxConfig* c, int old, int64_t n, const R* pos, int32_t* key,
                 R* wt, uint8_t* on) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int stride = 2 * g.ndim;
#pragma omp parallel for schedule(static) num_threads(ox_threads) if (ox_threads > 1)
    for (int64_t p = 0; p < n; p++)
        on[p] = (uint8_t)F(weight1)(&g, old, pos + p * stride, key + p,
                                     wt + p * (g.quad ? 27 : 8));
    return 0;
}

/* cell corners of a key: grdacc.f:193-202 (ic(1..8)) / massgn.f:155-170.
 * Corners outside the mesh (the reference writes past the array there)
 * are returned as -1.                                                   */
static int F(corners)(const F(og) * g, int32_t key, int32_t* ic) {
    const int na = g->na;
    if (g->quad) {
        /* massgn.f:180-193 / grdacc.f:271-283: the 3 x 3 x 3 nodes around
         * the central one, theta wrapping, planes and rings by flat offsets */
        const int c0 = key, tm = (key % na == 0) ? key - 1 + na : key - 1;
        const int tp = ((key + 1) % na == 0) ? key + 1 - na : key + 1;
        const int mid[3] = {tm, c0, tp};
        const int pl = g->ngz * na;
        int l = 0;
        for (int k = -1; k <= 1; k++)
            for (int j = -1; j <= 1; j++)
                for (int i = 0; i < 3; i++) {
                    int v = mid[i] + j * na + k * pl;
                    ic[l++] = (v < 0 || v >= g->mesh) ? -1 : v;
                }
        return 27;
    }
    int end = ((key + 1) % na) == 0;
    ic[0] = key;
    ic[1] = key + 1 - (end ? na : 0);
    ic[2] = key + na;
    ic[3] = ic[1] + na;
    if (g->ndim == 2) {
        for (int k = 0; k < 4; k++)
            if (ic[k] >= g->mesh) ic[k] = -1;
        return 4;
    }
    const int pl = g->ngz * na;
    ic[4] = key + pl;
    ic[5] = ic[1] + pl;
    ic[6] = ic[4] + na;
    ic[7] = ic[5] + na;
    for (int k = 0; k < 8; k++)
        if (ic[k] >= g->mesh) ic[k] = -1;
    return 8;
}

/* massgn (SRC/lib15/massgn.f:68-89 p2d, 140-172 p3d): accumulate, and
 * track the 1-based active ring range jrk = {jrad, krad}.                */
int F(ox_massgn)(const GxConfig* c, int64_t n, const int32_t* key, const R* wt,
                 const uint8_t* on, R* mass, int32_t* jrk) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int div = (g.ndim == 2) ? g.na : g.na * g.ngz;
    /* reference update order: w1, w3, w2, w4 (, w5, w7, w6, w8) */
    static const int ord4[4] = {0, 2, 1, 3};
    static const int ord8[8] = {0, 2, 1, 3, 4, 6, 5, 7};
    const int nt = ox_threads;
    /* threaded: each thread deposits a contiguous block of particles into
     * its own array; the arrays are summed in thread order */
    R* priv = (nt > 1) ? (R*)calloc((size_t)nt * g.mesh, sizeof(R)) : NULL;
    int32_t jlo[256], khi[256];
    for (int t = 0; t < nt && t < 256; t++) {
        jlo[t] = jrk[0];
        khi[t] = jrk[1];
    }
#pragma omp parallel num_threads(nt) if (nt > 1)
    {
        const int tid = OX_TID;
        R* dst = priv ? priv + (size_t)tid * g.mesh : mass;
        int64_t p0 = n * tid / nt, p1 = n * (tid + 1) / nt;
        int32_t ic[27];
        for (int64_t p = p0; p < p1; p++) {
            if (!on[p]) continue;
            int j = key[p] / div;
            /* quadratic: jrad = j (massgn.f:180) */
            const int jl = g.quad ? j : j + 1;
            if (jl < jlo[tid]) jlo[tid] = jl;
            if (j + 2 > khi[tid]) khi[tid] = j + 2;
            int nc = F(corners)(&g, key[p], ic);
            if (g.quad) {
                const R* w = wt + p * 27;
                for (int k = 0; k < 27; k++)
                    if (ic[k] >= 0) dst[ic[k]] += w[k];
                continue;
            }
            const R* w = wt + p * 8;
            const int* ord = (nc == 4) ? ord4 : ord8;
            for (int k = 0; k < nc; k++) {
                int cidx = ic[ord[k]];
                if (cidx >= 0) dst[cidx] += w[ord[k]];
            }
        }
    }
    for (int t = 0; t < nt; t++) {
        if (jlo[t] < jrk[0]) jrk[0] = jlo[t];
        if (khi[t] > jrk[1]) jrk[1] = khi[t];
    }
    if (priv) {
#pragma omp parallel for schedule(static) num_threads(nt)
        for (int64_t i = 0; i < g.mesh; i++) {
            R v = mass[i];
            for (int t = 0; t < nt; t++) v += priv[(size_t)t * g.mesh + i];
            mass[i] = v;
        }
        free(priv);
    }
    return 0;
}

/* masset: masscl + massgn over all particles + scaled (masset.f,
 * scaled.f:89-92) */
int F(ox_masset)(const GxConfig* c, int64_t n, const R* pos, R* mass, int32_t* jrk) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    int32_t* key = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    R* wt = (R*)malloc(sizeof(R) * 27 * (n ? n : 1));
    uint8_t* on = (uint8_t*)malloc(n ? n : 1);
    memset(mass, 0, sizeof(R) * g.mesh);
    jrk[0] = g.nr;
    jrk[1] = 0;
    F(ox_weight)(c, 0, n, pos, key, wt, on);
    F(ox_massgn)(c, n, key, wt, on, mass, jrk);
    R pm = (R)c->pmass;
    for (int i = 0; i < g.mesh; i++) mass[i] = mass[i] * pm;
    free(key);
    free(wt);
    free(on);
    return 0;
}

/* ------------------------------------------------------------------ */
/* field solve: p2fndf.f:25-66 (p2manl, p2conv, p2fsyn) and
 * p3fndf.f:36-104 (p3manl, p3conv, p3fsyn).  fields is [4][mesh]:
 * radial, azimuthal, vertical, potential, polar components.
 * Spectral scratch per ring: [m][part][kz], part 0 Aa 1 Ba 2 Ab 3 Bb
 * (a/b = azimuthal cos/sin row, A/B = vertical cos/sin part).           */
int F(ox_findf)(const GxConfig* c, const R* G, const R* mass, int lpot, int jrs, int krs,
                R* fields) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int nr = g.nr, na = g.na, ngz = g.ngz, ng = g.ng, nkz = g.nkz, mmax = g.mmax;
    const int nd = g.ndim;
    const int64_t mesh = g.mesh;
    memset(fields, 0, sizeof(R) * 4 * mesh);
    if (jrs < 1) jrs = 1;
    if (krs > nr) krs = nr;
    if (jrs > krs) return GX_ERR_STATE;
    const int ntypes = (nd == 3) ? (lpot ? 4 : 3) : (lpot ? 3 : 2);
    const int nspec = ng * 4 * nkz; /* per ring */
    R* spec = (R*)calloc((size_t)nr * nspec, sizeof(R));
    R* outs = (R*)calloc((size_t)nr * nspec, sizeof(R));
    R* row = (R*)malloc(sizeof(R) * (na > 2 * ngz ? na : 2 * ngz) * 2);
    /* per-thread a_m(z), b_m(z) scratch */
    R* ca_all = (R*)malloc(sizeof(R) * ngz * ng * ox_threads);
    R* cb_all = (R*)malloc(sizeof(R) * ngz * ng * ox_threads);
    /* twiddles formed in FP64, rounded to R: azimuth [m][j], vertical [k][z] */
    R* acos_ = (R*)malloc(sizeof(R) * ng * na);
    R* asin_ = (R*)malloc(sizeof(R) * ng * na);
    R* zcos_ = (R*)malloc(sizeof(R) * (ngz + 1) * ngz);
    R* zsin_ = (R*)malloc(sizeof(R) * (ngz + 1) * ngz);
    for (int m = 0; m < ng; m++)
        for (int j = 0; j < na; j++) {
            double ang = 2.0 * OX_PI * (double)m * (double)j / (double)na;
            acos_[m * na + j] = (R)cos(ang);
            asin_[m * na + j] = (R)sin(ang);
        }
    for (int k = 0; k <= ngz; k++)
        for (int z = 0; z < ngz; z++) {
            double ang = OX_PI * (double)k * (double)z / (double)ngz;
            zcos_[k * ngz + z] = (R)cos(ang);
            zsin_[k * ngz + z] = (R)sin(ang);
        }
#define SP(buf, ir, m, part, kz) buf[(((int64_t)(ir) * ng + (m)) * 4 + (part)) * nkz + (kz)]
    /* forward transforms of the active source rings */
#pragma omp parallel for schedule(dynamic) num_threads(ox_threads) if (ox_threads > 1)
    for (int ir = jrs - 1; ir < krs; ir++) {
        R* ca = ca_all + (size_t)OX_TID * ngz * ng;
        R* cb = cb_all + (size_t)OX_TID * ngz * ng;
        for (int iz = 0; iz < ngz; iz++) {
            const R* x = mass + ((int64_t)ir * ngz + iz) * na;
            for (int m = 0; m < ng; m++) {
                if (g.lg[m]) continue;
                R a = 0, b = 0;
                for (int j = 0; j < na; j++) {
                    a += x[j] * acos_[m * na + j];
                    b -= x[j] * asin_[m * na + j];
                }
                ca[iz * ng + m] = a;
                cb[iz * ng + m] = b;
            }
        }
        for (int m = 0; m < ng; m++) {
            if (g.lg[m]) continue;
            const int hasb = (m > 0 && m < mmax - 1);
            for (int ab = 0; ab < 2; ab++) {
                if (ab == 1 && !hasb) continue;
                const R* src = ab ? cb : ca;
                if (nd == 2) {
                    SP(spec, ir, m, 2 * ab, 0) = src[m];
                    continue;
                }
                /* zero-padded vertical FFT of length 2 ngz (p3manl.f:72-105) */
                for (int k = 0; k <= ngz; k++) {
                    R A = 0, B = 0;
                    for (int z = 0; z < ngz; z++) {
                        A += src[z * ng + m] * zcos_[k * ngz + z];
                        B -= src[z * ng + m] * zsin_[k * ngz + z];
                    }
                    SP(spec, ir, m, 2 * ab, k) = A;
                    SP(spec, ir, m, 2 * ab + 1, k) = B;
                }
            }
        }
    }
    for (int tt = 0; tt < ntypes; tt++) {
        int type = tt;
        if (nd == 2 && tt == 2) type = 3;
        R* fout = fields + (int64_t)type * mesh;
        if (type == 1 && ng == 1) continue; /* p3fndf.f:80-84 */
        memset(outs, 0, sizeof(R) * (size_t)nr * nspec);
        /* radial convolution (p2conv.f:114-181 / p3conv.f:137-230) */
        int mlo = 0, mhi = ng - 1;
        if (type == 1) {
            mlo = 1;
            mhi = ((ng < mmax - 1) ? ng : mmax - 1) - 1;
        }
        int klo = 0, khi = (nd == 3) ? ngz : 0;
        if (type == 2) {
            klo = 1;
            khi = ngz - 1;
        }
        for (int m = mlo; m <= mhi; m++) {
            if (g.lg[m]) continue;
            const int naskip = (m > 0 && m < mmax - 1);
            for (int kz = klo; kz <= khi; kz++) {
                const int nvskip = (nd == 3) && (kz > 0 && kz < ngz);
                const R* Gm = G + ((((int64_t)type * ng + m) * nkz + kz) * nr) * nr;
#pragma omp parallel for schedule(static) num_threads(ox_threads) if (ox_threads > 1)
                for (int ir = 0; ir < nr; ir++) {
                    R oAa = 0, oBa = 0, oAb = 0, oBb = 0;
                    for (int is = jrs - 1; is < krs; is++) {
                        R gv = Gm[(int64_t)is * nr + ir];
                        R iAa = SP(spec, is, m, 0, kz), iBa = SP(spec, is, m, 1, kz);
                        R iAb = SP(spec, is, m, 2, kz), iBb = SP(spec, is, m, 3, kz);
                        if (type == 0 || type == 3) {
                            oAa += gv * iAa;
                            if (naskip) oAb += gv * iAb;
                            if (nvskip) {
                                oBa += gv * iBa;
                                if (naskip) oBb += gv * iBb;
                            }
                        } else if (type == 1) {
                            oAa += gv * iAb;
                            oAb -= gv * iAa;
                            if (nvskip) {
                                oBa += gv * iBb;
                                oBb -= gv * iBa;
                            }
                        } else {
                            oAa += gv * iBa;
                            oBa -= gv * iAa;
                            if (naskip) {
                                oAb += gv * iBb;
                                oBb -= gv * iAb;
                            }
                        }
                    }
                    SP(outs, ir, m, 0, kz) = oAa;
                    SP(outs, ir, m, 1, kz) = oBa;
                    SP(outs, ir, m, 2, kz) = oAb;
                    SP(outs, ir, m, 3, kz) = oBb;
                }
            }
        }
        /* synthesis (p2fsyn.f:42-53 / p3fsyn.f:59-129) */
        const R scale = (nd == 3) ? (R)1 / (R)(2 * ngz * na) : (R)1 / (R)na;
#pragma omp parallel for schedule(dynamic) num_threads(ox_threads) if (ox_threads > 1)
        for (int ir = 0; ir < nr; ir++) {
            R* ca = ca_all + (size_t)OX_TID * ngz * ng;
            R* cb = cb_all + (size_t)OX_TID * ngz * ng;
            /* vertical synthesis of each active row */
            for (int m = 0; m < ng; m++) {
                if (g.lg[m]) continue;
                for (int ab = 0; ab < 2; ab++) {
                    R* dst = ab ? cb : ca;
                    if (nd == 2) {
                        dst[m] = SP(outs, ir, m, 2 * ab, 0);
                        continue;
                    }
                    for (int z = 0; z < ngz; z++) {
                        R s = SP(outs, ir, m, 2 * ab, 0) +
                              ((z & 1) ? -SP(outs, ir, m, 2 * ab, ngz) : SP(outs, ir, m, 2 * ab, ngz));
                        for (int k = 1; k < ngz; k++)
                            s += (R)2 * (SP(outs, ir, m, 2 * ab, k) * zcos_[k * ngz + z] -
                                         SP(outs, ir, m, 2 * ab + 1, k) * zsin_[k * ngz + z]);
                        dst[z * ng + m] = s;
                    }
                }
            }
            /* azimuthal synthesis of each plane */
            for (int iz = 0; iz < ngz; iz++) {
                R* y = fout + ((int64_t)ir * ngz + iz) * na;
                for (int j = 0; j < na; j++) {
                    R s = 0;
                    for (int m = 0; m < ng; m++) {
                        if (g.lg[m]) continue;
                        R a = ca[iz * ng + m];
                        if (m == 0) s += a;
                        else if (m == mmax - 1) s += (j & 1) ? -a : a;
                        else s += (R)2 * (a * acos_[m * na + j] - cb[iz * ng + m] * asin_[m * na + j]);
                    }
                    y[j] = scale * s;
                }
            }
        }
    }
#undef SP
    free(spec);
    free(outs);
    free(row);
    free(ca_all);
    free(cb_all);
    free(acos_);
    free(asin_);
    free(zcos_);
    free(zsin_);
    return 0;
}

/* polcat (SRC/lib15/polcat.f:22-41): (fr, ft) -> (fx, fy) in place */
int F(ox_polcat)(const GxConfig* c, R* fields) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int64_t mesh = g.mesh;
    const int nrow = g.nr * g.ngz;
    for (int j = 0; j < g.na; j++) {
#if MIRROR
        R t = (R)(2.0 * OX_PI * (double)(R)j / (double)(R)g.na);
#else
        R t = 2.0 * OX_PI * (double)j / (double)g.na;
#endif
        R cp = COS(t), sp = SIN(t);
        for (int i = 0; i < nrow; i++) {
            int64_t l = (int64_t)i * g.na + j;
            R fr = fields[l], ft = fields[mesh + l];
            fields[l] = fr * cp - ft * sp;
            fields[mesh + l] = fr * sp + ft * cp;
        }
    }
    return 0;
}

/* getacc/grdacc (SRC/lib15/getacc.f:36-162, grdacc.f:40-84, 189-266)
 * for particles at pos; fields hold Cartesian components after polcat.
 * acc is AoS ndim per particle; pot may be NULL.                        */
int F(ox_grdacc)(const GxConfig* c, int64_t n, const R* pos, const R* fields, int phys,
                 R* acc, R* pot) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int nd = g.ndim, stride = 2 * nd;
    const int64_t mesh = g.mesh;
#pragma omp parallel for schedule(static) num_threads(ox_threads) if (ox_threads > 1)
    for (int64_t p = 0; p < n; p++) {
        const R* q = pos + p * stride;
        R a[3] = {0, 0, 0}, ph = 0;
        int32_t key;
        R w[27];
        int32_t ic[27];
        int on = F(weight1)(&g, 1, q, &key, w);
        if (on) {
            int nc = F(corners)(&g, key, ic);
            for (int i = 0; i < nd; i++) {
                /* fields 0, 1 are fx, fy; 2 is fz */
                const R* fi = fields + (int64_t)i * mesh;
                for (int k = 0; k < nc; k++)
                    if (ic[k] >= 0) a[i] = a[i] + fi[ic[k]] * w[k];
            }
            if (phys) {
                const R* fp = fields + 3 * mesh;
                for (int k = 0; k < nc; k++)
                    if (ic[k] >= 0) ph = ph + fp[ic[k]] * w[k];
            }
            /* rigid halo, ISOT: frhalo.f:55-56, halfrc.f:30-60 */
            if (g.halo == 1) {
                R rr = 0;
                for (int i = 0; i < nd; i++) rr = rr + q[i] * q[i];
                rr = SQRT(rr);
                R fr = -g.halo_v2 * rr / (rr * rr + g.halo_rc * g.halo_rc);
                if (fr != (R)0) {
                    fr = fr / rr;
                    for (int i = 0; i < nd; i++) a[i] = a[i] + fr * q[i];
                }
                if (phys)
                    ph = ph + (R)0.5 * g.halo_v2 * LOG((R)1 + rr * rr / (g.halo_rc * g.halo_rc));
            }
            /* fixed axisymmetric force of a softened Kuz'min-Toomre disc
             * (the 'skip 0' card: getacc.f:118-121, axifrc.f, frdisc.f:27-29):
             * F(r) = -K r / (r^2 + Rs^2)^1.5, K = halo_v2, Rs = halo_rc;
             * potential -K / sqrt(r^2 + Rs^2) */
            if (g.halo == 2) {
                R r2 = 0;
                for (int i = 0; i < nd; i++) r2 = r2 + q[i] * q[i];
                const R d = r2 + g.halo_rc * g.halo_rc;
                const R sd = SQRT(d);
                const R fr = -g.halo_v2 / (d * sd);
                for (int i = 0; i < nd; i++) a[i] = a[i] + fr * q[i];
                if (phys) ph = ph - g.halo_v2 / sd;
            }
        }
        for (int i = 0; i < nd; i++) acc[p * nd + i] = a[i];
        if (pot) pot[p] = ph;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* galaxy main loop restated: nsteps x { findf; getacc; stpgrp; massgn;
 * scaled } (SRC/progs/galaxy.f:107-148, SRC/lib15/step.f:135-290,
 * stpgrp.f:26-32).  mass holds the scaled mass of the current positions
 * on entry and of the final positions on exit; fields (optional,
 * [4][mesh]) receive the Cartesian fields of the last solve.            */
int F(ox_step)(const GxConfig* c, const R* G, int64_t n, R* pos, R* mass, int32_t* jrk,
               int nsteps, int phys, R* fields) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int nd = g.ndim, stride = 2 * nd;
    R* fl = fields ? fields : (R*)malloc(sizeof(R) * 4 * (size_t)g.mesh);
    R* acc = (R*)malloc(sizeof(R) * nd * (n ? n : 1));
    for (int s = 0; s < nsteps; s++) {
        int lpot = phys && (s == nsteps - 1);
        F(ox_findf)(c, G, mass, lpot, jrk[0], jrk[1], fl);
        F(ox_polcat)(c, fl);
        F(ox_grdacc)(c, n, pos, fl, 0, acc, NULL);
#pragma omp parallel for schedule(static) num_threads(ox_threads) if (ox_threads > 1)
        for (int64_t p = 0; p < n; p++) {
            R* q = pos + p * stride;
            for (int i = 0; i < nd; i++) {
                q[nd + i] = q[nd + i] + acc[p * nd + i];
                q[i] = q[i] + q[nd + i];
            }
        }
        F(ox_masset)(c, n, pos, mass, jrk);
    }
    free(acc);
    if (!fields) free(fl);
    return 0;
}

/* the particle loop of step (SRC/lib15/step.f:186-242) for one step over
 * pos with given Cartesian fields: getacc, stpgrp, then massgn + scaled of
 * the new positions into mass (zeroed here) */
int F(ox_particle_pass)(const GxConfig* c, int64_t n, R* pos, const R* fields, R* mass,
                        int32_t* jrk) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int nd = g.ndim, stride = 2 * nd;
    R* acc = (R*)malloc(sizeof(R) * nd * (n ? n : 1));
    F(ox_grdacc)(c, n, pos, fields, 0, acc, NULL);
#pragma omp parallel for schedule(static) num_threads(ox_threads) if (ox_threads > 1)
    for (int64_t p = 0; p < n; p++) {
        R* q = pos + p * stride;
        for (int i = 0; i < nd; i++) {
            q[nd + i] = q[nd + i] + acc[p * nd + i];
            q[i] = q[i] + q[nd + i];
        }
    }
    free(acc);
    return F(ox_masset)(c, n, pos, mass, jrk);
}

/* ------------------------------------------------------------------ */
/* direct convolution with the filtered direct Green table for point
 * masses on mesh nodes (SRC/lib15/p3chkf.f:45-165, p2chkf.f:82-149).
 * mr, mt, mz are 1-based ring, spoke, plane; fields is [4][mesh] polar. */
int F(ox_direct_field)(const GxConfig* c, const R* D, int nmass, const int32_t* mr,
                       const int32_t* mt, const int32_t* mz, const R* mm, int lpot,
                       R* fields) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int nr = g.nr, na = g.na, ngz = g.ngz, nkz = g.nkz, nth = na / 2 + 1;
    const int64_t mesh = g.mesh;
    memset(fields, 0, sizeof(R) * 4 * mesh);
    const int nd = g.ndim;
    for (int type = 0; type < 4; type++) {
        if (nd == 2 && type == 2) continue;
        if (type == 3 && !lpot) continue;
        if (type == 1 && g.ng == 1) continue;
        const R sgna = (type == 1) ? (R)-1 : (R)1;
        const R sgnv = (type == 2) ? (R)-1 : (R)1;
        R* fo = fields + (int64_t)type * mesh;
        for (int n = 0; n < nmass; n++) {
            int is = mr[n] - 1, t0 = mt[n] - 1, z0 = mz[n] - 1;
            for (int ir = 0; ir < nr; ir++) {
                for (int iz = 0; iz < ngz; iz++) {
                    int dz = iz - z0;
                    int jz = dz < 0 ? -dz : dz;
                    if (nd == 3 && type == 2 && jz == 0) continue;
                    if (jz >= nkz) continue;
                    R sz = (dz < 0) ? sgnv : (R)1;
                    const R* d = D + ((((int64_t)type * nr + is) * nr + ir) * nkz + jz) * nth;
                    for (int it = 0; it < na; it++) {
                        int dt = ((it - t0) % na + na) % na;
                        R v;
                        if (dt <= na / 2) v = d[dt];
                        else v = sgna * d[na - dt];
                        if (type == 1 && (dt == 0 || dt == na / 2)) v = 0;
                        fo[((int64_t)ir * ngz + iz) * na + it] += mm[n] * sz * v;
                    }
                }
            }
        }
    }
    return 0;
}

#undef F
#undef CAT
#undef CAT_
