/*
 * gx_oracle_zone.h -- multiple time-step zones of the polar-grid step, FP64
 * (TEST INFRASTRUCTURE ONLY; see gx_oracle.h).  Included by gx_oracle.c
 * inside the FP64 instantiation of gx_oracle_tmpl.h (R = double, suffix f64).
 *
 * Restates, for the p2d/p3d grid with one grid and no guard zones:
 *   zoneno.f      zone of a position: the largest i with rad >= zbr(i)
 *                 (cylindrical radius in 2D, spherical in 3D: setrun.f:810)
 *   tsfac.f       time-step factor nstep(min(iz, nzones)) of a zone
 *   adjvls.f      velocities in units of the zone's step (lists 1..nlists-1)
 *   masscl.f:31-96  the step number of each new mass array, the older copy
 *   zoncmb.f:46-129 mzone of the next step; zone 1's array += the linear
 *                 interpolation in time of the other zones' arrays
 *   p2fndf.f:25-33  source ring range over all zones (krad running max)
 *   step.f:135-292  zones 1..mzone step; off-grid particles (list nlists)
 *                 step with the outermost zone when mzone = nzones (the
 *                 'offgrid' analysis switch) and feel no force
 *   getacc.f:141-150 accelerations x tsfac^2
 *   stpgrp.f:26-57  leapfrog; particles returning to the grid join zone nzones
 *   addoff.f:44-52  a particle leaving the grid moves to the outermost
 *                 zone's step
 *   rezgrp.f:28-60  zone changes after the step (outward only when the
 *                 old position is beyond the boundary too), chstep.f:22-32
 *
 * Zone codes: 1..nzones; nzones + 1 = off the grid.  Mass arrays zm, zo
 * are [nzones][mesh]; zm[0] is zone 1's array, which the combination turns
 * into the array the solve uses (scaled by pmass, scaled.f:89-92).
 */

#define CAT_(a, b) a##_##b
#define CAT(a, b) CAT_(a, b)
#define F(name) CAT(name, S)

static int ox_mzone(const OxZones* z, int istep) {
    int m = 1;
    if (z->nzones > 1)
        for (int i = 0; i < z->nzones; i++)
            if (istep % z->nstep[i] == 0) m = i + 1;
    return m;
}

static double ox_tsfac(const OxZones* z, int iz) {
    int i = iz < z->nzones ? iz : z->nzones;
    return (double)z->nstep[i - 1];
}

static int F(zoneno)(const OxZones* z, int nd, const R* q) {
    R r2 = q[0] * q[0] + q[1] * q[1];
    if (nd == 3) r2 = r2 + q[2] * q[2];
    R rad = SQRT(r2);
    int k = 1;
    for (int i = 1; i < z->nzones; i++)
        if (rad >= (R)z->zbr[i]) k = i + 1;
    return k;
}

/* chstep.f:22-32 (RVLF): redo the step from the old coordinates qo with the
 * step changed by tfac; a is the acceleration of the old step */
static void F(chstep)(int nd, const R* qo, R* q, R* a, R tfac) {
    for (int i = 0; i < nd; i++) {
        R vo = tfac * (qo[nd + i] + (R)0.5 * a[i] * ((R)1 - tfac));
        a[i] = a[i] * tfac * tfac;
        q[nd + i] = vo + a[i];
        q[i] = qo[i] + q[nd + i];
    }
}

int ox_zone_setup(const GxConfig* c, OxZones* z, int64_t n, double* pos, int32_t* zone) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int nd = g.ndim, st = 2 * nd;
    for (int64_t p = 0; p < n; p++) {
        double* q = pos + p * st;
        int32_t key;
        R w[27];
        if (!F(weight1)(&g, 1, q, &key, w)) {
            zone[p] = z->nzones + 1;
            continue;
        }
        zone[p] = F(zoneno)(z, nd, q);
        const double t = ox_tsfac(z, zone[p]);
        for (int i = 0; i < nd; i++) q[nd + i] = q[nd + i] * t;
    }
    z->istep = 0;
    for (int i = 0; i < GX_MAX_ZONES; i++) {
        z->lstep[i][0] = z->lstep[i][1] = -1;
        z->jrk[i][0] = g.nr;
        z->jrk[i][1] = 0;
    }
    return 0;
}

/* velocities back to base-step units (adjvls(.false.)) */
int ox_zone_unscale(const GxConfig* c, const OxZones* z, int64_t n, double* pos,
                    const int32_t* zone) {
    const int nd = c->ndim;
    for (int64_t p = 0; p < n; p++) {
        if (zone[p] > z->nzones) continue;
        const double t = ox_tsfac(z, zone[p]);
        for (int i = 0; i < nd; i++) pos[p * 2 * nd + nd + i] = pos[p * 2 * nd + nd + i] / t;
    }
    return 0;
}

/* masscl: step numbers of the new arrays, keep the older ones, clear */
static void F(zmasscl)(OxZones* z, int mzone, int normal, int64_t mesh, int nr, R* zm, R* zo) {
    int mstep[GX_MAX_ZONES];
    for (int k = 0; k < mzone; k++) {
        if (normal) mstep[k] = z->istep + z->nstep[k];
        else mstep[k] = z->istep > 0 ? ((z->istep - 1) / z->nstep[k] + 1) * z->nstep[k] : 0;
    }
    for (int k = 1; k < mzone; k++) {
        memcpy(zo + k * mesh, zm + k * mesh, sizeof(R) * mesh);
        z->lstep[k][0] = z->lstep[k][1];
        z->lstep[k][1] = mstep[k];
    }
    for (int k = 0; k < mzone; k++) {
        memset(zm + k * mesh, 0, sizeof(R) * mesh);
        z->jrk[k][0] = nr;
        z->jrk[k][1] = 0;
    }
}

/* zoncmb + scaled; then the source ring range of p2fndf */
static int F(zoncmb)(OxZones* z, int64_t mesh, R* zm, const R* zo, R pmass, int32_t* jrk,
                     int nr) {
    for (int k = 1; k < z->nzones; k++) {
        const int ns = z->nstep[k];
        int i = z->lstep[k][1] - z->istep;
        if (i < 0 || i > ns) return GX_ERR_STATE;
        if (i != ns) {
            const R fr = (R)1 - (R)i / (R)ns;
            for (int64_t j = 0; j < mesh; j++) zm[j] = zm[j] + fr * zm[k * mesh + j];
        }
        if (z->lstep[k][1] != z->istep) {
            i = z->istep - z->lstep[k][0];
            if (z->lstep[k][0] < 0 || i < 0 || i > ns) return GX_ERR_STATE;
            const R fr = (R)1 - (R)i / (R)ns;
            for (int64_t j = 0; j < mesh; j++) zm[j] = zm[j] + fr * zo[k * mesh + j];
        }
    }
    for (int64_t j = 0; j < mesh; j++) zm[j] = zm[j] * pmass;
    int jrs = nr, krs = 0;
    for (int k = 0; k < z->nzones; k++) {
        if (z->jrk[k][0] < jrs) jrs = z->jrk[k][0];
        if (z->jrk[k][1] > krs) krs = z->jrk[k][1];
        if (k > 0 && krs > z->jrk[k][1]) z->jrk[k][1] = krs;
    }
    jrk[0] = jrs;
    jrk[1] = krs;
    return 0;
}

/* massgn of the particles of zones 1..mzone (zone codes in zone[], mask
 * sel) into their zones' arrays */
static void F(zmassgn)(const GxConfig* c, OxZones* z, int mzone, int64_t n, const R* pos,
                       const int32_t* zone, const uint8_t* sel, int64_t mesh, R* zm) {
    int32_t* key = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
    R* wt = (R*)malloc(sizeof(R) * 27 * (n ? n : 1));
    uint8_t* on = (uint8_t*)malloc(n ? n : 1);
    uint8_t* onz = (uint8_t*)malloc(n ? n : 1);
    F(ox_weight)(c, 0, n, pos, key, wt, on);
    for (int k = 0; k < mzone; k++) {
        for (int64_t p = 0; p < n; p++)
            onz[p] = (uint8_t)(on[p] && zone[p] == k + 1 && (!sel || sel[p]));
        F(ox_massgn)(c, n, key, wt, onz, zm + k * mesh, z->jrk[k]);
    }
    free(key);
    free(wt);
    free(on);
    free(onz);
}

int ox_zone_masset(const GxConfig* c, OxZones* z, int64_t n, const double* pos,
                   const int32_t* zone, double* zm, double* zo, int32_t* jrk) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int64_t mesh = g.mesh;
    F(zmasscl)(z, z->nzones, 0, mesh, g.nr, zm, zo);
    F(zmassgn)(c, z, z->nzones, n, pos, zone, NULL, mesh, zm);
    return F(zoncmb)(z, mesh, zm, zo, (R)c->pmass, jrk, g.nr);
}

int ox_zone_step(const GxConfig* c, OxZones* z, const double* G, int64_t n, double* pos,
                 int32_t* zone, double* zm, double* zo, int32_t* jrk, int nsteps) {
    F(og) g;
    if (F(og_init)(c, &g)) return GX_ERR_ARG;
    const int nd = g.ndim, st = 2 * nd, nz = z->nzones, off = nz + 1;
    const int64_t mesh = g.mesh;
    R* fl = (R*)malloc(sizeof(R) * 4 * (size_t)mesh);
    R* acc = (R*)malloc(sizeof(R) * nd * (n ? n : 1));
    uint8_t* sel = (uint8_t*)malloc(n ? n : 1);
    int rc = 0;
    for (int s = 0; s < nsteps && !rc; s++) {
        const int mzone = ox_mzone(z, z->istep);
        F(ox_findf)(c, G, zm, 0, jrk[0], jrk[1], fl);
        F(ox_polcat)(c, fl);
        F(ox_grdacc)(c, n, pos, fl, 0, acc, NULL);
        F(zmasscl)(z, mzone, 1, mesh, g.nr, zm, zo);
        for (int64_t p = 0; p < n; p++) {
            const int z0 = zone[p];
            sel[p] = (uint8_t)(z0 <= mzone || (z0 == off && mzone == nz));
            if (!sel[p]) continue;
            R* q = pos + p * st;
            R qo[6], a[3];
            for (int i = 0; i < st; i++) qo[i] = q[i];
            const R t = (R)ox_tsfac(z, z0);
            for (int i = 0; i < nd; i++) a[i] = (z0 == off) ? (R)0 : acc[p * nd + i] * t * t;
            for (int i = 0; i < nd; i++) {
                q[nd + i] = q[nd + i] + a[i];
                q[i] = q[i] + q[nd + i];
            }
            int32_t key;
            R w[27];
            const int on = F(weight1)(&g, 1, q, &key, w);
            int iz = z0;
            if (z0 != off) {
                if (!on) {
                    iz = off;
                    if (z0 < nz) F(chstep)(nd, qo, q, a, (R)(ox_tsfac(z, nz) / ox_tsfac(z, z0)));
                }
            } else if (on) {
                iz = nz;
            }
            if (z0 != off && mzone > 1 && iz <= mzone) {
                int kz = F(zoneno)(z, nd, q);
                if (kz > mzone) kz = mzone;
                if (kz > iz) kz = F(zoneno)(z, nd, qo);
                if (kz != iz) {
                    F(chstep)(nd, qo, q, a, (R)(ox_tsfac(z, kz) / ox_tsfac(z, iz)));
                    iz = kz;
                }
            }
            zone[p] = iz;
        }
        F(zmassgn)(c, z, mzone, n, pos, zone, sel, mesh, zm);
        z->istep += 1;
        rc = F(zoncmb)(z, mesh, zm, zo, (R)c->pmass, jrk, g.nr);
    }
    free(fl);
    free(acc);
    free(sel);
    return rc;
}
