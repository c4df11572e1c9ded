/*
 * gx_oracle_adj.h -- FP64 adjoint of the 2D polar-grid PM step (TEST
 * INFRASTRUCTURE ONLY; see gx_oracle.h).  Included by gx_oracle.c inside the
 * FP64 instantiation of gx_oracle_tmpl.h (R = double, suffix f64).
 *
 * Objective: J = |A2(x_T)|, A2 = (1/n) sum_p e^{2 i phi_p} over all
 * particles, after nsteps of the step restated in ox_step_f64 (findf +
 * polcat, getacc/grdacc with the ISOT halo, stpgrp, massgn + scaled).
 * The adjoint runs the forward trajectory storing every state, then the
 * reverse sweep: with mu = lambda_v + lambda_x,
 *   lambda_v <- mu
 *   lambda_x <- lambda_x + (d a / d x)^T mu
 * where (d a / d x)^T mu has three parts: the slope of the interpolation
 * weights against the field, the halo's Jacobian, and the field's own
 * dependence on every position: psi = K^T (sum_p W(x_p) mu_p) with K the
 * linear map mass -> (fx, fy) (forward DFT, radial contraction, synthesis,
 * polcat), then lambda_x_p += pmass sum_c grad W_c(x_p) psi_c.
 * Halo parameters: dJ/d(halo_rc) and dJ/d(halo_v2) in config units.
 * 2D, one sector, mixed rings (stdpol or log map).
 */

#define CAT_(a, b) a##_##b
#define CAT(a, b) CAT_(a, b)
#define F(name) CAT(name, S)

/* weights and their x, y gradients of the interpolation cell (weight.f:61-101) */
static int F(wgrad2)(const F(og) * g, const R* q, int32_t* key, R* w, R (*dw)[2]) {
    R x = q[0], y = q[1];
    if (!F(weight1)(g, 1, q, key, w)) return 0;
    R rr = SQRT(x * x + y * y);
    if (rr <= 0) {
        for (int k = 0; k < 4; k++) dw[k][0] = dw[k][1] = 0;
        return 1;
    }
    R u = F(uofgr)(g, rr);
    R t = atan2(y, x) * (double)g->na / (2.0 * OX_PI);
    if (t < 0) t += (R)g->na;
    int ju = (int)u;
    if (ju > g->nr - 2) ju = g->nr - 2;
    R du = u - (R)ju, dt = t - (R)(int)t;
    R dudr = (g->rmap == GX_RMAP_STDPOL) ? 1.0 / (g->ua * (1.0 + rr)) : 1.0 / (g->ua * rr);
    R gu[2] = {dudr * x / rr, dudr * y / rr};
    R ts = (double)g->na / (2.0 * OX_PI) / (rr * rr);
    R gt[2] = {-y * ts, x * ts};
    for (int i = 0; i < 2; i++) {
        dw[0][i] = -(1 - dt) * gu[i] - (1 - du) * gt[i];
        dw[1][i] = -dt * gu[i] + (1 - du) * gt[i];
        dw[2][i] = (1 - dt) * gu[i] - du * gt[i];
        dw[3][i] = dt * gu[i] + du * gt[i];
    }
    return 1;
}

static double F(adj_a2)(int64_t n, const R* pos, double* a2) {
    double sre = 0, sim = 0;
    for (int64_t p = 0; p < n; p++) {
        const R* q = pos + 4 * p;
        double r2 = q[0] * q[0] + q[1] * q[1];
        if (r2 > 0) {
            sre += (q[0] * q[0] - q[1] * q[1]) / r2;
            sim += 2 * q[0] * q[1] / r2;
        }
    }
    a2[0] = n ? sre / n : 0;
    a2[1] = n ? sim / n : 0;
    return sqrt(a2[0] * a2[0] + a2[1] * a2[1]);
}

/* J of the trajectory: masset, then nsteps x (findf, polcat, getacc,
 * stpgrp, masset) from the records pos (n x 4, updated in place) */
int ox_adj_forward(const GxConfig* c, const double* G, int64_t n, double* pos, int nsteps,
                   double* a2, double* J) {
    F(og) g;
    if (F(og_init)(c, &g) || g.ndim != 2 || g.nsect != 1) return GX_ERR_ARG;
    double* mass = (double*)calloc((size_t)g.mesh, sizeof(double));
    int32_t jrk[2];
    F(ox_masset)(c, n, pos, mass, jrk);
    if (nsteps > 0) F(ox_step)(c, G, n, pos, mass, jrk, nsteps, 0, NULL);
    *J = F(adj_a2)(n, pos, a2);
    free(mass);
    return 0;
}

/* K^T of the 2D solve (ox_findf_f64 + ox_polcat_f64 restricted to fr, ft):
 * Q [2][mesh] (x, y components at the nodes) -> psi [mesh] */
static void F(adj_solveT)(const F(og) * g, const R* G, const R* Q, R* psi) {
    const int nr = g->nr, na = g->na, ng = g->ng, mmax = g->mmax;
    const int64_t mesh = g->mesh;
    const R scale = (R)1 / (R)na;
    R* gr = (R*)malloc(sizeof(R) * mesh);
    R* gt = (R*)malloc(sizeof(R) * mesh);
    for (int j = 0; j < na; j++) {
        R th = 2.0 * OX_PI * (double)j / (double)na, cp = COS(th), sp = SIN(th);
        for (int ir = 0; ir < nr; ir++) {
            int64_t l = (int64_t)ir * na + j;
            gr[l] = Q[l] * cp + Q[mesh + l] * sp;
            gt[l] = -Q[l] * sp + Q[mesh + l] * cp;
        }
    }
    /* synthesis^T: V[t][m][ir] = (sum_j g_t c_m(j), sum_j g_t s_m(j)) x scale */
    R* Va = (R*)calloc((size_t)2 * ng * nr, sizeof(R));
    R* Vb = (R*)calloc((size_t)2 * ng * nr, sizeof(R));
    for (int t = 0; t < 2; t++) {
        const R* gg = t ? gt : gr;
        for (int m = 0; m < ng; m++) {
            if (g->lg[m]) continue;
            for (int ir = 0; ir < nr; ir++) {
                R sa = 0, sb = 0;
                for (int j = 0; j < na; j++) {
                    R v = gg[(int64_t)ir * na + j];
                    double ang = 2.0 * OX_PI * (double)m * (double)j / (double)na;
                    if (m == 0) sa += v;
                    else if (m == mmax - 1) sa += (j & 1) ? -v : v;
                    else {
                        sa += 2 * v * cos(ang);
                        sb -= 2 * v * sin(ang);
                    }
                }
                Va[((int64_t)t * ng + m) * nr + ir] = scale * sa;
                Vb[((int64_t)t * ng + m) * nr + ir] = scale * sb;
            }
        }
    }
    /* radial contraction^T (p2conv.f:114-181 transposed) */
    R* Aa = (R*)calloc((size_t)ng * nr, sizeof(R));
    R* Ab = (R*)calloc((size_t)ng * nr, sizeof(R));
    for (int m = 0; m < ng; m++) {
        if (g->lg[m]) continue;
        const int hasb = (m > 0 && m < mmax - 1);
        const int ft_ok = (ng > 1) && (m >= 1) && (m <= ((ng < mmax - 1) ? ng : mmax - 1) - 1);
        const R* G0 = G + ((int64_t)(0 * ng + m) * nr) * nr;
        const R* G1 = G + ((int64_t)(1 * ng + m) * nr) * nr;
        for (int is = 0; is < nr; is++) {
            R sa = 0, sb = 0;
            for (int ir = 0; ir < nr; ir++) {
                R g0 = G0[(int64_t)is * nr + ir];
                sa += g0 * Va[(int64_t)m * nr + ir];
                if (hasb) sb += g0 * Vb[(int64_t)m * nr + ir];
                if (ft_ok) {
                    R g1 = G1[(int64_t)is * nr + ir];
                    sb += g1 * Va[((int64_t)ng + m) * nr + ir];
                    sa -= g1 * Vb[((int64_t)ng + m) * nr + ir];
                }
            }
            Aa[(int64_t)m * nr + is] = sa;
            Ab[(int64_t)m * nr + is] = hasb ? sb : 0;
        }
    }
    /* forward DFT^T: a_m = sum x cos, b_m = -sum x sin */
    for (int ir = 0; ir < nr; ir++)
        for (int j = 0; j < na; j++) {
            R s = 0;
            for (int m = 0; m < ng; m++) {
                if (g->lg[m]) continue;
                double ang = 2.0 * OX_PI * (double)m * (double)j / (double)na;
                s += Aa[(int64_t)m * nr + ir] * cos(ang) - Ab[(int64_t)m * nr + ir] * sin(ang);
            }
            psi[(int64_t)ir * na + j] = s;
        }
    free(gr);
    free(gt);
    free(Va);
    free(Vb);
    free(Aa);
    free(Ab);
}

/* gradient of J with respect to the initial records (grad n x 4) and the
 * halo parameters (dtheta[0] = dJ/d halo_rc, dtheta[1] = dJ/d halo_v2) */
int ox_adj_gradient(const GxConfig* c, const double* G, int64_t n, const double* pos0, int nsteps,
                    double* grad, double* dtheta, double* J) {
    F(og) g;
    if (F(og_init)(c, &g) || g.ndim != 2 || g.nsect != 1) return GX_ERR_ARG;
    const int64_t mesh = g.mesh;
    const double pm = c->pmass;
    double* traj = (double*)malloc(sizeof(double) * 4 * n * (size_t)(nsteps + 1));
    double* mass = (double*)calloc((size_t)mesh, sizeof(double));
    double* fl = (double*)malloc(sizeof(double) * 4 * mesh);
    double* Q = (double*)malloc(sizeof(double) * 2 * mesh);
    double* psi = (double*)malloc(sizeof(double) * mesh);
    double* lx = (double*)calloc((size_t)2 * n, sizeof(double));
    double* lv = (double*)calloc((size_t)2 * n, sizeof(double));
    double* mu = (double*)malloc(sizeof(double) * 2 * n);
    int32_t jrk[2];
    memcpy(traj, pos0, sizeof(double) * 4 * n);
    for (int s = 0; s < nsteps; s++) {
        double* cur = traj + (size_t)s * 4 * n;
        double* nxt = cur + 4 * n;
        memcpy(nxt, cur, sizeof(double) * 4 * n);
        F(ox_masset)(c, n, nxt, mass, jrk);
        F(ox_step)(c, G, n, nxt, mass, jrk, 1, 0, NULL);
    }
    double a2[2];
    *J = F(adj_a2)(n, traj + (size_t)nsteps * 4 * n, a2);
    /* dJ/dx_T */
    {
        const double* xT = traj + (size_t)nsteps * 4 * n;
        for (int64_t p = 0; p < n; p++) {
            double x = xT[4 * p], y = xT[4 * p + 1], r2 = x * x + y * y;
            if (r2 <= 0 || *J <= 0) continue;
            double fr = (x * x - y * y) / r2, fi = 2 * x * y / r2;
            /* dA2/dx = (1/n)(-2 i f y / r2), dA2/dy = (1/n)(2 i f x / r2) */
            double dxr = 2 * fi * y / r2 / n, dxi = -2 * fr * y / r2 / n;
            double dyr = -2 * fi * x / r2 / n, dyi = 2 * fr * x / r2 / n;
            lx[2 * p] = (a2[0] * dxr + a2[1] * dxi) / *J;
            lx[2 * p + 1] = (a2[0] * dyr + a2[1] * dyi) / *J;
        }
    }
    dtheta[0] = dtheta[1] = 0;
    const double v2 = g.halo_v2, rc = g.halo_rc;
    for (int s = nsteps - 1; s >= 0; s--) {
        const double* xs = traj + (size_t)s * 4 * n;
        F(ox_masset)(c, n, xs, mass, jrk);
        F(ox_findf)(c, G, mass, 0, jrk[0], jrk[1], fl);
        F(ox_polcat)(c, fl);
        memset(Q, 0, sizeof(double) * 2 * mesh);
        for (int64_t p = 0; p < n; p++) {
            mu[2 * p] = lv[2 * p] + lx[2 * p];
            mu[2 * p + 1] = lv[2 * p + 1] + lx[2 * p + 1];
        }
        for (int64_t p = 0; p < n; p++) {
            const double* q = xs + 4 * p;
            int32_t key, ic[8];
            double w[8], dw[4][2];
            double m0 = mu[2 * p], m1 = mu[2 * p + 1];
            lv[2 * p] = m0;
            lv[2 * p + 1] = m1;
            if (!F(wgrad2)(&g, q, &key, w, dw)) continue;
            F(corners)(&g, key, ic);
            for (int k = 0; k < 4; k++) {
                if (ic[k] < 0) continue;
                double fdot = fl[ic[k]] * m0 + fl[mesh + ic[k]] * m1;
                lx[2 * p] += dw[k][0] * fdot;
                lx[2 * p + 1] += dw[k][1] * fdot;
                Q[ic[k]] += w[k] * m0;
                Q[mesh + ic[k]] += w[k] * m1;
            }
            if (g.halo == 1) {
                double x = q[0], y = q[1], d = x * x + y * y + rc * rc;
                /* h = -v2 x / d: Jacobian -v2 (I / d - 2 x x^T / d^2) */
                double hxx = -v2 * (1 / d - 2 * x * x / (d * d));
                double hyy = -v2 * (1 / d - 2 * y * y / (d * d));
                double hxy = v2 * 2 * x * y / (d * d);
                lx[2 * p] += hxx * m0 + hxy * m1;
                lx[2 * p + 1] += hxy * m0 + hyy * m1;
                dtheta[1] += -(x * m0 + y * m1) / d;
                dtheta[0] += v2 * 2 * rc * (x * m0 + y * m1) / (d * d);
            }
        }
        F(adj_solveT)(&g, G, Q, psi);
        for (int64_t p = 0; p < n; p++) {
            int32_t key, ic[8];
            double w[8], dw[4][2];
            if (!F(wgrad2)(&g, xs + 4 * p, &key, w, dw)) continue;
            F(corners)(&g, key, ic);
            for (int k = 0; k < 4; k++) {
                if (ic[k] < 0) continue;
                lx[2 * p] += pm * dw[k][0] * psi[ic[k]];
                lx[2 * p + 1] += pm * dw[k][1] * psi[ic[k]];
            }
        }
    }
    for (int64_t p = 0; p < n; p++) {
        grad[4 * p] = lx[2 * p];
        grad[4 * p + 1] = lx[2 * p + 1];
        grad[4 * p + 2] = lv[2 * p];
        grad[4 * p + 3] = lv[2 * p + 1];
    }
    free(traj);
    free(mass);
    free(fl);
    free(Q);
    free(psi);
    free(lx);
    free(lv);
    free(mu);
    return 0;
}

#undef F
#undef CAT
#undef CAT_
