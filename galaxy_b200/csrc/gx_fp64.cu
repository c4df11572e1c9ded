// gx_fp64.cu -- the plain FP64 GPU path: the same step as the mixed path
// (weight/massgn, p2/p3 manl-conv-fsyn, polcat, grdacc, stpgrp) written the
// straightforward way: FP64 everywhere, one thread per output element,
// FP64 atomic deposit, one kernel per reference routine, no fusion and no
// graph.  It is the baseline the mixed path's particle-steps/s is quoted
// against, and the FP64 reference for force errors at sizes the CPU oracle
// cannot reach.
#include <algorithm>

#include "gx_common.cuh"

__constant__ int c64_act_m[260];

struct Cell64 {
    int key;
    double du, dt, dz;
};

// weight.f:61-101 / 196-250 in FP64
__device__ __forceinline__ Cell64 cell64(const DevGeo& g, double x, double y, double z, bool old) {
    Cell64 c;
    c.key = -1;
    c.du = c.dt = c.dz = 0.0;
    double rr = sqrt(x * x + y * y);
    if (rr > g.rgrid_d) return c;
    if (g.ndim == 3 && fabs(z) > g.zm_d) return c;
    if (rr < g.rinh_d) return c;
    double u = (g.rmap == GX_RMAP_STDPOL) ? log(1.0 + rr) / g.ua_d : log(rr) / g.ua_d + g.uoffs_d;
    double t = 0.0;
    if (g.ndim == 2 || rr > 0.0) {
        t = atan2(y, x) * (double)g.na / (2.0 * GX_PI);
        if (t < 0.0) t += (double)g.na;
    }
    if (!old && g.nsect > 1) t = fmod(t, g.thmax_d);
    int ju = (int)u;
    if (ju > g.nr - 2) ju = g.nr - 2;
    int jt = (int)t;
    if (jt >= g.na) jt = g.na - 1;
    c.du = u - ju;
    c.dt = t - jt;
    if (g.ndim == 2) {
        c.key = ju * g.na + jt;
    } else {
        double zz = (z + g.zm_d) / g.dzg_d;
        int jz = (int)zz;
        if (jz < 0) jz = 0;
        if (jz > g.ngz - 2) jz = g.ngz - 2;
        c.dz = zz - jz;
        c.key = (ju * g.ngz + jz) * g.na + jt;
    }
    return c;
}

__device__ __forceinline__ void weights64(const DevGeo& g, const Cell64& c, double* w) {
    if (g.ndim == 2) {
        double dd = c.du * c.dt;
        w[0] = 1.0 - c.du - c.dt + dd;
        w[1] = c.dt - dd;
        w[2] = c.du - dd;
        w[3] = dd;
        w[4] = w[5] = w[6] = w[7] = 0.0;
    } else {
        w[0] = (1.0 - c.dt) * (1.0 - c.dz) * (1.0 - c.du);
        w[1] = c.dt * (1.0 - c.dz) * (1.0 - c.du);
        w[2] = (1.0 - c.dt) * c.dz * (1.0 - c.du);
        w[3] = c.dt * c.dz * (1.0 - c.du);
        w[4] = (1.0 - c.dt) * (1.0 - c.dz) * c.du;
        w[5] = c.dt * (1.0 - c.dz) * c.du;
        w[6] = (1.0 - c.dt) * c.dz * c.du;
        w[7] = c.dt * c.dz * c.du;
    }
}

__global__ void k64_weights(DevGeo g, const double* __restrict__ P, int64_t cap, int64_t n, bool old,
                            int32_t* __restrict__ key, double* __restrict__ W,
                            int32_t* __restrict__ jrk) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double z = (g.ndim == 3) ? P[2 * cap + i] : 0.0;
    Cell64 c = cell64(g, P[i], P[cap + i], z, old);
    key[i] = c.key;
    double w[8];
    weights64(g, c, w);
    for (int k = 0; k < 8; k++) W[k * cap + i] = w[k];
    if (jrk && c.key >= 0) {
        int ring = c.key / (g.na * g.ngz);
        atomicMin(&jrk[0], ring + 1);
        atomicMax(&jrk[1], ring + 2);
    }
}

__global__ void k64_deposit(DevGeo g, const int32_t* __restrict__ key, const double* __restrict__ W,
                            int64_t cap, int64_t n, double* __restrict__ mass) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = key[i];
    if (k < 0) return;
    int ic[8];
    int nc = gx_corners(g, k, ic);
    for (int q = 0; q < nc; q++)
        if (ic[q] >= 0) atomicAdd(&mass[ic[q]], W[q * cap + i]);
}

__global__ void k64_scale(double* __restrict__ a, int n, double s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] *= s;
}

// azimuthal analysis: thread per (ring, plane, active harmonic)
__global__ void k64_fwd_az(DevGeo g, int nact, const int32_t* __restrict__ jrk,
                           const double* __restrict__ mass, double* __restrict__ az) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t tot = (int64_t)g.nr * g.ngz * nact;
    if (i >= tot) return;
    int a = i % nact;
    int iz = (i / nact) % g.ngz;
    int ir = (int)(i / ((int64_t)nact * g.ngz));
    if (ir < jrk[0] - 1 || ir > min(jrk[1], g.nr) - 1) return;
    int m = c64_act_m[a];
    const double* x = mass + ((int64_t)ir * g.ngz + iz) * g.na;
    double sa = 0, sb = 0;
    for (int j = 0; j < g.na; j++) {
        double s, co;
        sincospi(2.0 * (double)((m * j) % g.na) / (double)g.na, &s, &co);
        sa += x[j] * co;
        sb -= x[j] * s;
    }
    az[2 * i] = sa;
    az[2 * i + 1] = sb;
}

// vertical analysis: thread per (active harmonic, kz, ring) -> spec[a][k][ir][4]
__global__ void k64_fwd_z(DevGeo g, int nact, const int32_t* __restrict__ jrk,
                          const double* __restrict__ az, double* __restrict__ spec) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t tot = (int64_t)nact * g.nkz * g.nr;
    if (i >= tot) return;
    int ir = i % g.nr;
    int k = (i / g.nr) % g.nkz;
    int a = (int)(i / ((int64_t)g.nr * g.nkz));
    double o[4] = {0, 0, 0, 0};
    if (!(ir < jrk[0] - 1 || ir > min(jrk[1], g.nr) - 1)) {
        for (int z = 0; z < g.ngz; z++) {
            const double* c = az + ((((int64_t)ir * g.ngz + z) * nact) + a) * 2;
            if (g.ndim == 2) {
                o[0] += c[0];
                o[2] += c[1];
            } else {
                double s, co;
                sincospi((double)(((int64_t)k * z) % (2 * g.ngz)) / (double)g.ngz, &s, &co);
                o[0] += c[0] * co;
                o[1] -= c[0] * s;
                o[2] += c[1] * co;
                o[3] -= c[1] * s;
            }
        }
    }
    for (int q = 0; q < 4; q++) spec[i * 4 + q] = o[q];
}

// radial convolution: thread per (type, a, k, ir)
__global__ void k64_conv(DevGeo g, int nact, int tmask, const double* __restrict__ G,
                         const double* __restrict__ spec, double* __restrict__ out,
                         const int32_t* __restrict__ jrk) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t per = (int64_t)nact * g.nkz * g.nr;
    if (i >= 4 * per) return;
    int t = (int)(i / per);
    int64_t r = i - t * per;
    int ir = r % g.nr;
    int k = (r / g.nr) % g.nkz;
    int a = (int)(r / ((int64_t)g.nr * g.nkz));
    int m = c64_act_m[a];
    double o[4] = {0, 0, 0, 0};
    bool valid = (tmask >> t) & 1;
    if (t == 1) valid = valid && m >= 1 && m <= min(g.ng, g.mmax - 1) - 1;
    if (t == 2) valid = valid && g.ndim == 3 && k >= 1 && k <= g.ngz - 1;
    if (valid) {
        int js = max(jrk[0], 1) - 1, ks = min(jrk[1], g.nr) - 1;
        const double* Gt = G + ((((int64_t)t * g.ng + m) * g.nkz + k) * g.nr) * g.nr;
        for (int is = js; is <= ks; is++) {
            double gv = Gt[(int64_t)is * g.nr + ir];
            const double* s = spec + ((((int64_t)a * g.nkz + k) * g.nr) + is) * 4;
            if (t == 0 || t == 3) {
                o[0] += gv * s[0]; o[1] += gv * s[1]; o[2] += gv * s[2]; o[3] += gv * s[3];
            } else if (t == 1) {
                o[0] += gv * s[2]; o[2] -= gv * s[0]; o[1] += gv * s[3]; o[3] -= gv * s[1];
            } else {
                o[0] += gv * s[1]; o[1] -= gv * s[0]; o[2] += gv * s[3]; o[3] -= gv * s[2];
            }
        }
    }
    for (int q = 0; q < 4; q++) out[i * 4 + q] = o[q];
}

// vertical synthesis: thread per (type, ring, plane, a) -> rows[t][ir][z][a][2]
__global__ void k64_syn_z(DevGeo g, int nact, const double* __restrict__ out,
                          double* __restrict__ rows) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t per = (int64_t)g.nr * g.ngz * nact;
    if (i >= 4 * per) return;
    int t = (int)(i / per);
    int64_t r = i - t * per;
    int a = r % nact;
    int z = (r / nact) % g.ngz;
    int ir = (int)(r / ((int64_t)nact * g.ngz));
    const int64_t opere = (int64_t)nact * g.nkz * g.nr;
    double ra = 0, rb = 0;
    for (int k = 0; k < g.nkz; k++) {
        const double* o = out + ((int64_t)t * opere + ((int64_t)a * g.nkz + k) * g.nr + ir) * 4;
        if (g.ndim == 2) {
            ra = o[0];
            rb = o[2];
            break;
        }
        double wa, wb;
        if (k == 0) {
            wa = 1.0;
            wb = 0.0;
        } else if (k == g.ngz) {
            wa = (z & 1) ? -1.0 : 1.0;
            wb = 0.0;
        } else {
            double s, co;
            sincospi((double)(((int64_t)k * z) % (2 * g.ngz)) / (double)g.ngz, &s, &co);
            wa = 2.0 * co;
            wb = -2.0 * s;
        }
        ra += o[0] * wa + o[1] * wb;
        rb += o[2] * wa + o[3] * wb;
    }
    rows[2 * i] = ra;
    rows[2 * i + 1] = rb;
}

// azimuthal synthesis + scale + polcat: thread per node
__global__ void k64_syn_az(DevGeo g, int nact, int tmask, const double* __restrict__ rows,
                           double* __restrict__ polar, double* __restrict__ field) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= g.mesh) return;
    int j = i % g.na;
    int64_t rz = i / g.na;  // ir * ngz + z
    const int64_t per = (int64_t)g.nr * g.ngz * nact;
    const double scale = (g.ndim == 3) ? 1.0 / (2.0 * g.ngz * g.na) : 1.0 / g.na;
    double v[4];
    for (int t = 0; t < 4; t++) {
        double s = 0;
        if ((tmask >> t) & 1) {
            for (int a = 0; a < nact; a++) {
                int m = c64_act_m[a];
                const double* r = rows + (t * per + rz * nact + a) * 2;
                if (m == 0) s += r[0];
                else if (m == g.mmax - 1) s += (j & 1) ? -r[0] : r[0];
                else {
                    double sn, co;
                    sincospi(2.0 * (double)((m * j) % g.na) / (double)g.na, &sn, &co);
                    s += 2.0 * (r[0] * co - r[1] * sn);
                }
            }
        }
        v[t] = s * scale;
    }
    const int64_t mesh = g.mesh;
    for (int t = 0; t < 4; t++) polar[t * mesh + i] = v[t];
    double sn, co;
    sincospi(2.0 * (double)j / (double)g.na, &sn, &co);
    field[i] = v[0] * co - v[1] * sn;
    field[mesh + i] = v[0] * sn + v[1] * co;
    field[2 * mesh + i] = v[2];
    field[3 * mesh + i] = v[3];
}

// grdacc in FP64: thread per particle
__global__ void k64_gather(DevGeo g, const double* __restrict__ P, int64_t cap, int64_t n,
                           const double* __restrict__ F, double* __restrict__ acc,
                           double* __restrict__ pot) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nd = g.ndim;
    double x = P[i], y = P[cap + i], z = (nd == 3) ? P[2 * cap + i] : 0.0;
    double a[3] = {0, 0, 0}, ph = 0;
    Cell64 c = cell64(g, x, y, z, true);
    if (c.key >= 0) {
        double w[8];
        int ic[8];
        weights64(g, c, w);
        int nc = gx_corners(g, c.key, ic);
        const int64_t mesh = g.mesh;
        for (int k = 0; k < nc; k++) {
            if (ic[k] < 0) continue;
            for (int d = 0; d < nd; d++) a[d] += F[d * mesh + ic[k]] * w[k];
            ph += F[3 * mesh + ic[k]] * w[k];
        }
        if (g.halo == 1) {
            double r2 = x * x + y * y + ((nd == 3) ? z * z : 0.0);
            double rr = sqrt(r2);
            double fr = -g.halo_v2_d * rr / (r2 + g.halo_rc2_d);
            if (fr != 0.0) {
                fr /= rr;
                a[0] += fr * x;
                a[1] += fr * y;
                if (nd == 3) a[2] += fr * z;
            }
            ph += 0.5 * g.halo_v2_d * log(1.0 + r2 / g.halo_rc2_d);
        } else if (g.halo == 2) {
            // fixed softened Kuz'min-Toomre disc force (frdisc.f:27-29)
            const double d = x * x + y * y + ((nd == 3) ? z * z : 0.0) + g.halo_rc2_d;
            const double sd = sqrt(d);
            const double f = -g.halo_v2_d / (d * sd);
            a[0] += f * x;
            a[1] += f * y;
            if (nd == 3) a[2] += f * z;
            ph -= g.halo_v2_d / sd;
        }
    }
    for (int d = 0; d < nd; d++) acc[d * cap + i] = a[d];
    if (pot) pot[i] = ph;
}

// stpgrp in FP64
__global__ void k64_push(DevGeo g, double* __restrict__ P, int64_t cap, int64_t n,
                         const double* __restrict__ acc) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nd = g.ndim;
    for (int d = 0; d < nd; d++) {
        double v = P[(nd + d) * cap + i] + acc[d * cap + i];
        P[(nd + d) * cap + i] = v;
        P[d * cap + i] = P[d * cap + i] + v;
    }
}

__global__ void k64_to_f32_aos(const double* __restrict__ a, int64_t cap, int64_t n, int nd,
                               float* __restrict__ out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int d = 0; d < nd; d++) out[i * nd + d] = (float)a[d * cap + i];
}
__global__ void k64_to_f32(const double* __restrict__ a, int64_t n, float* __restrict__ out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)a[i];
}

// ---------------------------------------------------------------------------
static inline unsigned nblk(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int gx_fp64_masset(GxCtx* c) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    GX_CUDA(c, cudaMemsetAsync(c->mass64, 0, sizeof(double) * g.mesh, c->stream));
    int32_t jrk[2] = {g.nr, 0};
    GX_CUDA(c, cudaMemcpyAsync(c->jrk_d, jrk, sizeof jrk, cudaMemcpyHostToDevice, c->stream));
    if (n > 0) {
        k64_weights<<<nblk(n, 256), 256, 0, c->stream>>>(g, c->p64, c->cap, n, false, c->key64,
                                                        c->w64, c->jrk_d);
        GX_LAUNCHED(c);
        k64_deposit<<<nblk(n, 256), 256, 0, c->stream>>>(g, c->key64, c->w64, c->cap, n, c->mass64);
        GX_LAUNCHED(c);
    }
    k64_scale<<<nblk(g.mesh, 256), 256, 0, c->stream>>>(c->mass64, g.mesh, (double)c->cfg.pmass);
    GX_LAUNCHED(c);
    return GX_OK;
}

int gx_fp64_findf(GxCtx* c, int lpot, bool) {
    const DevGeo& g = c->g;
    const int nact = c->spec.nact;
    GX_CUDA(c, cudaMemcpyToSymbolAsync(c64_act_m, c->spec.m, sizeof(int) * 260, 0,
                                       cudaMemcpyHostToDevice, c->stream));
    double *az = c->az64, *rows = c->rows64;
    int tmask = 1 | 2 | (g.ndim == 3 ? 4 : 0) | (lpot ? 8 : 0);
    if (g.ng == 1) tmask &= ~2;
    int64_t n1 = (int64_t)g.nr * g.ngz * nact;
    GX_CUDA(c, cudaMemsetAsync(az, 0, sizeof(double) * 2 * n1, c->stream));
    k64_fwd_az<<<nblk(n1, 128), 128, 0, c->stream>>>(g, nact, c->jrk_d, c->mass64, az);
    GX_LAUNCHED(c);
    int64_t n2 = (int64_t)nact * g.nkz * g.nr;
    k64_fwd_z<<<nblk(n2, 128), 128, 0, c->stream>>>(g, nact, c->jrk_d, az, c->spec64);
    GX_LAUNCHED(c);
    k64_conv<<<nblk(4 * n2, 128), 128, 0, c->stream>>>(g, nact, tmask, c->green64, c->spec64,
                                                       c->out64, c->jrk_d);
    GX_LAUNCHED(c);
    k64_syn_z<<<nblk(4 * n1, 128), 128, 0, c->stream>>>(g, nact, c->out64, rows);
    GX_LAUNCHED(c);
    k64_syn_az<<<nblk(g.mesh, 128), 128, 0, c->stream>>>(g, nact, tmask, rows, c->polar64,
                                                         c->field64);
    GX_LAUNCHED(c);
    c->have_field = true;
    c->field_pot = lpot != 0;
    return GX_OK;
}

int gx_fp64_getacc(GxCtx* c, float* acc, float* pot) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    if (n == 0) return GX_OK;
    double* pot64 = c->pot64;
    k64_gather<<<nblk(n, 256), 256, 0, c->stream>>>(g, c->p64, c->cap, n, c->field64, c->acc64, pot64);
    GX_LAUNCHED(c);
    k64_to_f32_aos<<<nblk(n, 256), 256, 0, c->stream>>>(c->acc64, c->cap, n, g.ndim, c->pacc);
    GX_LAUNCHED(c);
    k64_to_f32<<<nblk(n, 256), 256, 0, c->stream>>>(pot64, n, c->ppot);
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaMemcpyAsync(acc, c->pacc, sizeof(float) * g.ndim * n, cudaMemcpyDeviceToHost,
                               c->stream));
    if (pot)
        GX_CUDA(c, cudaMemcpyAsync(pot, c->ppot, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    return GX_OK;
}

int gx_fp64_step(GxCtx* c, int nsteps, int phys) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    for (int s = 0; s < nsteps; s++) {
        int rc = gx_fp64_findf(c, phys && s == nsteps - 1, true);
        if (rc) return rc;
        if (n > 0) {
            k64_gather<<<nblk(n, 256), 256, 0, c->stream>>>(g, c->p64, c->cap, n, c->field64,
                                                           c->acc64, nullptr);
            GX_LAUNCHED(c);
            k64_push<<<nblk(n, 256), 256, 0, c->stream>>>(g, c->p64, c->cap, n, c->acc64);
            GX_LAUNCHED(c);
        }
        rc = gx_fp64_masset(c);
        if (rc) return rc;
    }
    c->have_field = false;
    return GX_OK;
}
