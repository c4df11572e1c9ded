// gx_diag.cu -- time-centring (tmcent) and the global integrals (icheck).
#include <algorithm>
#include <vector>

#include "gx_common.cuh"

// grid + halo acceleration and the two potentials, mixed path
__device__ __forceinline__ void accel_parts(const DevGeo& g, const float4* __restrict__ F, float x,
                                            float y, float z, float* a, float& pgrid,
                                            float& phalo) {
    a[0] = a[1] = a[2] = 0.f;
    pgrid = phalo = 0.f;
    CellW cw = gx_cell(g, x, y, z, true);
    if (cw.key < 0) return;
    float w[27];
    int ic[27];
    int nc = 27;
    if (g.quad) {
        gx_weights27(cw, w);
        gx_corners27(g, cw.row, cw.jt, ic);
    } else {
        gx_weights(g, cw, w);
        nc = gx_corners(g, cw.key, ic);
    }
    for (int k = 0; k < nc; k++) {
        if (ic[k] < 0) continue;
        const float4 f = F[ic[k]];
        a[0] += f.x * w[k];
        a[1] += f.y * w[k];
        a[2] += f.z * w[k];
        pgrid += f.w * w[k];
    }
    if (g.halo == 1) {
        float r2 = x * x + y * y + ((g.ndim == 3) ? z * z : 0.f);
        float rr = sqrtf(r2);
        float fr = -g.halo_v2 * rr / (r2 + g.halo_rc2);
        if (fr != 0.f) {
            fr /= rr;
            a[0] += fr * x;
            a[1] += fr * y;
            if (g.ndim == 3) a[2] += fr * z;
        }
        phalo = 0.5f * g.halo_v2 * logf(1.f + r2 / g.halo_rc2);
    } else if (g.halo == 2) {
        gx_disc_force(g, x, y, z, a[0], a[1], a[2], phalo);
    }
}

// with time-step zones: the acceleration of a zone's own step
// (getacc.f:141-150, x nstep^2); none off the grid.  Returns the zone's
// step factor.
__device__ __forceinline__ float zone_scale(const ZoneTab& zt, const int32_t* __restrict__ zone,
                                            int64_t i, float* a, float& pg, float& ph) {
    if (!zone) return 1.f;
    const int iz = zone[i];
    const float t = (float)zt.nstep[min(iz, zt.nz) - 1];
    if (iz > zt.nz) {
        a[0] = a[1] = a[2] = 0.f;
        pg = ph = 0.f;
    } else if (iz > 1) {
        for (int d = 0; d < 3; d++) a[d] *= t * t;
    }
    return t;
}

// tmcgrp.f (RVLF): v <- v - fac * a, fac = +1/2 to start, -1/2 to undo
__global__ void k_tmcent(DevGeo g, float* __restrict__ P, int64_t cap, int64_t n,
                         const float4* __restrict__ F, float fac, const int32_t* __restrict__ zone,
                         ZoneTab zt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nd = g.ndim;
    float z = (nd == 3) ? P[2 * cap + i] : 0.f;
    float a[3], pg, ph;
    accel_parts(g, F, P[i], P[cap + i], z, a, pg, ph);
    zone_scale(zt, zone, i, a, pg, ph);
    for (int d = 0; d < nd; d++) P[(nd + d) * cap + i] -= fac * a[d];
}

// per-block FP64 partial sums of the icheck integrals (icheck.f:61-92) with
// time-centred velocities v + a/2 (cencds.f:38-48): ke, pe, lz, virial,
// a2_re, a2_im, mass, count
#define NDSUM 8
__global__ void k_icheck(DevGeo g, const float* __restrict__ P, int64_t cap, int64_t n,
                         const float4* __restrict__ F, double pm, double* __restrict__ part,
                         const int32_t* __restrict__ zone, ZoneTab zt) {
    __shared__ double sh[NDSUM][256];
    double acc[NDSUM] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int nd = g.ndim;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        float x = P[i], y = P[cap + i], z = (nd == 3) ? P[2 * cap + i] : 0.f;
        float a[3], pg, ph;
        accel_parts(g, F, x, y, z, a, pg, ph);
        CellW cw = gx_cell(g, x, y, z, true);
        if (cw.key < 0) continue;
        // time-centred velocity in base-step units (cencds.f:26-35)
        float az[3] = {a[0], a[1], a[2]};
        const double t = zone_scale(zt, zone, i, az, pg, ph);
        if (zone && zone[i] > zt.nz) a[0] = a[1] = a[2] = 0.f;
        double v[3], q[3] = {x, y, z};
        for (int d = 0; d < nd; d++)
            v[d] = ((double)P[(nd + d) * cap + i] + 0.5 * (double)az[d]) / t;
        double ke = 0, vir = 0;
        for (int d = 0; d < nd; d++) {
            ke += v[d] * v[d];
            vir += q[d] * (double)a[d];
        }
        acc[0] += pm * ke;
        acc[1] += 0.5 * pm * (double)pg + pm * (double)ph;
        acc[2] += pm * (v[1] * q[0] - v[0] * q[1]);
        acc[3] += pm * vir;
        double r2 = q[0] * q[0] + q[1] * q[1];
        if (r2 > 0) {
            acc[4] += pm * (q[0] * q[0] - q[1] * q[1]) / r2;
            acc[5] += pm * 2.0 * q[0] * q[1] / r2;
        }
        acc[6] += pm;
        acc[7] += 1.0;
    }
    for (int k = 0; k < NDSUM; k++) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < NDSUM; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < NDSUM; k++) part[blockIdx.x * NDSUM + k] = sh[k][0];
}

// FP64 path versions
__global__ void k64_tmcent(DevGeo g, double* __restrict__ P, int64_t cap, int64_t n,
                           const double* __restrict__ acc, double fac) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int d = 0; d < g.ndim; d++) P[(g.ndim + d) * cap + i] -= fac * acc[d * cap + i];
}

int gx_fp64_getacc(GxCtx* c, float* acc, float* pot);

extern "C" int gx_tmcent(GxCtx* c, int start) {
    if (!c) return GX_ERR_ARG;
    if (!c->have_field) return c->err = "no fields (call gx_findf)", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    const int64_t n = c->n;
    if (n == 0) return GX_OK;
    const float fac = start ? 0.5f : -0.5f;
    int rc = gx_dense(c);
    if (rc) return rc;
    if (c->fp64) {
        std::vector<float> tmp((size_t)c->g.ndim * n);
        rc = gx_fp64_getacc(c, tmp.data(), nullptr);  // fills acc64
        if (rc) return rc;
        k64_tmcent<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, c->p64, c->cap, n,
                                                                      c->acc64, (double)fac);
    } else {
        k_tmcent<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
            c->g, c->pbuf[c->cur], c->cap, n, c->field, fac,
            c->nzones > 1 ? c->pzone[c->cur] : nullptr, c->zt);
    }
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

extern "C" int gx_icheck(GxCtx* c, GxDiag* d) {
    if (!c || !d) return GX_ERR_ARG;
    if (!c->have_field) return c->err = "no fields (call gx_findf with lpot)", GX_ERR_STATE;
    if (c->fp64) return c->err = "gx_icheck runs on the mixed path", GX_ERR_ARG;
    cudaSetDevice(c->dev);
    int rc = gx_dense(c);
    if (rc) return rc;
    const int nb = 148 * 4;
    double* part = nullptr;
    GX_CUDA(c, cudaMallocAsync((void**)&part, sizeof(double) * NDSUM * nb, c->stream));
    k_icheck<<<nb, 256, 0, c->stream>>>(c->g, c->pbuf[c->cur], c->cap, c->n, c->field,
                                        (double)c->cfg.pmass, part,
                                        c->nzones > 1 ? c->pzone[c->cur] : nullptr, c->zt);
    GX_LAUNCHED(c);
    std::vector<double> h((size_t)NDSUM * nb);
    GX_CUDA(c, cudaMemcpyAsync(h.data(), part, sizeof(double) * NDSUM * nb, cudaMemcpyDeviceToHost,
                               c->stream));
    GX_CUDA(c, cudaFreeAsync(part, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    double s[NDSUM] = {0};
    for (int b = 0; b < nb; b++)
        for (int k = 0; k < NDSUM; k++) s[k] += h[(size_t)b * NDSUM + k];
    d->ke = s[0];
    d->pe = s[1];
    d->lz = s[2];
    d->virial = s[3];
    d->a2_re = s[6] > 0 ? s[4] / s[6] : 0.0;
    d->a2_im = s[6] > 0 ? s[5] / s[6] : 0.0;
    d->n_on_grid = (int64_t)s[7];
    return GX_OK;
}

// ---------------------------------------------------------------------------
// danl (densty.f:82-118, 190-250): the mass projected onto one plane, as a
// surface density (ring i spans grofu(i - 1/2) .. grofu(i + 1/2), the first
// from grofu(0)), Fourier-analysed ring by ring; per ring the m = 0 term
// (the sum over spokes) and, for m = 1 .. ng - 1, the cosine and sine sums
// over it (zero where the ring is empty or the m = 0 term is below 1e-6 of
// them).  One block per ring, FP64 sums.
template <typename T>
__global__ void k_danl(DevGeo g, const T* __restrict__ mass, const float* __restrict__ cfac,
                       float* __restrict__ w) {
    extern __shared__ double sig[];  // [na]
    __shared__ double red[2][32];
    const int ir = blockIdx.x, na = g.na, ngz = (g.ndim == 3) ? g.ngz : 1, ng = g.ng;
    const double c = (double)cfac[ir];
    for (int j = threadIdx.x; j < na; j += blockDim.x) {
        double s = 0.0;
        for (int iz = 0; iz < ngz; iz++) s += (double)mass[((size_t)ir * ngz + iz) * na + j];
        sig[j] = c * s;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    double c0 = 0.0;
    for (int m = 0; m < ng; m++) {
        double a = 0.0, b = 0.0;
        for (int j = threadIdx.x; j < na; j += blockDim.x) {
            const int mj = (int)(((int64_t)m * j) % na);
            double sn, cs;
            sincospi(2.0 * (double)mj / (double)na, &sn, &cs);
            a += sig[j] * cs;
            b += sig[j] * sn;
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            red[0][warp] = a;
            red[1][warp] = b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            a = b = 0.0;
            for (int k = 0; k < nwarp; k++) {
                a += red[0][k];
                b += red[1][k];
            }
            float re = 0.f, im = 0.f;
            if (m == 0) {
                c0 = a;
                re = (float)a;
            } else if (c0 > 0.0 && c0 > 1e-6 * fmax(fabs(a), fabs(b))) {
                re = (float)(a / c0);
                im = (float)(b / c0);
            }
            w[(size_t)ir * ng + m] = re;
            w[(size_t)ng * g.nr + (size_t)ir * ng + m] = im;
        }
        __syncthreads();
    }
}

extern "C" int gx_danl(GxCtx* c, double sigmaf, float* w) {
    if (!c || !w || !(sigmaf > 0.0)) return GX_ERR_ARG;
    if (!c->have_mass) return c->err = "no mass array (call gx_masset)", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    const DevGeo& g = c->g;
    // surface-density factor of every ring: sigmaf / area, area = alpha/2 (r2^2 - r1^2)
    std::vector<float> cf(g.nr);
    auto grofu = [&](float u) {
        return (g.rmap == GX_RMAP_STDPOL) ? expf(g.ua * u) - 1.f : expf(g.ua * (u - g.uoffs));
    };
    float r1 = grofu(0.f);
    for (int i = 0; i < g.nr; i++) {
        const float r2 = grofu((float)(i + 1) - 0.5f);
        const float area = 0.5f * g.alpha * (r2 * r2 - r1 * r1);
        cf[i] = (float)(sigmaf / (double)area);
        r1 = r2;
    }
    const size_t nw = (size_t)2 * g.ng * g.nr;
    float *dc = nullptr, *dw = nullptr;
    GX_CUDA(c, cudaMallocAsync((void**)&dc, sizeof(float) * g.nr, c->stream));
    GX_CUDA(c, cudaMallocAsync((void**)&dw, sizeof(float) * nw, c->stream));
    GX_CUDA(c, cudaMemcpyAsync(dc, cf.data(), sizeof(float) * g.nr, cudaMemcpyHostToDevice, c->stream));
    const size_t sm = sizeof(double) * g.na;
    if (c->fp64)
        k_danl<double><<<g.nr, 128, sm, c->stream>>>(g, c->mass64, dc, dw);
    else
        k_danl<float><<<g.nr, 128, sm, c->stream>>>(g, c->mass, dc, dw);
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaMemcpyAsync(w, dw, sizeof(float) * nw, cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaFreeAsync(dc, c->stream));
    GX_CUDA(c, cudaFreeAsync(dw, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}
