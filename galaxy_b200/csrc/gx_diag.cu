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
        gx_corners27(g, cw.key, ic);
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
    if (c->fp64) {
        std::vector<float> tmp((size_t)c->g.ndim * n);
        int rc = gx_fp64_getacc(c, tmp.data(), nullptr);  // fills acc64
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
