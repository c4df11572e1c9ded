// gx_green.cu -- Green-table construction on the device in FP64 (greenm).
//
// Restates p2grnm (SRC/lib15/p2grnm.f:99-203) and p3grnm
// (SRC/lib15/p3grnm.f:94-263): the softened kernels radfor/azifor/vrtfor/
// grnfun (radfor.f:25-38, azifor.f:25-37, vrtfor.f, sftpot.f:20-37,
// softm.f:15-27) are sampled at the spoke angles and plane separations,
// cosine- or sine-transformed in angle (FFTPACK rcost/rsint conventions,
// unnormalised, i.e. the full-circle DFT of the even/odd kernel), filtered
// (m >= ng and skipped harmonics dropped), and in 3D cosine- or
// sine-transformed over the ngz + 1 plane separations (the doubled-grid
// vertical convolution).  Layout [type][m][kz][is][ir] (ir fastest; the
// record layout of p3gwrt.f:47-64).  The reference builds in FP32 and
// re-reads the table from its .grt file every step; here it is built once
// in FP64 and kept resident (FP32 copy for the mixed path).
#include "gx_common.cuh"

struct KerParams {
    int tsoft;
    double softl, softl2;
};

__device__ __forceinline__ double softm_d(double ds) {
    if (ds <= 0.0) return 0.0;
    if (ds < 1.0) return 4.0 * ds * ds * ds * (0.333333333 - 0.3 * ds * ds + 0.125 * ds * ds * ds);
    if (ds < 2.0)
        return -1.0 / 15.0 +
               ds * ds * ds * (2.6666667 - 3.0 * ds + 1.2 * ds * ds - 0.166666667 * ds * ds * ds);
    return 1.0;
}

// kernel of component `type` at field (rf, th, zf) from a unit source at (rs, 0, 0)
__device__ __forceinline__ double kernel_d(const KerParams& k, int type, double rs, double rf,
                                           double cth, double sth, double zf) {
    double d2 = rs * rs + rf * rf - 2.0 * rs * rf * cth + zf * zf;
    if (type == 3) {  // grnfun -> sftpot
        if (k.tsoft == GX_SOFT_PLUMMER) return -1.0 / sqrt(d2 + k.softl2);
        double x = sqrt(d2) / k.softl;
        if (x <= 0.0) return -1.4 / k.softl;
        if (x < 1.0) return (-1.4 + x * x * (0.6666667 - 0.3 * x * x + 0.1 * x * x * x)) / k.softl;
        if (x < 2.0)
            return (-1.6 + 1.0 / (15.0 * x) +
                    x * x * (1.33333333 - x + 0.3 * x * x - 0.033333333 * x * x * x)) /
                   k.softl;
        return -1.0 / sqrt(d2);
    }
    double num = (type == 0) ? (rs * cth - rf) : (type == 1) ? (-rs * sth) : (-zf);
    if (k.tsoft == GX_SOFT_PLUMMER) {
        double v = d2 + k.softl2;
        return num / (v * sqrt(v));
    }
    if (type == 2 ? (zf == 0.0) : !(d2 > 0.0)) return 0.0;
    return num * softm_d(sqrt(d2) / k.softl) / (d2 * sqrt(d2));
}

__device__ __forceinline__ double grofu_d(const DevGeo& g, double u) {
    if (g.rmap == GX_RMAP_STDPOL) return exp(g.ua_d * u) - 1.0;
    return exp(g.ua_d * (u - g.uoffs_d));
}

// Stage 1: angular transform.  One thread per (type, is, ir, iz); it
// samples the kernel at every needed angle and accumulates the harmonics
// m < ng.  Output tmp[type][m][iz][is][ir] (iz over the plane separations
// 0..nkz-1 of that type; unused slots stay zero).
template <int NM>
__global__ void k_green_theta(DevGeo g, KerParams kp, const uint8_t* __restrict__ lg,
                              double* __restrict__ tmp, int type) {
    const int nr = g.nr, na = g.na, ng = g.ng, nkz = g.nkz, mmax = g.mmax;
    int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t total = (int64_t)nkz * nr * nr;
    if (tid >= total) return;
    int ir = tid % nr;
    int is = (tid / nr) % nr;
    int iz = (int)(tid / ((int64_t)nr * nr));
    const bool azim = (type == 1), vert = (type == 2);
    if (g.ndim == 3 && vert && (iz == 0 || iz == g.ngz)) return;  // odd in z: zero there
    double rs = grofu_d(g, (double)is), rf = grofu_d(g, (double)ir);
    double zf = (g.ndim == 3) ? g.dzg_d * (double)iz : 0.0;
    double acc[NM];
    const int nm = ng < NM ? ng : NM;
#pragma unroll
    for (int m = 0; m < NM; m++) acc[m] = 0.0;
    // angles theta_k = 2 pi k / na, k = 0 .. na/2 (cosine types) or 1 .. na/2-1 (sine type)
    const int k1 = azim ? 1 : 0, k2 = azim ? mmax - 2 : mmax - 1;
    for (int k = k1; k <= k2; k++) {
        double sth, cth;
        sincospi(2.0 * (double)k / (double)na, &sth, &cth);
        double f = kernel_d(kp, type, rs, rf, cth, sth, zf);
        // weight of sample k: rcost end points count once, interior twice;
        // rsint interior points twice
        double wk = (!azim && (k == 0 || k == mmax - 1)) ? 1.0 : 2.0;
        double fw = f * wk;
        // harmonics by angle-addition recurrence on (cos m th, sin m th)
        double cm = 1.0, sm = 0.0;
#pragma unroll
        for (int m = 0; m < NM; m++) {
            acc[m] += azim ? fw * sm : fw * cm;
            double cn = cm * cth - sm * sth;
            sm = sm * cth + cm * sth;
            cm = cn;
        }
    }
#pragma unroll
    for (int m = 0; m < NM; m++) {
        if (m >= nm) break;
        bool drop = (m >= ng) || lg[m];
        if (g.ndim == 2) drop = (m >= ng) || (m % g.nsect != 0);
        if (azim && (m == 0 || m >= mmax - 1)) drop = true;
        double v = drop ? 0.0 : acc[m];
        tmp[((((int64_t)type * ng + m) * nkz + iz) * nr + is) * nr + ir] = v;
    }
}

// Stage 2 (3D): vertical transform over the ngz + 1 plane separations.
// One thread per (type, m, is, ir).  Cosine types: FFTPACK rcost on
// nkz = ngz + 1 points; vertical force: rsint on the ngz - 1 interior points.
__global__ void k_green_z(DevGeo g, const double* __restrict__ tmp, double* __restrict__ G,
                          int type) {
    const int nr = g.nr, ng = g.ng, nkz = g.nkz, ngz = g.ngz;
    extern __shared__ double tw[];  // tw[i] = cos(pi i / ngz), tw[2 ngz + i] = sin(pi i / ngz)
    for (int i = threadIdx.x; i < 2 * ngz; i += blockDim.x) {
        double sn, cs;
        sincospi((double)i / (double)ngz, &sn, &cs);
        tw[i] = cs;
        tw[2 * ngz + i] = sn;
    }
    __syncthreads();
    int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t total = (int64_t)ng * nr * nr;
    if (tid >= total) return;
    int ir = tid % nr;
    int is = (tid / nr) % nr;
    int m = (int)(tid / ((int64_t)nr * nr));
    const double* src = tmp + (((int64_t)type * ng + m) * nkz) * nr * nr + (int64_t)is * nr + ir;
    double* dst = G + (((int64_t)type * ng + m) * nkz) * nr * nr + (int64_t)is * nr + ir;
    const int64_t st = (int64_t)nr * nr;
    const bool vert = (type == 2);
    for (int kz = 0; kz <= ngz; kz++) {
        double s = 0.0;
        if (!vert) {
            s = src[0] + ((kz & 1) ? -src[ngz * st] : src[ngz * st]);
            int idx = kz;
            for (int j = 1; j < ngz; j++) {
                s += 2.0 * src[j * st] * tw[idx];
                idx += kz;
                if (idx >= 2 * ngz) idx -= 2 * ngz;
            }
        } else if (kz > 0 && kz < ngz) {
            int idx = kz;
            for (int j = 1; j < ngz; j++) {
                s += 2.0 * src[j * st] * tw[2 * ngz + idx];
                idx += kz;
                if (idx >= 2 * ngz) idx -= 2 * ngz;
            }
        }
        dst[kz * st] = s;
    }
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

int gx_green_build_dev(GxCtx* c) {
    const DevGeo& g = c->g;
    if (g.ng > 64) return c->err = "ng > 64 not supported by the Green builder", GX_ERR_RANGE;
    const int64_t per = (int64_t)g.ng * g.nkz * g.nr * g.nr;
    const int64_t total = 4 * per;
    KerParams kp;
    kp.tsoft = g.tsoft;
    kp.softl = (double)c->cfg.softl;
    kp.softl2 = kp.softl * kp.softl;
    uint8_t* lg = nullptr;
    double* tmp = nullptr;
    double* G64 = nullptr;
    GX_CUDA(c, cudaMallocAsync((void**)&lg, 260, c->stream));
    GX_CUDA(c, cudaMemcpyAsync(lg, c->geo.lg, 260, cudaMemcpyHostToDevice, c->stream));
    GX_CUDA(c, cudaMallocAsync((void**)&tmp, sizeof(double) * total, c->stream));
    GX_CUDA(c, cudaMemsetAsync(tmp, 0, sizeof(double) * total, c->stream));
    for (int type = 0; type < 4; type++) {
        if (g.ndim == 2 && type == 2) continue;
        if (type == 1 && g.ng == 1) continue;
        int64_t nt = (int64_t)g.nkz * g.nr * g.nr;
        int bs = 128;
        unsigned nb = (unsigned)((nt + bs - 1) / bs);
        if (g.ng <= 8) k_green_theta<8><<<nb, bs, 0, c->stream>>>(g, kp, lg, tmp, type);
        else if (g.ng <= 16) k_green_theta<16><<<nb, bs, 0, c->stream>>>(g, kp, lg, tmp, type);
        else if (g.ng <= 32) k_green_theta<32><<<nb, bs, 0, c->stream>>>(g, kp, lg, tmp, type);
        else k_green_theta<64><<<nb, bs, 0, c->stream>>>(g, kp, lg, tmp, type);
        GX_LAUNCHED(c);
    }
    if (g.ndim == 3) {
        GX_CUDA(c, cudaMallocAsync((void**)&G64, sizeof(double) * total, c->stream));
        GX_CUDA(c, cudaMemsetAsync(G64, 0, sizeof(double) * total, c->stream));
        for (int type = 0; type < 4; type++) {
            if (type == 1 && g.ng == 1) continue;
            int64_t nt = (int64_t)g.ng * g.nr * g.nr;
            int bs = 128;
            k_green_z<<<(unsigned)((nt + bs - 1) / bs), bs, sizeof(double) * 4 * g.ngz,
                        c->stream>>>(g, tmp, G64, type);
            GX_LAUNCHED(c);
        }
        GX_CUDA(c, cudaFreeAsync(tmp, c->stream));
    } else {
        G64 = tmp;
    }
    if (c->fp64) {
        if (c->green64) cudaFree(c->green64);
        c->green64 = G64;
    } else {
        if (!c->green32) GX_CUDA(c, cudaMalloc((void**)&c->green32, sizeof(float) * total));
        int bs = 256;
        k_to_f32<<<(unsigned)((total + bs - 1) / bs), bs, 0, c->stream>>>(G64, c->green32, total);
        GX_LAUNCHED(c);
        GX_CUDA(c, cudaFreeAsync(G64, c->stream));
    }
    GX_CUDA(c, cudaFreeAsync(lg, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_green = true;
    return GX_OK;
}
