// gx_solve.cu -- field solve of the mixed-precision path (findf).
//
//   k_fwd3 / k_fwd2   p3manl.f:62-109 / p2manl.f:32-45: per ring, the
//                     azimuthal real DFT of every plane restricted to the
//                     active harmonics (the m = 0 term summed in FP64), then
//                     (3D) the zero-padded length-2 ngz vertical DFT.  Both
//                     are small GEMMs against twiddle matrices held in
//                     shared memory; only the active harmonics are formed.
//   k_conv            p3conv.f:137-230 / p2conv.f:114-181: for every
//                     (harmonic, vertical wavenumber) the dense radial
//                     contraction with the FP32 Green table of each field
//                     type, the Green matrix streamed from HBM once per step.
//   synthesis         p3fsyn.f / p2fsyn.f fused with polcat: gx_synth.cu.
// FFTPACK conventions (SRC/utils/sfftpack): forward a_m = sum x cos,
// b_m = -sum x sin; backward x_j = a_0 + (-1)^j a_N + 2 sum (a cos - b sin).
#include <algorithm>

#include "gx_common.cuh"

__constant__ int c_act_m[260];

__host__ __device__ static inline int ru4(int x) { return (x + 3) & ~3; }

// C[M][N] = A[M][K] * B[K][N] in shared memory, 4x4 register tiles.
// A rows are read up to ru4(M) (must be addressable), B is read as float4
// rows (ldb % 4 == 0, columns up to ru4(N) addressable).  epi(r0, c0, acc)
// receives each tile.
template <class Epi>
__device__ __forceinline__ void sgemm44(int M, int N, int K, const float* A, int lda,
                                        const float* B, int ldb, Epi epi) {
    const int tilesN = (N + 3) >> 2, tilesM = (M + 3) >> 2, nt = tilesM * tilesN;
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        const int tm = t / tilesN, tn = t - tm * tilesN;
        const int r0 = tm * 4, c0 = tn * 4;
        float acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
        const float* ap = A + (size_t)r0 * lda;
        const float* bp = B + c0;
#pragma unroll 4
        for (int k = 0; k < K; k++) {
            const float4 b = *reinterpret_cast<const float4*>(bp + (size_t)k * ldb);
            const float a0 = ap[k], a1 = ap[lda + k], a2 = ap[2 * lda + k], a3 = ap[3 * lda + k];
            acc[0][0] += a0 * b.x; acc[0][1] += a0 * b.y; acc[0][2] += a0 * b.z; acc[0][3] += a0 * b.w;
            acc[1][0] += a1 * b.x; acc[1][1] += a1 * b.y; acc[1][2] += a1 * b.z; acc[1][3] += a1 * b.w;
            acc[2][0] += a2 * b.x; acc[2][1] += a2 * b.y; acc[2][2] += a2 * b.z; acc[2][3] += a2 * b.w;
            acc[3][0] += a3 * b.x; acc[3][1] += a3 * b.y; acc[3][2] += a3 * b.z; acc[3][3] += a3 * b.w;
        }
        epi(r0, c0, acc);
    }
}

// forward azimuthal twiddles T[j][2a] = cos(2 pi m_a j / na), T[j][2a+1] = -sin(...)
__device__ void build_taz(float* T, int na, int nact, int ncp) {
    for (int i = threadIdx.x; i < na * ncp; i += blockDim.x) {
        int j = i / ncp, c = i - j * ncp;
        float v = 0.f;
        if (c < 2 * nact) {
            int m = c_act_m[c >> 1];
            int idx = (int)(((int64_t)m * j) % na);
            float s, co;
            sincospif(2.0f * (float)idx / (float)na, &s, &co);
            v = (c & 1) ? -s : co;
        }
        T[i] = v;
    }
}

// ---------------------------------------------------------------------------
// 3D forward transform, one CTA per active source ring.
__global__ void k_fwd3(DevGeo g, int nact, int ncp, const int32_t* __restrict__ jrk,
                       const float* __restrict__ mass, float4* __restrict__ S) {
    extern __shared__ __align__(16) float sm[];
    const int na = g.na, ngz = g.ngz, nkz = g.nkz, nr = g.nr;
    const int ir = blockIdx.x;
    // only the rings that hold mass are transformed (p3fndf.f:44-57); the
    // others get a zero spectrum so that the sum over ranks stays exact
    if (ir < jrk[0] - 1 || ir > min(jrk[1], nr) - 1) {
        for (int i = threadIdx.x; i < nact * nkz; i += blockDim.x)
            S[(size_t)i * nr + ir] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const int ldx = na + 1;
    const int r0sz = max(ru4(ngz) * ldx, ru4(2 * nkz) * ngz);
    float* X = sm;                       // [ru4(ngz)][na + 1], later Tz [ru4(2 nkz)][ngz]
    float* T = X + r0sz;                 // [na][ncp]
    float* C1 = T + na * ncp;            // [ru4(ngz)][ncp]
    const float* src = mass + (size_t)ir * ngz * na;
    for (int i = threadIdx.x; i < ngz * na; i += blockDim.x) {
        int z = i / na, j = i - z * na;
        X[z * ldx + j] = src[i];
    }
    for (int i = ngz * ldx + threadIdx.x; i < ru4(ngz) * ldx; i += blockDim.x) X[i] = 0.f;
    build_taz(T, na, nact, ncp);
    __syncthreads();
    sgemm44(ngz, ncp, na, X, ldx, T, ncp, [&](int r0, int c0, float (&acc)[4][4]) {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) C1[(r0 + i) * ncp + c0 + j] = acc[i][j];
    });
    __syncthreads();
    // m = 0 (when active) in FP64
    if (c_act_m[0] == 0) {
        for (int z = threadIdx.x; z < ngz; z += blockDim.x) {
            double s = 0.0;
            for (int j = 0; j < na; j++) s += (double)X[z * ldx + j];
            C1[z * ncp] = (float)s;
        }
    }
    __syncthreads();
    // vertical twiddles Tz[2k][z] = cos(pi k z / ngz), Tz[2k+1][z] = -sin(...)
    float* Tz = X;
    for (int i = threadIdx.x; i < ru4(2 * nkz) * ngz; i += blockDim.x) {
        int r = i / ngz, z = i - r * ngz;
        int k = r >> 1;
        float v = 0.f;
        if (k < nkz) {
            int idx = (int)(((int64_t)k * z) % (2 * ngz));
            float s, co;
            sincospif((float)idx / (float)ngz, &s, &co);
            v = (r & 1) ? -s : co;
        }
        Tz[i] = v;
    }
    __syncthreads();
    sgemm44(2 * nkz, ncp, ngz, Tz, ngz, C1, ncp, [&](int r0, int c0, float (&acc)[4][4]) {
        // rows r0 = 2k, 2k+1, 2k+2, 2k+3; cols c0 = 2a, 2a+1, 2a+2, 2a+3
#pragma unroll
        for (int dk = 0; dk < 2; dk++) {
            int k = (r0 >> 1) + dk;
            if (k >= nkz) continue;
#pragma unroll
            for (int da = 0; da < 2; da++) {
                int a = (c0 >> 1) + da;
                if (a >= nact) continue;
                float4 v = make_float4(acc[2 * dk][2 * da], acc[2 * dk + 1][2 * da],
                                       acc[2 * dk][2 * da + 1], acc[2 * dk + 1][2 * da + 1]);
                S[((size_t)a * nkz + k) * nr + ir] = v;
            }
        }
    });
}

// 2D forward transform, RB rings per CTA.
#define RB2 16
__global__ void k_fwd2(DevGeo g, int nact, int ncp, const float* __restrict__ mass,
                       float4* __restrict__ S) {
    extern __shared__ __align__(16) float sm[];
    const int na = g.na, nr = g.nr;
    const int ldx = na + 1;
    const int jr1 = nr - 1;
    const int ir0 = blockIdx.x * RB2;
    float* X = sm;                   // [RB2][na + 1]
    float* T = X + RB2 * ldx;        // [na][ncp]
    for (int i = threadIdx.x; i < RB2 * na; i += blockDim.x) {
        int r = i / na, j = i - r * na;
        int ir = ir0 + r;
        X[r * ldx + j] = (ir <= jr1) ? mass[(size_t)ir * na + j] : 0.f;
    }
    build_taz(T, na, nact, ncp);
    __syncthreads();
    sgemm44(RB2, ncp, na, X, ldx, T, ncp, [&](int r0, int c0, float (&acc)[4][4]) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int ir = ir0 + r0 + i;
            if (ir > jr1) continue;
            double s0 = 0.0;
            bool m0 = (c0 == 0) && (c_act_m[0] == 0);
            if (m0)
                for (int j = 0; j < na; j++) s0 += (double)X[(r0 + i) * ldx + j];
#pragma unroll
            for (int da = 0; da < 2; da++) {
                int a = (c0 >> 1) + da;
                if (a >= nact) continue;
                float av = (m0 && da == 0) ? (float)s0 : acc[i][2 * da];
                S[(size_t)a * nr + ir] = make_float4(av, 0.f, acc[i][2 * da + 1], 0.f);
            }
        }
    });
}

// ---------------------------------------------------------------------------
// radial contraction; grid (nact, nkz); 8 warps split the source rings.
// Types: 0 radial, 1 azimuthal, 2 vertical, 3 potential (p3conv.f:173-226).
template <bool VEC>
__global__ void __launch_bounds__(256) k_conv(DevGeo g, int nact, int tmask,
                                              const float* __restrict__ G,
                                              const float4* __restrict__ S,
                                              float4* __restrict__ O,
                                              const int32_t* __restrict__ jrk) {
    extern __shared__ __align__(16) float4 sh4[];
    const int nr = g.nr, nkz = g.nkz, ng = g.ng, mmax = g.mmax, ngz = g.ngz;
    // source rings jrs..krs (p3conv.f:149-150)
    const int js = max(jrk[0], 1) - 1, ks = min(jrk[1], nr) - 1;
    const int a = blockIdx.x, k = blockIdx.y, m = c_act_m[a];
    float4* Sin = sh4;              // [nr]
    float4* part = sh4 + nr;        // [8][nr]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < nr; i += blockDim.x)
        Sin[i] = (i >= js && i <= ks) ? S[((size_t)a * nkz + k) * nr + i] : make_float4(0, 0, 0, 0);
    __syncthreads();
    for (int t = 0; t < 4; t++) {
        if (!((tmask >> t) & 1)) continue;
        bool valid = true;
        if (t == 1) valid = (m >= 1) && (m <= min(ng, mmax - 1) - 1);
        if (t == 2) valid = (g.ndim == 3) && (k >= 1) && (k <= ngz - 1);
        float4* out = O + (((size_t)t * nact + a) * nkz + k) * nr;
        if (!valid) {
            for (int i = threadIdx.x; i < nr; i += blockDim.x) out[i] = make_float4(0, 0, 0, 0);
            continue;
        }
        const float* Gt = G + ((((size_t)t * ng + m) * nkz + k) * nr) * (size_t)nr;
        for (int ib = 0; ib < nr; ib += 128) {
            const int ir0 = ib + lane * 4;
            float4 acc[4];
#pragma unroll
            for (int q = 0; q < 4; q++) acc[q] = make_float4(0, 0, 0, 0);
            if (ir0 < nr) {
#pragma unroll 4
                for (int is = js + warp; is <= ks; is += 8) {
                    float gv[4];
                    const float* gp = Gt + (size_t)is * nr + ir0;
                    if (VEC) {
                        float4 g4 = __ldg(reinterpret_cast<const float4*>(gp));
                        gv[0] = g4.x; gv[1] = g4.y; gv[2] = g4.z; gv[3] = g4.w;
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; q++) gv[q] = (ir0 + q < nr) ? __ldg(gp + q) : 0.f;
                    }
                    const float4 s = Sin[is];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float gq = gv[q];
                        if (t == 0 || t == 3) {
                            acc[q].x += gq * s.x; acc[q].y += gq * s.y;
                            acc[q].z += gq * s.z; acc[q].w += gq * s.w;
                        } else if (t == 1) {
                            acc[q].x += gq * s.z; acc[q].z -= gq * s.x;
                            acc[q].y += gq * s.w; acc[q].w -= gq * s.y;
                        } else {
                            acc[q].x += gq * s.y; acc[q].y -= gq * s.x;
                            acc[q].z += gq * s.w; acc[q].w -= gq * s.z;
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; q++)
                    if (ir0 + q < nr) part[warp * nr + ir0 + q] = acc[q];
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            float4 s = part[i];
            for (int w = 1; w < 8; w++) {
                float4 p = part[w * nr + i];
                s.x += p.x; s.y += p.y; s.z += p.z; s.w += p.w;
            }
            out[i] = s;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
static int set_act(GxCtx* c) {
    GX_CUDA(c, cudaMemcpyToSymbolAsync(c_act_m, c->spec.m, sizeof(int) * 260, 0,
                                       cudaMemcpyHostToDevice, c->stream));
    return GX_OK;
}

static size_t fwd3_smem(const DevGeo& g, int ncp) {
    int ldx = g.na + 1;
    int r0sz = std::max(ru4(g.ngz) * ldx, ru4(2 * g.nkz) * g.ngz);
    return sizeof(float) * ((size_t)r0sz + (size_t)g.na * ncp + (size_t)ru4(g.ngz) * ncp);
}
// findf for the mixed path: mass -> field (and optional polar copy)
int gx_mixed_findf(GxCtx* c, int lpot, bool polcat_only_field) {
    const DevGeo& g = c->g;
    const int nact = c->spec.nact;
    if (nact == 0) return c->err = "no active harmonics", GX_ERR_ARG;
    const int ncp = ru4(2 * nact);
    int rc = set_act(c);
    if (rc) return rc;
    float* polar = nullptr;
    if (!polcat_only_field) {
        if (!c->polar) GX_CUDA(c, cudaMalloc((void**)&c->polar, sizeof(float) * 4 * g.mesh));
        polar = c->polar;
    }
    int tmask = 1 | 2 | (g.ndim == 3 ? 4 : 0) | (lpot ? 8 : 0);
    if (g.ng == 1) tmask &= ~2;
    rc = gx_phase_mark(c, PH_FWD);
    if (rc) return rc;
    rc = gx_comm_reduce_range(c);
    if (rc) return rc;
    if (g.ndim == 3) {
        size_t sm = fwd3_smem(g, ncp);
        GX_CUDA(c, cudaFuncSetAttribute(k_fwd3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_fwd3<<<g.nr, 512, sm, c->stream>>>(g, nact, ncp, c->jrk_d, c->mass, c->specS);
        GX_LAUNCHED(c);
    } else {
        size_t sm = sizeof(float) * ((size_t)RB2 * (g.na + 1) + (size_t)g.na * ncp);
        GX_CUDA(c, cudaFuncSetAttribute(k_fwd2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        int nb = (g.nr + RB2 - 1) / RB2;
        k_fwd2<<<nb, 256, sm, c->stream>>>(g, nact, ncp, c->mass, c->specS);
        GX_LAUNCHED(c);
    }
    rc = gx_comm_reduce_spectrum(c);
    if (rc) return rc;
    rc = gx_phase_mark(c, PH_CONV);
    if (rc) return rc;
    {
        size_t sm = sizeof(float4) * (size_t)g.nr * 9;
        dim3 grid(nact, g.nkz);
        bool vec = (g.nr % 4) == 0;
        if (vec) {
            GX_CUDA(c, cudaFuncSetAttribute(k_conv<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            k_conv<true><<<grid, 256, sm, c->stream>>>(g, nact, tmask, c->green32, c->specS, c->specO, c->jrk_d);
        } else {
            GX_CUDA(c, cudaFuncSetAttribute(k_conv<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            k_conv<false><<<grid, 256, sm, c->stream>>>(g, nact, tmask, c->green32, c->specS, c->specO, c->jrk_d);
        }
        GX_LAUNCHED(c);
    }
    rc = gx_phase_mark(c, PH_SYN);
    if (rc) return rc;
    rc = gx_synthesis(c, tmask, polar);
    if (rc) return rc;
    rc = gx_phase_end(c);
    if (rc) return rc;
    c->have_field = true;
    c->field_pot = lpot != 0;
    return GX_OK;
}

// ---------------------------------------------------------------------------
// grid access
__global__ void k_field_comp(const float4* __restrict__ F, float* __restrict__ out, int n, int comp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = F[i];
    out[i] = comp == 0 ? v.x : comp == 1 ? v.y : comp == 2 ? v.z : v.w;
}
__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
__global__ void k_f2d(const float* __restrict__ a, double* __restrict__ b, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}

extern "C" int gx_get_grid(GxCtx* c, int which, float* out) {
    if (!c || !out || which < 0 || which > 6) return GX_ERR_ARG;
    cudaSetDevice(c->dev);
    const int mesh = c->g.mesh;
    float* tmp = nullptr;
    GX_CUDA(c, cudaMallocAsync((void**)&tmp, sizeof(float) * mesh, c->stream));
    const int bs = 256, nb = (mesh + bs - 1) / bs;
    int rc = GX_OK;
    if (which == GX_GRID_MASS) {
        if (!c->have_mass) rc = GX_ERR_STATE, c->err = "no mass array";
        else if (c->fp64) k_d2f<<<nb, bs, 0, c->stream>>>(c->mass64, tmp, mesh);
        else GX_CUDA(c, cudaMemcpyAsync(tmp, c->mass, sizeof(float) * mesh, cudaMemcpyDeviceToDevice, c->stream));
    } else if (which >= GX_GRID_FR && which <= GX_GRID_POT) {
        int comp = which - GX_GRID_FR;
        if (c->fp64) {
            if (!c->have_field) rc = GX_ERR_STATE, c->err = "no fields";
            else k_d2f<<<nb, bs, 0, c->stream>>>(c->polar64 + (size_t)comp * mesh, tmp, mesh);
        } else if (comp >= 2 && c->have_field) {
            k_field_comp<<<nb, bs, 0, c->stream>>>(c->field, tmp, mesh, comp);
        } else if (!c->polar || !c->have_field) {
            rc = GX_ERR_STATE, c->err = "polar fields need gx_findf_polar";
        } else {
            GX_CUDA(c, cudaMemcpyAsync(tmp, c->polar + (size_t)comp * mesh, sizeof(float) * mesh,
                                       cudaMemcpyDeviceToDevice, c->stream));
        }
    } else {
        int comp = which - GX_GRID_FX;
        if (!c->have_field) rc = GX_ERR_STATE, c->err = "no fields";
        else if (c->fp64) k_d2f<<<nb, bs, 0, c->stream>>>(c->field64 + (size_t)comp * mesh, tmp, mesh);
        else k_field_comp<<<nb, bs, 0, c->stream>>>(c->field, tmp, mesh, comp);
    }
    if (rc == GX_OK) {
        GX_CUDA(c, cudaGetLastError());
        GX_CUDA(c, cudaMemcpyAsync(out, tmp, sizeof(float) * mesh, cudaMemcpyDeviceToHost, c->stream));
    }
    GX_CUDA(c, cudaFreeAsync(tmp, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return rc;
}

extern "C" int gx_set_mass(GxCtx* c, const float* mass) {
    if (!c || !mass) return GX_ERR_ARG;
    cudaSetDevice(c->dev);
    const DevGeo& g = c->g;
    const int mesh = g.mesh;
    // active ring range of the installed masses (p3ckst.f sets jrad/krad)
    int jr = g.nr, kr = 0;
    const int per = g.ngz * g.na;
    for (int ir = 0; ir < g.nr; ir++)
        for (int i = 0; i < per; i++)
            if (mass[(size_t)ir * per + i] != 0.f) {
                jr = std::min(jr, ir + 1);
                kr = std::max(kr, ir + 1);
                break;
            }
    c->jrs = jr;
    c->krs = kr;
    int32_t jrk[2] = {jr, kr};
    GX_CUDA(c, cudaMemcpyAsync(c->jrk_d, jrk, sizeof jrk, cudaMemcpyHostToDevice, c->stream));
    if (c->fp64) {
        float* tmp = nullptr;
        GX_CUDA(c, cudaMallocAsync((void**)&tmp, sizeof(float) * mesh, c->stream));
        GX_CUDA(c, cudaMemcpyAsync(tmp, mass, sizeof(float) * mesh, cudaMemcpyHostToDevice, c->stream));
        k_f2d<<<(mesh + 255) / 256, 256, 0, c->stream>>>(tmp, c->mass64, mesh);
        GX_LAUNCHED(c);
        GX_CUDA(c, cudaFreeAsync(tmp, c->stream));
    } else {
        GX_CUDA(c, cudaMemcpyAsync(c->mass, mass, sizeof(float) * mesh, cudaMemcpyHostToDevice, c->stream));
    }
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_mass = true;
    c->have_field = false;
    return GX_OK;
}
