// gx_synth.cu -- field synthesis of the mixed path (p3fsyn.f:59-129,
// p2fsyn.f:34-56) fused with polcat (polcat.f:22-41).
//
// The inverse transforms are small GEMMs against twiddle tables built once
// per context; both exploit the symmetry of a real inverse DFT:
//   k_synz   vertical synthesis r(z) = sum_k A_k wA(k,z) + B_k wB(k,z) over
//            the ngz + 1 wavenumbers of the doubled grid, only for the
//            physical planes.  With E/O the sums over even/odd k,
//            r(z) = EA + OA + EB + OB and r(ngz - z) = EA - OA - EB + OB, so
//            each pass of the k loop yields two planes.
//   k_synaz  azimuthal synthesis with the 1/(2 ngz na) (2D: 1/na) scale:
//            C = sum_a (a_m 2cos m th), S = sum_a (b_m (-2 sin m th)),
//            f(j) = C + S and f(na - j) = C - S; then the rotation to
//            (fx, fy) and one float4 (fx, fy, fz, phi) store per node.
#include <algorithm>

#include "gx_common.cuh"

struct ActList {
    int m[64];
};

struct SynTab {
    const float* WAe;  // [KE][ru4(Z0)]  wA(2i, z), the planes of one wavenumber contiguous
    const float* WBe;  // [KE][ru4(Z0)]  wB(2i, z)
    const float* WAo;  // [KO][ru4(Z0)]  wA(2i+1, z)
    const float* WBo;  // [KO][ru4(Z0)]  wB(2i+1, z)
    const float* TC;   // [nact][njp]    cosine row weights (scaled)
    const float* TS;   // [nact][njp]    sine row weights (scaled)
    const float* CS;   // [2][njp]       cos, sin of the spoke angles 2 pi j / na (polcat)
    int Z0, KE, KO, njp;
};

__host__ __device__ static inline int ru4s(int x) { return (x + 3) & ~3; }

static void syn_dims(const DevGeo& g, int& Z0, int& KE, int& KO, int& njp) {
    Z0 = g.ngz / 2 + 1;
    KE = g.ngz / 2 + 1;          // k = 0, 2, ..., <= ngz
    KO = (g.ngz + 1) / 2;        // k = 1, 3, ..., <= ngz
    njp = ru4s(g.na / 2 + 1);
}

__device__ __forceinline__ float wA(int k, int z, int ngz) {
    if (k == 0) return 1.f;
    if (k == ngz) return (z & 1) ? -1.f : 1.f;
    int idx = (int)(((int64_t)k * z) % (2 * ngz));
    return 2.f * cospif((float)idx / (float)ngz);
}
__device__ __forceinline__ float wB(int k, int z, int ngz) {
    if (k <= 0 || k >= ngz) return 0.f;
    int idx = (int)(((int64_t)k * z) % (2 * ngz));
    return -2.f * sinpif((float)idx / (float)ngz);
}

__global__ void k_syntab(DevGeo g, ActList act, int nact, float scale, float* WAe, float* WBe,
                         float* WAo, float* WBo, float* TC, float* TS, float* CS, int Z0, int KE,
                         int KO, int njp) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nz = ru4s(Z0);
    if (tid < nz * KE) {
        int i = tid / nz, z = tid - i * nz;
        WAe[tid] = (z < Z0) ? wA(2 * i, z, g.ngz) : 0.f;
        WBe[tid] = (z < Z0) ? wB(2 * i, z, g.ngz) : 0.f;
    }
    if (tid < nz * KO) {
        int i = tid / nz, z = tid - i * nz;
        WAo[tid] = (z < Z0) ? wA(2 * i + 1, z, g.ngz) : 0.f;
        WBo[tid] = (z < Z0) ? wB(2 * i + 1, z, g.ngz) : 0.f;
    }
    if (tid < njp) {
        float sn = 0.f, cs = 1.f;
        if (tid <= g.na / 2) sincospif(2.0f * (float)tid / (float)g.na, &sn, &cs);
        CS[tid] = cs;
        CS[njp + tid] = sn;
    }
    if (tid < nact * njp) {
        int a = tid / njp, j = tid - a * njp;
        int m = act.m[a];
        float c = 0.f, s = 0.f;
        if (j <= g.na / 2) {
            int idx = (int)(((int64_t)m * j) % g.na);
            float sn, cs;
            sincospif(2.0f * (float)idx / (float)g.na, &sn, &cs);
            if (m == 0) c = 1.f;
            else if (m == g.mmax - 1) c = (j & 1) ? -1.f : 1.f;
            else {
                c = 2.f * cs;
                s = -2.f * sn;
            }
        }
        TC[tid] = c * scale;
        TS[tid] = s * scale;
    }
}

// vertical synthesis, one CTA per (ring, field type); R[t][ir][z][ncp]
#define SYNZ_THREADS 576
__global__ void __launch_bounds__(SYNZ_THREADS) k_synz(DevGeo g, int nact, int ncp, int tmask,
                                             const float4* __restrict__ O, SynTab tb,
                                             float* __restrict__ R) {
    extern __shared__ __align__(16) float sm[];
    const int ir = blockIdx.x, t = blockIdx.y;
    if (!((tmask >> t) & 1)) return;
    const int nr = g.nr, nkz = g.nkz, ngz = g.ngz;
    float* Rt = R + (((size_t)t * nr + ir) * ngz) * ncp;
    const float4* Ot = O + (size_t)t * nact * nkz * nr;
    if (g.ndim == 2) {
        for (int c = threadIdx.x; c < ncp; c += blockDim.x) {
            const int a = c >> 1;
            float v = 0.f;
            if (a < nact) {
                float4 o = Ot[(size_t)a * nr + ir];
                v = (c & 1) ? o.z : o.x;
            }
            Rt[c] = v;
        }
        return;
    }
    const int Z0 = tb.Z0, KE = tb.KE, KO = tb.KO, nz4 = ru4s(Z0);
    float* sWAe = sm;
    float* sWBe = sWAe + nz4 * KE;
    float* sWAo = sWBe + nz4 * KE;
    float* sWBo = sWAo + nz4 * KO;
    float* Ae = sWBo + nz4 * KO;        // [KE][ncp]
    float* Be = Ae + KE * ncp;
    float* Ao = Be + KE * ncp;          // [KO][ncp]
    float* Bo = Ao + KO * ncp;
    // the four twiddle tables are one contiguous block of 2 nz4 (KE + KO)
    // floats in global memory, in the order of the shared copies
    {
        const float4* src = reinterpret_cast<const float4*>(tb.WAe);
        float4* dst = reinterpret_cast<float4*>(sWAe);
        const int n4 = (2 * nz4 * (KE + KO)) >> 2;
        for (int i = threadIdx.x; i < n4; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    // spectrum of this ring: rows k, columns (a-row, b-row) of each harmonic
    for (int i = threadIdx.x; i < nkz * nact; i += blockDim.x) {
        const int k = i / nact, a = i - k * nact;
        const float4 o = Ot[((size_t)a * nkz + k) * nr + ir];
        const int h = k >> 1;
        float* A = (k & 1) ? Ao : Ae;
        float* B = (k & 1) ? Bo : Be;
        A[h * ncp + 2 * a] = o.x;
        B[h * ncp + 2 * a] = o.y;
        A[h * ncp + 2 * a + 1] = o.z;
        B[h * ncp + 2 * a + 1] = o.w;
    }
    for (int i = threadIdx.x; i < (KE + KO) * (ncp - 2 * nact); i += blockDim.x) {
        const int w = ncp - 2 * nact;
        const int h = i / w, c = 2 * nact + (i - h * w);
        if (h < KE) {
            Ae[h * ncp + c] = 0.f;
            Be[h * ncp + c] = 0.f;
        } else {
            Ao[(h - KE) * ncp + c] = 0.f;
            Bo[(h - KE) * ncp + c] = 0.f;
        }
    }
    __syncthreads();
    // 4x4 tiles of (z, column); the four sums of a tile (even/odd kz x A/B
    // part) go to four adjacent lanes, recombined by shuffles:
    // lo = EA + OA + EB + OB, hi = EA - OA - EB + OB
    const int tilesN = ncp >> 2, tilesM = nz4 >> 2, nt = tilesM * tilesN;
    const int per = blockDim.x / 4, role = threadIdx.x & 3;
    const float* Sp = (role == 0) ? Ae : (role == 1) ? Be : (role == 2) ? Ao : Bo;
    const float* Wp = (role == 0) ? sWAe : (role == 1) ? sWBe : (role == 2) ? sWAo : sWBo;
    const int KR = (role < 2) ? KE : KO;
    const float hs = (role == 0 || role == 3) ? 1.f : -1.f;
    for (int t0 = 0; t0 < nt; t0 += per) {
        const int tile = t0 + threadIdx.x / 4;
        const bool act = tile < nt;
        const int tm = act ? tile / tilesN : 0, tn = act ? tile - tm * tilesN : 0;
        const int z0 = tm * 4, c0 = tn * 4;
        float acc[4][4];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[r][q] = 0.f;
        const int kr = act ? KR : 0;
#pragma unroll 4
        for (int i = 0; i < kr; i++) {
            const float4 v = *reinterpret_cast<const float4*>(Sp + i * ncp + c0);
            const float4 w4 = *reinterpret_cast<const float4*>(Wp + i * nz4 + z0);
            const float w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int r = 0; r < 4; r++) {
                acc[r][0] += w[r] * v.x; acc[r][1] += w[r] * v.y; acc[r][2] += w[r] * v.z; acc[r][3] += w[r] * v.w;
            }
        }
        float lo[4][4], hi[4][4];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                lo[r][q] = acc[r][q];
                hi[r][q] = hs * acc[r][q];
            }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1)
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    lo[r][q] += __shfl_xor_sync(0xffffffffu, lo[r][q], o);
                    hi[r][q] += __shfl_xor_sync(0xffffffffu, hi[r][q], o);
                }
        if (!act || role > 1) continue;
        // role 0 writes the planes z, role 1 the mirrored planes ngz - z
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int z = z0 + r;
            if (z >= Z0) continue;
            if (role == 0) {
                *reinterpret_cast<float4*>(Rt + (size_t)z * ncp + c0) =
                    make_float4(lo[r][0], lo[r][1], lo[r][2], lo[r][3]);
            } else {
                const int zm = ngz - z;
                if (z >= 1 && zm != z && zm < ngz)
                    *reinterpret_cast<float4*>(Rt + (size_t)zm * ncp + c0) =
                        make_float4(hi[r][0], hi[r][1], hi[r][2], hi[r][3]);
            }
        }
    }
}

#define SYN_ZB 16
// azimuthal synthesis + polcat, one CTA per (ring, SYN_ZB planes)
__global__ void __launch_bounds__(256) k_synaz(DevGeo g, int nact, int ncp, int tmask,
                                              const float* __restrict__ R, SynTab tb,
                                              float4* __restrict__ F, float* __restrict__ polar) {
    extern __shared__ __align__(16) float sm[];
    const int ir = blockIdx.x, zb = blockIdx.y * SYN_ZB;
    const int nr = g.nr, ngz = g.ngz, na = g.na, njp = tb.njp;
    const int nz = min(SYN_ZB, ngz - zb);
    float* TC = sm;                      // [nact][njp]
    float* TS = TC + nact * njp;
    float* CS = TS + nact * njp;         // [2][njp]
    float* Rs = CS + 2 * njp;            // [4][SYN_ZB][ncp]
    {
        // TC, TS and CS are one contiguous block of 2 (nact + 1) njp floats
        const float4* src = reinterpret_cast<const float4*>(tb.TC);
        float4* dst = reinterpret_cast<float4*>(TC);
        const int n4 = (2 * (nact + 1) * njp) >> 2;
        for (int i = threadIdx.x; i < n4; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    for (int i = threadIdx.x; i < 4 * SYN_ZB * ncp; i += blockDim.x) {
        const int t = i / (SYN_ZB * ncp), rem = i - t * SYN_ZB * ncp;
        const int z = rem / ncp, c = rem - z * ncp;
        float v = 0.f;
        if (((tmask >> t) & 1) && z < nz) v = R[(((size_t)t * nr + ir) * ngz + zb + z) * ncp + c];
        Rs[i] = v;
    }
    __syncthreads();
    const int nq = njp >> 2, half = na / 2;
    const size_t mesh = g.mesh;
    for (int it = threadIdx.x; it < nz * nq; it += blockDim.x) {
        const int z = it / nq, j0 = (it - z * nq) * 4;
        float C[4][4], S[4][4];
#pragma unroll
        for (int t = 0; t < 4; t++)
#pragma unroll
            for (int q = 0; q < 4; q++) C[t][q] = S[t][q] = 0.f;
        for (int a = 0; a < nact; a++) {
            const float4 tc = *reinterpret_cast<const float4*>(TC + a * njp + j0);
            const float4 ts = *reinterpret_cast<const float4*>(TS + a * njp + j0);
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const float2 r = *reinterpret_cast<const float2*>(Rs + (t * SYN_ZB + z) * ncp + 2 * a);
                const float rc = r.x, rs = r.y;
                C[t][0] += rc * tc.x; C[t][1] += rc * tc.y; C[t][2] += rc * tc.z; C[t][3] += rc * tc.w;
                S[t][0] += rs * ts.x; S[t][1] += rs * ts.y; S[t][2] += rs * ts.z; S[t][3] += rs * ts.w;
            }
        }
        const size_t rowb = ((size_t)ir * ngz + zb + z) * na;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int j = j0 + q;
            if (j > half) continue;
            const float cs = CS[j], sn = CS[njp + j];
            {
                const float fr = C[0][q] + S[0][q], ft = C[1][q] + S[1][q];
                const float fz = C[2][q] + S[2][q], ph = C[3][q] + S[3][q];
                F[rowb + j] = make_float4(fr * cs - ft * sn, fr * sn + ft * cs, fz, ph);
                if (polar) {
                    polar[rowb + j] = fr;
                    polar[mesh + rowb + j] = ft;
                    polar[2 * mesh + rowb + j] = fz;
                    polar[3 * mesh + rowb + j] = ph;
                }
            }
            if (j > 0 && j < half) {
                const int jm = na - j;  // angle -theta_j: cos same, sin negated
                const float fr = C[0][q] - S[0][q], ft = C[1][q] - S[1][q];
                const float fz = C[2][q] - S[2][q], ph = C[3][q] - S[3][q];
                F[rowb + jm] = make_float4(fr * cs + ft * sn, -fr * sn + ft * cs, fz, ph);
                if (polar) {
                    polar[rowb + jm] = fr;
                    polar[mesh + rowb + jm] = ft;
                    polar[2 * mesh + rowb + jm] = fz;
                    polar[3 * mesh + rowb + jm] = ph;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
int gx_synthesis(GxCtx* c, int tmask, float* polar) {
    const DevGeo& g = c->g;
    const int nact = c->spec.nact;
    const int ncp = ru4s(2 * nact);
    int Z0, KE, KO, njp;
    syn_dims(g, Z0, KE, KO, njp);
    const int nz4 = ru4s(Z0);
    const size_t nWe = (size_t)nz4 * KE, nWo = (size_t)nz4 * KO, nT = (size_t)nact * njp;
    if (!c->syntab) {
        if (nact > 64) return c->err = "more than 64 active harmonics", GX_ERR_RANGE;
        const size_t tot = 2 * nWe + 2 * nWo + 2 * nT + 2 * (size_t)njp;
        GX_CUDA(c, cudaMalloc((void**)&c->syntab, sizeof(float) * tot));
        ActList act;
        for (int a = 0; a < 64; a++) act.m[a] = a < nact ? c->spec.m[a] : 0;
        const float scale = (g.ndim == 3) ? 1.0f / (float)(2 * g.ngz * g.na) : 1.0f / (float)g.na;
        float* b = c->syntab;
        const size_t mx = std::max(std::max(nWe, nWo), std::max(nT, (size_t)njp));
        k_syntab<<<(unsigned)((mx + 255) / 256), 256, 0, c->stream>>>(
            g, act, nact, scale, b, b + nWe, b + 2 * nWe, b + 2 * nWe + nWo, b + 2 * nWe + 2 * nWo,
            b + 2 * nWe + 2 * nWo + nT, b + 2 * nWe + 2 * nWo + 2 * nT, Z0, KE, KO, njp);
        GX_LAUNCHED(c);
    }
    if (!c->synR) GX_CUDA(c, cudaMalloc((void**)&c->synR, sizeof(float) * 4 * g.nr * g.ngz * ncp));
    const float* b = c->syntab;
    SynTab tb{b, b + nWe, b + 2 * nWe, b + 2 * nWe + nWo, b + 2 * nWe + 2 * nWo,
              b + 2 * nWe + 2 * nWo + nT, b + 2 * nWe + 2 * nWo + 2 * nT, Z0, KE, KO, njp};
    {
        const size_t sm = sizeof(float) * (2 * nWe + 2 * nWo + (size_t)(KE + KO) * 2 * ncp);
        GX_CUDA(c, cudaFuncSetAttribute(k_synz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        dim3 grid(g.nr, 4);
        k_synz<<<grid, SYNZ_THREADS, sm, c->stream>>>(g, nact, ncp, tmask, c->specO, tb, c->synR);
        GX_LAUNCHED(c);
    }
    {
        const size_t sm = sizeof(float) * (2 * nT + 2 * (size_t)njp + (size_t)4 * SYN_ZB * ncp);
        GX_CUDA(c, cudaFuncSetAttribute(k_synaz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        dim3 grid(g.nr, (g.ngz + SYN_ZB - 1) / SYN_ZB);
        k_synaz<<<grid, 256, sm, c->stream>>>(g, nact, ncp, tmask, c->synR, tb, c->field, polar);
        GX_LAUNCHED(c);
    }
    return GX_OK;
}
