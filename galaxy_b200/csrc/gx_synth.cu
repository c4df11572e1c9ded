// gx_synth.cu -- field synthesis of the mixed path (p3fsyn.f:59-129,
// p2fsyn.f:34-56) fused with polcat (polcat.f:22-41).
//
// The inverse transforms are small GEMMs against twiddle tables built once
// per context.  In 3D, k_syn_ring does the vertical and the azimuthal
// synthesis and polcat of one ring per CTA (grids whose ring data fit in
// shared memory, unless GX_FLAG_ROWBLOCK_TRANSFORMS); the general kernels
// below take any grid.  Both exploit the symmetry of a real inverse DFT:
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

#include "gx_bulk.cuh"
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
    const float* TP;   // [nkz][szr_stride(Z0)] k even: wA(k, z), odd: wB(k, z)  (the P sum)
    const float* TQ;   // [nkz][szr_stride(Z0)] k even: wB(k, z), odd: wA(k, z)  (the Q sum)
    int Z0, KE, KO, njp;
};

__host__ __device__ static inline int ru4s(int x) { return (x + 3) & ~3; }
// row stride of TP / TQ: whole 16-plane blocks, and 8 (mod 32) floats so
// that the 16-byte table loads of a quarter warp in k_synz_ring (4
// consecutive wavenumbers x 2 four-plane groups) fall on 8 different groups
// of 4 banks
__host__ __device__ static inline int szr_stride(int Z0) { return (((Z0 + 15) & ~15) + 23) / 32 * 32 + 8; }

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
                         float* WAo, float* WBo, float* TC, float* TS, float* CS, float* TP, float* TQ,
                         int Z0, int KE, int KO, int njp) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nz = ru4s(Z0);
    const int nzt = szr_stride(Z0);
    if (TP && tid < nzt * g.nkz) {
        const int k = tid / nzt, z = tid - k * nzt;
        const float a = (z < Z0) ? wA(k, z, g.ngz) : 0.f, b = (z < Z0) ? wB(k, z, g.ngz) : 0.f;
        TP[tid] = (k & 1) ? b : a;
        TQ[tid] = (k & 1) ? a : b;
    }
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

// vertical synthesis, one CTA per (ring, field type); R[t][ir][z][ncp].
// With P = EA + OB and Q = OA + EB (E/O: even/odd wavenumbers, A/B: the
// two parts of the spectrum), plane z is P + Q and plane ngz - z is P - Q.
// Two threads own a 4 x 4 (plane, column) tile of P and Q, each summing
// every other wavenumber pair, combined by a shuffle; per pair a thread
// reads one float4 of each twiddle table (the planes of a wavenumber are
// contiguous) and one float4 of each spectrum part, for 64 FMAs.  The four
// twiddle tables start on different shared-memory banks.
#define SYNZ_THREADS 288
__device__ __forceinline__ int synz_pad(int start, int want) {
    return ((want - start) % 32 + 32) % 32;  // floats to add so that start lands on bank want
}
__global__ void __launch_bounds__(SYNZ_THREADS) k_synz(DevGeo g, int nact, int ncp, int tmask,
                                             const float4* __restrict__ O, SynTab tb,
                                             float* __restrict__ R, const int32_t* __restrict__ frk) {
    extern __shared__ __align__(16) float sm[];
    const int ir = blockIdx.x, t = blockIdx.y;
    if (!((tmask >> t) & 1)) return;
    if (frk && (ir + 1 < frk[0] || ir + 1 > frk[1])) return;  // partial grid (p3fsyn jrf..krf)
    const int nr = g.nr, nkz = g.nkz, ngz = g.ngz;
    float* Rt = R + (((size_t)t * nr + ir) * ngz) * ncp;
    // this ring's spectrum, one contiguous block [kz][a] (ring-major [t][ir][kz][a])
    const float4* Ot = O + (((size_t)t * nr + ir) * nkz) * nact;
    if (g.ndim == 2) {
        for (int c = threadIdx.x; c < ncp; c += blockDim.x) {
            const int a = c >> 1;
            float v = 0.f;
            if (a < nact) {
                float4 o = Ot[a];
                v = (c & 1) ? o.z : o.x;
            }
            Rt[c] = v;
        }
        return;
    }
    const int Z0 = tb.Z0, KE = tb.KE, KO = tb.KO, nz4 = ru4s(Z0);
    const int tE = KE * nz4, tO = KO * nz4;
    float* sWAe = sm;
    float* sWBe = sWAe + tE;
    sWBe += synz_pad((int)(sWBe - sm), 8);
    float* sWAo = sWBe + tE;
    sWAo += synz_pad((int)(sWAo - sm), 16);
    float* sWBo = sWAo + tO;
    sWBo += synz_pad((int)(sWBo - sm), 24);
    float* Ae = sWBo + tO;              // [KE][ncp]
    float* Be = Ae + KE * ncp;
    float* Ao = Be + KE * ncp;          // [KO][ncp]
    float* Bo = Ao + KO * ncp;
    // eight loads in flight per thread: the prologue is bound by the latency
    // of L2 (twiddles) and of scattered HBM reads (spectrum)
    {
        // the tables lie one after another in global memory: WAe, WBe, WAo, WBo
        const float4* src = reinterpret_cast<const float4*>(tb.WAe);
        float* dsts[4] = {sWAe, sWBe, sWAo, sWBo};
        const int n4[4] = {tE >> 2, tE >> 2, tO >> 2, tO >> 2};
        for (int q = 0; q < 4; q++) {
            float4* d = reinterpret_cast<float4*>(dsts[q]);
            for (int b = threadIdx.x; b < n4[q]; b += 8 * blockDim.x) {
                float4 v[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int i = b + u * blockDim.x;
                    if (i < n4[q]) v[u] = __ldg(src + i);
                }
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int i = b + u * blockDim.x;
                    if (i < n4[q]) d[i] = v[u];
                }
            }
            src += n4[q];
        }
    }
    // spectrum of this ring: rows k, columns (a-row, b-row) of each harmonic
    for (int b = threadIdx.x; b < nkz * nact; b += 8 * blockDim.x) {
        float4 o[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int i = b + u * blockDim.x;
            if (i < nkz * nact) o[u] = __ldg(Ot + i);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int i = b + u * blockDim.x;
            if (i < nkz * nact) {
                const int k = i / nact, a = i - k * nact;
                const int h = k >> 1;
                float* A = (k & 1) ? Ao : Ae;
                float* B = (k & 1) ? Bo : Be;
                A[h * ncp + 2 * a] = o[u].x;
                B[h * ncp + 2 * a] = o[u].y;
                A[h * ncp + 2 * a + 1] = o[u].z;
                B[h * ncp + 2 * a + 1] = o[u].w;
            }
        }
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
    const int tilesN = ncp >> 2, nt = (nz4 >> 2) * tilesN;
    const int ks = threadIdx.x & 1;
    for (int t0 = 0; t0 < nt; t0 += blockDim.x >> 1) {
        const int tile = t0 + (threadIdx.x >> 1);
        const bool act = tile < nt;
        const int tm = act ? tile / tilesN : 0, tn = act ? tile - tm * tilesN : 0;
        const int z0 = tm * 4, c0 = tn * 4;
        float P[4][4], Q[4][4];
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int q = 0; q < 4; q++) P[r][q] = Q[r][q] = 0.f;
        const int kend = act ? KE : 0;
#pragma unroll 2
        for (int i = ks; i < kend; i += 2) {
            const float4 we = *reinterpret_cast<const float4*>(sWAe + i * nz4 + z0);
            const float4 ve = *reinterpret_cast<const float4*>(Ae + i * ncp + c0);
            const float4 wb = *reinterpret_cast<const float4*>(sWBe + i * nz4 + z0);
            const float4 vb = *reinterpret_cast<const float4*>(Be + i * ncp + c0);
            const float w1[4] = {we.x, we.y, we.z, we.w}, w2[4] = {wb.x, wb.y, wb.z, wb.w};
#pragma unroll
            for (int r = 0; r < 4; r++) {
                P[r][0] += w1[r] * ve.x; P[r][1] += w1[r] * ve.y; P[r][2] += w1[r] * ve.z; P[r][3] += w1[r] * ve.w;
                Q[r][0] += w2[r] * vb.x; Q[r][1] += w2[r] * vb.y; Q[r][2] += w2[r] * vb.z; Q[r][3] += w2[r] * vb.w;
            }
            if (i < KO) {
                const float4 wo = *reinterpret_cast<const float4*>(sWAo + i * nz4 + z0);
                const float4 vo = *reinterpret_cast<const float4*>(Ao + i * ncp + c0);
                const float4 wq = *reinterpret_cast<const float4*>(sWBo + i * nz4 + z0);
                const float4 vq = *reinterpret_cast<const float4*>(Bo + i * ncp + c0);
                const float w3[4] = {wo.x, wo.y, wo.z, wo.w}, w4[4] = {wq.x, wq.y, wq.z, wq.w};
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    Q[r][0] += w3[r] * vo.x; Q[r][1] += w3[r] * vo.y; Q[r][2] += w3[r] * vo.z; Q[r][3] += w3[r] * vo.w;
                    P[r][0] += w4[r] * vq.x; P[r][1] += w4[r] * vq.y; P[r][2] += w4[r] * vq.z; P[r][3] += w4[r] * vq.w;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                P[r][q] += __shfl_xor_sync(0xffffffffu, P[r][q], 1);
                Q[r][q] += __shfl_xor_sync(0xffffffffu, Q[r][q], 1);
            }
        if (!act || ks) continue;
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int z = z0 + r;
            if (z >= Z0) continue;
            *reinterpret_cast<float4*>(Rt + (size_t)z * ncp + c0) =
                make_float4(P[r][0] + Q[r][0], P[r][1] + Q[r][1], P[r][2] + Q[r][2], P[r][3] + Q[r][3]);
            const int zm = ngz - z;
            if (z >= 1 && zm != z && zm < ngz)
                *reinterpret_cast<float4*>(Rt + (size_t)zm * ncp + c0) =
                    make_float4(P[r][0] - Q[r][0], P[r][1] - Q[r][1], P[r][2] - Q[r][2], P[r][3] - Q[r][3]);
        }
    }
}

// ---------------------------------------------------------------------------
// The same vertical synthesis on the tensor cores, persistent: P and Q are
// two small GEMMs per (ring, type), P = WAe^T Ae + WBo^T Bo and
// Q = WBe^T Be + WAo^T Ao (M = planes, N = columns, K = wavenumbers of one
// parity), computed with mma.sync m16n8k8 TF32 and three products per
// operand split x = hi + lo (hi = x rounded to TF32): lo hi + hi lo + hi hi
// with FP32 accumulation, so the result keeps FP32-class accuracy.  One CTA
// per SM loads the four twiddle tables once, split into their TF32 hi and
// lo parts ([i][64] each, the planes of row i stored at z ^ 8 (i & 3); 200 KB
// of shared memory with the spectrum), and walks its (ring, type) items; the spectrum of
// the next item is loaded into registers while the tensor cores work on the
// current one, then written to the [i][72] spectrum buffer.  Both layouts
// give bank-conflict-free fragment loads.  Warp w owns columns 8w .. 8w + 7.
#define SZT_K 64    // wavenumbers of one parity at most (KE, KO <= 64)
#define SZT_SS 72   // spectrum row stride: columns (ncp <= 72, 9 warps x 8)
#define SZT_PF 8    // spectrum float4 prefetched per thread (nkz nact <= 8 x 288)
__device__ __forceinline__ uint32_t syn_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return r & 0xffffe000u;
}
// not volatile: the accumulator operands carry every dependency, so the
// compiler may interleave independent products to hide their latency
__device__ __forceinline__ void syn_mma(float* d, const uint32_t* a, const uint32_t* b) {
    asm(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ void syn_split(float v, uint32_t& hi, uint32_t& lo) {
    hi = syn_tf32(v);
    lo = syn_tf32(v - __uint_as_float(hi));
}

static bool gx_synz_tc_ok(const DevGeo& g, int nact, int ncp) {
    int Z0, KE, KO, njp;
    syn_dims(g, Z0, KE, KO, njp);
    return g.ndim == 3 && Z0 <= 64 && KE <= SZT_K && KO <= SZT_K && ncp <= SZT_SS &&
           g.nkz * nact <= SZT_PF * SYNZ_THREADS;
}

// item it of a CTA's walk: (type, ring) with the type's bit in tmask and the
// ring inside the partial-grid range; false for items to skip
__device__ __forceinline__ bool szt_item(const DevGeo& g, int it, int tmask, const int32_t* frk,
                                         int& t, int& ir) {
    t = it / g.nr;
    ir = it - t * g.nr;
    if (!((tmask >> t) & 1)) return false;
    if (frk && (ir + 1 < frk[0] || ir + 1 > frk[1])) return false;
    return true;
}

__global__ void __launch_bounds__(SYNZ_THREADS, 1) k_synz_tc(DevGeo g, int nact, int ncp, int tmask,
                                                             const float4* __restrict__ O, SynTab tb,
                                                             float* __restrict__ R,
                                                             const int32_t* __restrict__ frk,
                                                             const int32_t* __restrict__ zr) {
    extern __shared__ __align__(16) float sm[];
    const int nr = g.nr, nkz = g.nkz, ngz = g.ngz;
    const int Z0 = tb.Z0, KE = tb.KE, KO = tb.KO, nz4 = ru4s(Z0);
    // the planes wanted (all, or those the next particle pass reads: the
    // planes holding mass, one wider each side); a tile of 16 planes z is
    // summed when z or its mirror ngz - z is wanted
    const int zlo = zr ? max(zr[0] - 1, 0) : 0, zhi = zr ? min(zr[1] + 1, ngz - 1) : ngz - 1;
    bool need[4];
#pragma unroll
    for (int a = 0; a < 4; a++) {
        const int z0 = 16 * a, z1 = min(16 * a + 15, Z0 - 1);
        need[a] = (z0 <= zhi && z1 >= zlo) || (ngz - z1 <= zhi && ngz - z0 >= zlo);
    }
    const int kte = (KE + 7) >> 3, kto = (KO + 7) >> 3;  // k-steps of 8 per parity
    const int nitems = 4 * nr, nsp = nkz * nact;
    uint32_t* sWh = reinterpret_cast<uint32_t*>(sm);  // [4][SZT_K][64]: WAe, WBe, WAo, WBo, TF32 hi
    uint32_t* sWl = sWh + 4 * SZT_K * 64;              // the same, lo = W - hi in TF32
    float* sS = sm + 8 * SZT_K * 64;                   // [4][SZT_K][SZT_SS]: Ae, Be, Ao, Bo
    {
        // twiddle tables once per CTA, split into TF32 hi and lo parts; rows
        // past KE / KO (to the k-step) and planes past nz4 are zero
        const float* srcs[4] = {tb.WAe, tb.WBe, tb.WAo, tb.WBo};
        const int rows[4] = {KE, KE, KO, KO}, prow[4] = {8 * kte, 8 * kte, 8 * kto, 8 * kto};
        for (int q = 0; q < 4; q++) {
            const float4* src = reinterpret_cast<const float4*>(srcs[q]);
            uint4* dh = reinterpret_cast<uint4*>(sWh + q * SZT_K * 64);
            uint4* dl = reinterpret_cast<uint4*>(sWl + q * SZT_K * 64);
            const int n4 = prow[q] * 16, w4 = nz4 >> 2;
            for (int b = threadIdx.x; b < n4; b += 8 * blockDim.x) {
                float4 v[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int e = b + u * blockDim.x, i = e >> 4, z4 = e & 15;
                    v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (e < n4 && i < rows[q] && z4 < w4) v[u] = __ldg(src + i * w4 + z4);
                }
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int e = b + u * blockDim.x, i = e >> 4, z4 = e & 15;
                    if (e < n4) {
                        uint4 h, l;
                        syn_split(v[u].x, h.x, l.x);
                        syn_split(v[u].y, h.y, l.y);
                        syn_split(v[u].z, h.z, l.z);
                        syn_split(v[u].w, h.w, l.w);
                        dh[i * 16 + (z4 ^ (2 * (i & 3)))] = h;
                        dl[i * 16 + (z4 ^ (2 * (i & 3)))] = l;
                    }
                }
            }
        }
        // the spectrum buffer's padding (columns past 2 nact, rows past KE /
        // KO to the k-step) is zero for every item: the items write only
        // their data region
        for (int i = threadIdx.x; i < 4 * SZT_K * SZT_SS; i += blockDim.x) {
            const int q = i / (SZT_K * SZT_SS), rem = i - q * SZT_K * SZT_SS;
            const int h = rem / SZT_SS, c = rem - h * SZT_SS;
            const int rq = (q < 2) ? KE : KO, pq = (q < 2) ? 8 * kte : 8 * kto;
            if (h < pq && (h >= rq || c >= 2 * nact)) sS[i] = 0.f;
        }
    }
    // the first item's spectrum into registers
    float4 pf[SZT_PF];
    int it = blockIdx.x, t = 0, ir = 0;
    bool act = (it < nitems) && szt_item(g, it, tmask, frk, t, ir);
    if (act) {
        const float4* Ot = O + (((size_t)t * nr + ir) * nkz) * nact;
#pragma unroll
        for (int u = 0; u < SZT_PF; u++) {
            const int i = threadIdx.x + u * blockDim.x;
            if (i < nsp) pf[u] = __ldg(Ot + i);
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = lane >> 2, c4 = lane & 3;
    const int n0 = 8 * warp, mt = (Z0 + 15) >> 4, sw = 8 * c4;
    for (; it < nitems; it += gridDim.x) {
        const bool cur = act;
        const int tc = t, irc = ir;
        __syncthreads();  // the previous item's fragments are read
        if (cur) {
#pragma unroll
            for (int u = 0; u < SZT_PF; u++) {
                const int i = threadIdx.x + u * blockDim.x;
                if (i < nsp) {
                    const int k = i / nact, a = i - k * nact;
                    const int h = k >> 1;
                    float* A = sS + ((k & 1) ? 2 : 0) * SZT_K * SZT_SS;
                    float* B = A + SZT_K * SZT_SS;
                    A[h * SZT_SS + 2 * a] = pf[u].x;
                    B[h * SZT_SS + 2 * a] = pf[u].y;
                    A[h * SZT_SS + 2 * a + 1] = pf[u].z;
                    B[h * SZT_SS + 2 * a + 1] = pf[u].w;
                }
            }
        }
        __syncthreads();
        // the next item's spectrum in flight while this one is summed
        const int nx = it + gridDim.x;
        act = (nx < nitems) && szt_item(g, nx, tmask, frk, t, ir);
        if (act) {
            const float4* Ot = O + (((size_t)t * nr + ir) * nkz) * nact;
#pragma unroll
            for (int u = 0; u < SZT_PF; u++) {
                const int i = threadIdx.x + u * blockDim.x;
                if (i < nsp) pf[u] = __ldg(Ot + i);
            }
        }
        if (!cur || n0 >= ncp) continue;
        float accP[4][4], accQ[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int r = 0; r < 4; r++) accP[a][r] = accQ[a][r] = 0.f;
#pragma unroll
        for (int part = 0; part < 2; part++) {
            // even wavenumbers: P += WAe Ae, Q += WBe Be; odd: P += WBo Bo, Q += WAo Ao
            const uint32_t* WPh = sWh + (part ? 3 : 0) * SZT_K * 64;
            const uint32_t* WPl = sWl + (part ? 3 : 0) * SZT_K * 64;
            const uint32_t* WQh = sWh + (part ? 2 : 1) * SZT_K * 64;
            const uint32_t* WQl = sWl + (part ? 2 : 1) * SZT_K * 64;
            const float* SP = sS + (part ? 3 : 0) * SZT_K * SZT_SS;
            const float* SQ = sS + (part ? 2 : 1) * SZT_K * SZT_SS;
            const int kt = part ? kto : kte;
            for (int kb = 0; kb < kt; kb++) {
                const int i0 = 8 * kb + c4, i1 = i0 + 4;
                uint32_t bPh[2], bPl[2], bQh[2], bQl[2];
                syn_split(SP[i0 * SZT_SS + n0 + q], bPh[0], bPl[0]);
                syn_split(SP[i1 * SZT_SS + n0 + q], bPh[1], bPl[1]);
                syn_split(SQ[i0 * SZT_SS + n0 + q], bQh[0], bQl[0]);
                syn_split(SQ[i1 * SZT_SS + n0 + q], bQh[1], bQl[1]);
#pragma unroll
                for (int a = 0; a < 4; a++) {
                    if (a >= mt) break;
                    if (!need[a]) continue;
                    const int m0 = (16 * a + q) ^ sw, m1 = (16 * a + q + 8) ^ sw;
                    const int o0 = i0 * 64 + m0, o1 = i0 * 64 + m1, o2 = i1 * 64 + m0, o3 = i1 * 64 + m1;
                    const uint32_t aph[4] = {WPh[o0], WPh[o1], WPh[o2], WPh[o3]};
                    const uint32_t apl[4] = {WPl[o0], WPl[o1], WPl[o2], WPl[o3]};
                    const uint32_t aqh[4] = {WQh[o0], WQh[o1], WQh[o2], WQh[o3]};
                    const uint32_t aql[4] = {WQl[o0], WQl[o1], WQl[o2], WQl[o3]};
                    // the P and Q chains interleaved
                    syn_mma(accP[a], apl, bPh);
                    syn_mma(accQ[a], aql, bQh);
                    syn_mma(accP[a], aph, bPl);
                    syn_mma(accQ[a], aqh, bQl);
                    syn_mma(accP[a], aph, bPh);
                    syn_mma(accQ[a], aqh, bQh);
                }
            }
        }
        // c0, c1: plane 16 a + q, columns c, c + 1; c2, c3: plane 16 a + q + 8.
        // Plane z is P + Q and plane ngz - z is P - Q.
        const int c = n0 + 2 * c4;
        if (c >= ncp) continue;
        float* Rt = R + (((size_t)tc * nr + irc) * ngz) * ncp;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            if (a >= mt) break;
            if (!need[a]) continue;
#pragma unroll
            for (int hrow = 0; hrow < 2; hrow++) {
                const int z = 16 * a + q + 8 * hrow;
                if (z >= Z0) continue;
                const float p0 = accP[a][2 * hrow], p1 = accP[a][2 * hrow + 1];
                const float q0 = accQ[a][2 * hrow], q1 = accQ[a][2 * hrow + 1];
                *reinterpret_cast<float2*>(Rt + (size_t)z * ncp + c) = make_float2(p0 + q0, p1 + q1);
                const int zm = ngz - z;
                if (z >= 1 && zm != z && zm < ngz)
                    *reinterpret_cast<float2*>(Rt + (size_t)zm * ncp + c) = make_float2(p0 - q0, p1 - q1);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The vertical synthesis of one ring per CTA, all four field types, in FP32:
// the ring's spectra O[t][ir][k][a] (four bulk copies) and the tables TP, TQ
// (two) come into shared memory on one mbarrier.  For the rows y of the
// needed 16-row blocks (as k_synz_tc: a block is summed when its planes or
// their mirrors ngz - y are wanted) P[y][c] = sum_k TP[k][y] s_P(k, c) and
// Q[y][c] = sum_k TQ[k][y] s_Q(k, c), where s_P is the cosine part A of the
// spectrum at even k and the sine part B at odd k, s_Q the other; plane y is
// P + Q and plane ngz - y is P - Q.  A thread owns 4 rows x 2 (type,
// harmonic) pairs (both columns 2a, 2a + 1 of each, P and Q: 32 sums); the
// wavenumber sum is split over 4 adjacent lanes by k mod 4 (so each lane's
// k have one parity and its spectrum parts are fixed) and added by
// shuffles.  A warp takes 4 row groups x 2 pairs: its table loads are 4 x 4
// distinct 16-byte words, its spectrum loads 2 x 4.  With m = 0 active its
// column is summed apart (2 warps), its sine column is zero.
#define SZR_THREADS 512
#define SZR_WARPS (SZR_THREADS / 32)
#define SZR_MAXBLK 64  // 16-row blocks at most (Z0 <= 1024)
// the field type of the n-th set bit of tmask
__device__ __forceinline__ int nth_type(int tmask, int n) {
    int t = 0;
#pragma unroll
    for (int b = 0; b < 4; b++)
        if ((tmask >> b) & 1) {
            if (n == 0) t = b;
            n--;
        }
    return t;
}
__global__ void __launch_bounds__(SZR_THREADS, 1) k_syn_ring(DevGeo g, int nact, int a0, int ncp, int tmask,
                                                             const float4* __restrict__ O, SynTab tb,
                                                             float* __restrict__ R, float4* __restrict__ F,
                                                             float* __restrict__ polar,
                                                             const int32_t* __restrict__ frk,
                                                             const int32_t* __restrict__ zr,
                                                             int32_t* __restrict__ errword) {
    extern __shared__ __align__(128) float sm[];
    __shared__ uint64_t bar;
    __shared__ int s_blk[SZR_MAXBLK], s_nblk;
    const int ir = blockIdx.x;
    if (frk && (ir + 1 < frk[0] || ir + 1 > frk[1])) return;  // rings no moving particle reads
    const int nr = g.nr, nkz = g.nkz, ngz = g.ngz, Z0 = tb.Z0, nz4 = szr_stride(Z0);
    float4* OS = reinterpret_cast<float4*>(sm);            // [4][nkz][nact]
    float* TP = sm + (size_t)16 * nkz * nact;              // [nkz][nz4]
    float* TQ = TP + (size_t)nkz * nz4;
    const int zlo = zr ? max(zr[0] - 1, 0) : 0, zhi = zr ? min(zr[1] + 1, ngz - 1) : ngz - 1;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t ob = (uint32_t)(nkz * nact) * 16u, tb4 = (uint32_t)(nkz * nz4) * 4u;
        uint32_t tot = 2 * tb4;
        for (int t = 0; t < 4; t++)
            if ((tmask >> t) & 1) tot += ob;
        mbar_expect_tx(&bar, tot);
        bulk_g2s(TP, tb.TP, tb4, &bar);
        bulk_g2s(TQ, tb.TQ, tb4, &bar);
        for (int t = 0; t < 4; t++)
            if ((tmask >> t) & 1)
                bulk_g2s(OS + (size_t)t * nkz * nact, O + ((size_t)t * nr + ir) * nkz * nact, ob, &bar);
    }
    if (!__syncthreads_and(mbar_wait(&bar, 0))) {
        if (threadIdx.x == 0) {
            atomicExch(errword, 6);
            mbar_wait(&bar, 0);  // the copies in flight land before the CTA leaves
        }
        return;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, ks = lane & 3, tl = lane >> 2;
    const int yg = tl & 3, pl = tl >> 2, par = ks & 1;
    // the field types wanted (tmask) and the 16-row blocks summed
    const int nty = __popc(tmask & 15);
    if (threadIdx.x == 0) {
        int n = 0;
        for (int yb = 0; yb < Z0; yb += 16) {
            const int y1 = min(yb + 15, Z0 - 1);
            if ((yb <= zhi && y1 >= zlo) || (ngz - y1 <= zhi && ngz - yb >= zlo)) s_blk[n++] = yb;
        }
        s_nblk = n;
    }
    __syncthreads();
    const int nblk = s_nblk;
    const int nh = nact - a0, nu = nty * nh, npair = (nu + 1) >> 1, npg = (npair + 1) >> 1;
    // units: (block, 2 pairs) for the harmonics a >= a0, then (block, 2 types)
    // for m = 0; dealt to the warps in turn
    const int nmain = nblk * npg, nunit = nmain + (a0 ? nblk * 2 : 0);
    for (int un = warp; un < nunit; un += SZR_WARPS) {
        if (un < nmain) {
            const int y = s_blk[un / npg] + 4 * yg;
            const int p = (un % npg) * 2 + pl;
            int tu[2], au[2];
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int uu = min(2 * p + u, nu - 1);
                const int ti = uu / nh;
                tu[u] = nth_type(tmask, ti);
                au[u] = a0 + (uu - ti * nh);
            }
            float P[2][4][2], Q[2][4][2];
#pragma unroll
            for (int u = 0; u < 2; u++)
#pragma unroll
                for (int i = 0; i < 4; i++) P[u][i][0] = P[u][i][1] = Q[u][i][0] = Q[u][i][1] = 0.f;
            const float4* o0 = OS + (size_t)tu[0] * nkz * nact + au[0];
            const float4* o1 = OS + (size_t)tu[1] * nkz * nact + au[1];
            // P takes the cosine part (x, z) at even k, the sine part (y, w) at
            // odd k, Q the other; a lane's k have one parity, so it sums the
            // cosine part against tx and the sine part against ty (TP and TQ
            // in its parity's roles) into P and Q, swapped at odd parity below
            const float* tx = par ? TQ : TP;
            const float* ty = par ? TP : TQ;
#pragma unroll 2
            for (int k = ks; k < nkz; k += 4) {
                const float4 ta = *reinterpret_cast<const float4*>(tx + (size_t)k * nz4 + y);
                const float4 tb4 = *reinterpret_cast<const float4*>(ty + (size_t)k * nz4 + y);
                const float4 s0 = o0[(size_t)k * nact], s1 = o1[(size_t)k * nact];
                const float tav[4] = {ta.x, ta.y, ta.z, ta.w}, tbv[4] = {tb4.x, tb4.y, tb4.z, tb4.w};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    P[0][i][0] += tav[i] * s0.x; P[0][i][1] += tav[i] * s0.z;
                    Q[0][i][0] += tbv[i] * s0.y; Q[0][i][1] += tbv[i] * s0.w;
                    P[1][i][0] += tav[i] * s1.x; P[1][i][1] += tav[i] * s1.z;
                    Q[1][i][0] += tbv[i] * s1.y; Q[1][i][1] += tbv[i] * s1.w;
                }
            }
            if (par) {
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int c = 0; c < 2; c++) {
                            const float t = P[u][i][c];
                            P[u][i][c] = Q[u][i][c];
                            Q[u][i][c] = t;
                        }
            }
#pragma unroll
            for (int o = 1; o < 4; o <<= 1)
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int c = 0; c < 2; c++) {
                            P[u][i][c] += __shfl_xor_sync(0xffffffffu, P[u][i][c], o);
                            Q[u][i][c] += __shfl_xor_sync(0xffffffffu, Q[u][i][c], o);
                        }
            if (ks != 0 || p >= npair) continue;
#pragma unroll
            for (int u = 0; u < 2; u++) {
                if (2 * p + u >= nu) continue;
                float* Rt = R + (((size_t)tu[u] * nr + ir) * ngz) * ncp + 2 * au[u];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int z = y + i;
                    if (z >= Z0) continue;
                    *reinterpret_cast<float2*>(Rt + (size_t)z * ncp) =
                        make_float2(P[u][i][0] + Q[u][i][0], P[u][i][1] + Q[u][i][1]);
                    const int zm = ngz - z;
                    if (z >= 1 && zm != z && zm < ngz)
                        *reinterpret_cast<float2*>(Rt + (size_t)zm * ncp) =
                            make_float2(P[u][i][0] - Q[u][i][0], P[u][i][1] - Q[u][i][1]);
                }
            }
        } else {
            // m = 0: 4 row groups x 2 types per unit, the cosine column only
            const int um = un - nmain;
            const int y = s_blk[um >> 1] + 4 * yg;
            const int tt = (um & 1) * 2 + pl;  // 0..3
            const float4* os = OS + (size_t)tt * nkz * nact;
            float Pc[4] = {0.f, 0.f, 0.f, 0.f}, Qc[4] = {0.f, 0.f, 0.f, 0.f};
            const float* tx = par ? TQ : TP;
            const float* ty = par ? TP : TQ;
            for (int k = ks; k < nkz; k += 4) {
                const float4 ta = *reinterpret_cast<const float4*>(tx + (size_t)k * nz4 + y);
                const float4 tb4 = *reinterpret_cast<const float4*>(ty + (size_t)k * nz4 + y);
                const float4 sv = os[(size_t)k * nact];
                Pc[0] += ta.x * sv.x; Pc[1] += ta.y * sv.x; Pc[2] += ta.z * sv.x; Pc[3] += ta.w * sv.x;
                Qc[0] += tb4.x * sv.y; Qc[1] += tb4.y * sv.y; Qc[2] += tb4.z * sv.y; Qc[3] += tb4.w * sv.y;
            }
            if (par) {
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float t = Pc[i];
                    Pc[i] = Qc[i];
                    Qc[i] = t;
                }
            }
#pragma unroll
            for (int o = 1; o < 4; o <<= 1)
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    Pc[i] += __shfl_xor_sync(0xffffffffu, Pc[i], o);
                    Qc[i] += __shfl_xor_sync(0xffffffffu, Qc[i], o);
                }
            if (ks == 0 && ((tmask >> tt) & 1)) {
                float* Rt = R + (((size_t)tt * nr + ir) * ngz) * ncp;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int z = y + i;
                    if (z >= Z0) continue;
                    *reinterpret_cast<float2*>(Rt + (size_t)z * ncp) = make_float2(Pc[i] + Qc[i], 0.f);
                    const int zm = ngz - z;
                    if (z >= 1 && zm != z && zm < ngz)
                        *reinterpret_cast<float2*>(Rt + (size_t)zm * ncp) = make_float2(Pc[i] - Qc[i], 0.f);
                }
            }
        }
    }
    // ---- azimuthal synthesis and polcat of the ring (as k_synaz) ----
    // R of the planes [zlo, zhi] comes back from L2 (written above by this
    // CTA: visible after the barrier; loads that bypass L1), the tables TC,
    // TS, CS with it; both into the space the spectra and TP / TQ held
    __syncthreads();
    const int nzw = zhi - zlo + 1;
    if (nzw <= 0) return;
    const int njp = tb.njp, na = g.na, nq = njp >> 2, half = na / 2;
    float* TCs = sm;                         // [nact][njp]
    float* TSs = TCs + (size_t)nact * njp;   // [nact][njp]
    float* CSs = TSs + (size_t)nact * njp;   // [2][njp]
    float* Rs = CSs + 2 * njp;               // [4][nzw][ncp]
    {
        const float4* src = reinterpret_cast<const float4*>(tb.TC);
        float4* dst = reinterpret_cast<float4*>(TCs);
        const int n4 = (2 * (nact + 1) * njp) >> 2;
        for (int i = threadIdx.x; i < n4; i += blockDim.x) dst[i] = __ldg(src + i);
        const int nrow4 = (nzw * ncp) >> 2;
        for (int t = 0; t < 4; t++) {
            float4* d = reinterpret_cast<float4*>(Rs + (size_t)t * nzw * ncp);
            if ((tmask >> t) & 1) {
                const float4* s4 = reinterpret_cast<const float4*>(R + (((size_t)t * nr + ir) * ngz + zlo) * ncp);
                for (int i = threadIdx.x; i < nrow4; i += blockDim.x) d[i] = __ldcg(s4 + i);
            } else {
                for (int i = threadIdx.x; i < nrow4; i += blockDim.x) d[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
    }
    __syncthreads();
    const size_t mesh = g.mesh;
    for (int it = threadIdx.x; it < nzw * nq; it += blockDim.x) {
        const int z = it / nq, j0 = (it - z * nq) * 4;
        float C[4][4], S[4][4];
#pragma unroll
        for (int t = 0; t < 4; t++)
#pragma unroll
            for (int q = 0; q < 4; q++) C[t][q] = S[t][q] = 0.f;
        for (int a = 0; a < nact; a++) {
            const float4 tc = *reinterpret_cast<const float4*>(TCs + a * njp + j0);
            const float4 ts = *reinterpret_cast<const float4*>(TSs + a * njp + j0);
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const float2 r = *reinterpret_cast<const float2*>(Rs + ((size_t)t * nzw + z) * ncp + 2 * a);
                C[t][0] += r.x * tc.x; C[t][1] += r.x * tc.y; C[t][2] += r.x * tc.z; C[t][3] += r.x * tc.w;
                S[t][0] += r.y * ts.x; S[t][1] += r.y * ts.y; S[t][2] += r.y * ts.z; S[t][3] += r.y * ts.w;
            }
        }
        const size_t rowb = ((size_t)ir * ngz + zlo + z) * na;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int j = j0 + q;
            if (j > half) continue;
            const float cs = CSs[j], sn = CSs[njp + j];
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

// shared memory of k_syn_ring, bytes; 0 when the ring's data do not fit
static size_t syn_ring_smem(const DevGeo& g, int nact, int Z0, int njp, int ncp) {
    // vertical part: the four types' spectra (float4 per wavenumber and
    // harmonic), TP and TQ; azimuthal part: TC, TS, CS and R of every plane
    const size_t v = (size_t)4 * sizeof(float4) * g.nkz * nact + (size_t)2 * sizeof(float) * g.nkz * szr_stride(Z0);
    const size_t a = sizeof(float) * ((size_t)2 * (nact + 1) * njp + (size_t)4 * g.ngz * ncp);
    const size_t b = std::max(v, a);
    return (g.ndim == 3 && (Z0 + 15) / 16 <= SZR_MAXBLK && b <= 220 * 1024) ? b : 0;
}

#define SYN_ZB 16
// 288 threads: the SYN_ZB x njp / 4 (plane, 4-spoke) items of a CTA (528 at
// 256 spokes) take two passes instead of two and a sliver
#define SYNAZ_THREADS 288
// azimuthal synthesis + polcat, one CTA per (ring, SYN_ZB planes)
__global__ void __launch_bounds__(SYNAZ_THREADS) k_synaz(DevGeo g, int nact, int ncp, int tmask,
                                              const float* __restrict__ R, SynTab tb,
                                              float4* __restrict__ F, float* __restrict__ polar,
                                              const int32_t* __restrict__ frk,
                                              const int32_t* __restrict__ zr,
                                              const float4* __restrict__ O2) {
    extern __shared__ __align__(16) float sm[];
    const int ir = blockIdx.x, zb = blockIdx.y * SYN_ZB;
    if (frk && (ir + 1 < frk[0] || ir + 1 > frk[1])) return;  // rings no moving particle reads
    const int nr = g.nr, ngz = g.ngz, na = g.na, njp = tb.njp;
    // with zr, only the planes the next particle pass reads: those holding
    // mass, one wider each side (a particle's interpolation cell may sit one
    // plane off its deposit cell); the block's planes [zb0, zb1)
    int zb0 = zb, zb1 = min(zb + SYN_ZB, ngz);
    if (zr) {
        zb0 = max(zb0, zr[0] - 1);
        zb1 = min(zb1, zr[1] + 2);
        if (zb1 <= zb0) return;
    }
    const int nz = zb1 - zb0;
    float* TC = sm;                      // [nact][njp]
    float* TS = TC + nact * njp;
    float* CS = TS + nact * njp;         // [2][njp]
    float* Rs = CS + 2 * njp;            // [4][SYN_ZB][ncp]
    {
        // TC, TS and CS are one contiguous block of 2 (nact + 1) njp floats
        const float4* src = reinterpret_cast<const float4*>(tb.TC);
        float4* dst = reinterpret_cast<float4*>(TC);
        const int n4 = (2 * (nact + 1) * njp) >> 2;
        for (int b = threadIdx.x; b < n4; b += 4 * blockDim.x) {
            float4 v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int i = b + u * blockDim.x;
                if (i < n4) v[u] = __ldg(src + i);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int i = b + u * blockDim.x;
                if (i < n4) dst[i] = v[u];
            }
        }
    }
    for (int b = threadIdx.x; b < 4 * SYN_ZB * ncp; b += 8 * blockDim.x) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int i = b + u * blockDim.x;
            const int t = i / (SYN_ZB * ncp), rem = i - t * SYN_ZB * ncp;
            const int z = rem / ncp, c = rem - z * ncp;
            v[u] = 0.f;
            if (i < 4 * SYN_ZB * ncp && ((tmask >> t) & 1) && z < nz) {
                if (O2) {
                    // 2D: the ring's contracted spectrum itself (no vertical
                    // part): column 2a the cosine term, 2a + 1 the sine term
                    const int a = c >> 1;
                    if (a < nact) {
                        const float4 o = __ldg(O2 + ((size_t)t * nr + ir) * nact + a);
                        v[u] = (c & 1) ? o.z : o.x;
                    }
                } else {
                    v[u] = __ldg(R + (((size_t)t * nr + ir) * ngz + zb0 + z) * ncp + c);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int i = b + u * blockDim.x;
            if (i < 4 * SYN_ZB * ncp) Rs[i] = v[u];
        }
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
        const size_t rowb = ((size_t)ir * ngz + zb0 + z) * na;
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
int gx_synthesis(GxCtx* c, int tmask, float* polar, const int32_t* frk, const int32_t* zr) {
    const DevGeo& g = c->g;
    const int nact = c->spec.nact;
    const int ncp = ru4s(2 * nact);
    int Z0, KE, KO, njp;
    syn_dims(g, Z0, KE, KO, njp);
    const int nz4 = ru4s(Z0);
    const size_t nWe = (size_t)nz4 * KE, nWo = (size_t)nz4 * KO, nT = (size_t)nact * njp;
    const size_t nTk = g.ndim == 3 ? (size_t)szr_stride(Z0) * g.nkz : 0;  // TP, TQ
    if (!c->syntab) {
        if (nact > 64) return c->err = "more than 64 active harmonics", GX_ERR_RANGE;
        const size_t tot = 2 * nWe + 2 * nWo + 2 * nT + 2 * (size_t)njp + 2 * nTk;
        GX_CUDA(c, cudaMalloc((void**)&c->syntab, sizeof(float) * tot));
        ActList act;
        for (int a = 0; a < 64; a++) act.m[a] = a < nact ? c->spec.m[a] : 0;
        const float scale = (g.ndim == 3) ? 1.0f / (float)(2 * g.ngz * g.na) : 1.0f / (float)g.na;
        float* b = c->syntab;
        const size_t mx = std::max(std::max(std::max(nWe, nWo), std::max(nT, (size_t)njp)), nTk);
        float* tk = b + 2 * nWe + 2 * nWo + 2 * nT + 2 * njp;
        k_syntab<<<(unsigned)((mx + 255) / 256), 256, 0, c->stream>>>(
            g, act, nact, scale, b, b + nWe, b + 2 * nWe, b + 2 * nWe + nWo, b + 2 * nWe + 2 * nWo,
            b + 2 * nWe + 2 * nWo + nT, b + 2 * nWe + 2 * nWo + 2 * nT, nTk ? tk : nullptr, nTk ? tk + nTk : nullptr,
            Z0, KE, KO, njp);
        GX_LAUNCHED(c);
    }
    if (!c->synR) GX_CUDA(c, cudaMalloc((void**)&c->synR, sizeof(float) * 4 * g.nr * g.ngz * ncp));
    const float* b = c->syntab;
    const float* tk = b + 2 * nWe + 2 * nWo + 2 * nT + 2 * njp;
    SynTab tb{b, b + nWe, b + 2 * nWe, b + 2 * nWe + nWo, b + 2 * nWe + 2 * nWo,
              b + 2 * nWe + 2 * nWo + nT, b + 2 * nWe + 2 * nWo + 2 * nT, tk, tk + nTk, Z0, KE, KO, njp};
    if (g.ndim == 3) {
        const size_t smr =
            (c->cfg.flags & GX_FLAG_ROWBLOCK_TRANSFORMS) ? 0 : syn_ring_smem(g, nact, Z0, njp, ncp);
        if (smr) {
            // vertical and azimuthal synthesis and polcat of one ring per CTA
            const int a0 = c->spec.m[0] == 0 ? 1 : 0;
            GX_CUDA(c, cudaFuncSetAttribute(k_syn_ring, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr));
            k_syn_ring<<<g.nr, SZR_THREADS, smr, c->stream>>>(g, nact, a0, ncp, tmask, c->specO, tb, c->synR,
                                                               c->field, polar, frk, zr, c->errword);
            GX_LAUNCHED(c);
            return GX_OK;
        }
        if (gx_synz_tc_ok(g, nact, ncp)) {
            // the tables, three bank pads of at most 31 floats, the spectrum
            int sms = 148;
            GX_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev));
            const size_t sm = sizeof(float) * (8 * SZT_K * 64 + 4 * SZT_K * SZT_SS);
            GX_CUDA(c, cudaFuncSetAttribute(k_synz_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            k_synz_tc<<<std::min(sms, 4 * g.nr), SYNZ_THREADS, sm, c->stream>>>(g, nact, ncp, tmask, c->specO,
                                                                              tb, c->synR, frk, zr);
        } else {
            const size_t sm = sizeof(float) * (2 * nWe + 2 * nWo + 3 * 32 + (size_t)(KE + KO) * 2 * ncp);
            GX_CUDA(c, cudaFuncSetAttribute(k_synz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            dim3 grid(g.nr, 4);
            k_synz<<<grid, SYNZ_THREADS, sm, c->stream>>>(g, nact, ncp, tmask, c->specO, tb, c->synR, frk);
        }
        GX_LAUNCHED(c);
    }
    {
        const size_t sm = sizeof(float) * (2 * nT + 2 * (size_t)njp + (size_t)4 * SYN_ZB * ncp);
        GX_CUDA(c, cudaFuncSetAttribute(k_synaz, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        dim3 grid(g.nr, (g.ngz + SYN_ZB - 1) / SYN_ZB);
        // 2D has no vertical part: the azimuthal synthesis reads the contracted spectrum
        k_synaz<<<grid, SYNAZ_THREADS, sm, c->stream>>>(g, nact, ncp, tmask, c->synR, tb, c->field, polar, frk,
                                                        g.ndim == 3 ? zr : nullptr,
                                                        g.ndim == 3 ? nullptr : c->specO);
        GX_LAUNCHED(c);
    }
    return GX_OK;
}
