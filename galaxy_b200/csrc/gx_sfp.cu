// gx_sfp.cu -- SFP (smooth-field-particle) Abel-Jacobi method: coefficient
// sum (sfpadd/sfpsum, scaled) and force evaluation (sfpacc).
//
// The reference tabulates U_nm(r/maxr) at nrtab radii and interpolates
// per particle (sfptab.f:43-78, sfpval.f:24-52), then accumulates
// C[n, +m] += U cos(m phi), C[n, -m] += U sin(m phi) in FP64
// (sfpadd.f:37-93).  Each U_nm(p) = p^m P_nm(p^2) with P_nm a polynomial of
// degree n + k (ajfun.f:33-47); with e = m mod 2, U_nm / p^e is a polynomial
// in p^2 of degree n + k + (m - e)/2, so with x = 2 p^2 - 1 it is exactly a
// Chebyshev series sum_d a_nmd T_d(x).  (Keeping the even power of p inside
// the series keeps its coefficients of the size of U itself; dividing out all
// of p^m would blow them up near the centre.)  The sum over particles
// factors through the moment matrix
//     M[d][c] = sum_p T_d(x_p) g_c(p),  g = (1, p^e cos m phi, p^e sin m phi)
// and C[n, m, .] = sum_d a_nmd M[d][c(m, .)].  M is a GEMM with K = N
// (particles): it runs on the tensor cores with mma.sync m16n8k16 FP16,
// each operand split into an FP16 hi and lo part (three products, FP32
// accumulate per warp over a chunk of particles, chunks summed in FP64).
// Each lane computes its particle's features once and stores them as a row
// of the warp's shared-memory tiles; transposing tile loads (ldmatrix
// .trans) turn those rows into the MMA fragments.
// a_nmd are formed once on the host in FP64 from the roots and
// coefficients of the basis (Chebyshev interpolation at 64 nodes).
#include <cuda_fp16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "gx_common.cuh"

#define SFP_CHUNK 1024  // particles per warp-chunk (FP32 accumulation span)
#define SFP_MAXMOM (64 * 48)  // moments: [D][NCP] (D <= 64, NCP <= 32), or the tcgen05 path's raw [64][48]

struct GxSfp {
    GxSfpBasis b;
    std::vector<double> roots, xcoeff;
    int dev = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::string err;
    int nfun = 0;
    std::vector<int> msel, nsel;
    int D = 32;   // Chebyshev terms
    int NC = 0;   // feature columns 2 maxm + 1
    std::vector<double> acheb;  // [nfun][D]
    double maxr = 1.0;
    int64_t n = 0, cap = 0;
    float* xy = nullptr;        // [2][cap]
    float* vel = nullptr;       // [2][cap] velocities of the SFP-driven step
    float4* ftab = nullptr;     // [maxm + 1][SFP_NT] force table of the SFP-driven step
    std::vector<double> qs_h;   // host staging of the force series
    float* part = nullptr;      // per-warp partial moments
    double* mom = nullptr;      // [D][NCP] FP64 moments
    double* qc = nullptr;       // device force series [2][maxm+1][D]
    double* upart = nullptr;    // per-CTA FP64 partial rows of the tcgen05 path
    double* slab = nullptr;     // [2 nsm][nmom] FP64 first-stage sums of the partials
    int32_t* errword = nullptr; // device error word (bounded waits)
    int nsm = 0;
    float last_ms = 0.f;
    int64_t launches = 0;
};

static std::string g_sfp_err;

// ---------------------------------------------------------------------------
// host: ajfun in FP64 (ajfun.f:33-47) and its Chebyshev coefficients
static double ajfun_h(const GxSfp* s, int m, int n, double r) {
    const GxSfpBasis& b = s->b;
    const double* xc = s->xcoeff.data() + ((size_t)m * (b.maxn + 1) + n) * (b.k + 1);
    const double* rt = s->roots.data() + ((size_t)m * (b.maxn + 1) + n) * b.maxn;
    const double r2 = r * r, x = 1.0 - r2;
    double f = xc[0];
    for (int i = 1; i <= b.k; i++) f += xc[i] * pow(x, i);
    for (int i = 0; i < n; i++) f *= (r2 - rt[i] * rt[i]);
    return GX_PI / (double)sqrtf(2.0f) * f;  // pi / sqrt(2.), sqrt in single precision
}

static void cheb_coeffs(GxSfp* s) {
    const int NN = 64;
    s->acheb.assign((size_t)s->nfun * s->D, 0.0);
    std::vector<double> vals(NN);
    for (int f = 0; f < s->nfun; f++) {
        const int m = s->msel[f], n = s->nsel[f];
        for (int j = 0; j < NN; j++) {
            double xj = cos(GX_PI * (j + 0.5) / NN);
            double p = sqrt(0.5 * (xj + 1.0));
            // U_nm / p^(m mod 2): ajfun_h leaves out the r^m factor
            vals[j] = ajfun_h(s, m, n, p) * pow(p, (double)(m - (m & 1)));
        }
        for (int d = 0; d < s->D; d++) {
            double acc = 0;
            for (int j = 0; j < NN; j++) acc += vals[j] * cos(d * GX_PI * (j + 0.5) / NN);
            s->acheb[(size_t)f * s->D + d] = (d == 0 ? 1.0 : 2.0) * acc / NN;
        }
    }
}

// ---------------------------------------------------------------------------
// device helpers
// round to TF32 (nearest, ties away) and clear the 13 low mantissa bits, so
// that the returned bits are exactly the TF32 value as an FP32 number
__device__ __forceinline__ uint32_t f2tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return r & 0xffffe000u;
}

// one m16n8k16 FP16 product with FP32 accumulation, D += A B
__device__ __forceinline__ void mma_f16(float* d, const uint32_t* a, const uint32_t* b) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// the same with D = A B (no accumulator input)
__device__ __forceinline__ void mma_f16_0(float* d, const uint32_t* a, const uint32_t* b) {
    asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%10,%10,%10,%10};\n"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]), "f"(0.f));
}
// four / two transposed 8 x 8 FP16 tiles (rows of 16 bytes at the lanes' addresses)
__device__ __forceinline__ void ldsm_t4(uint32_t* r, uint32_t addr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_t2(uint32_t* r, uint32_t addr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(addr));
}
// v0 + v1 split into FP16 pairs: hi = (v0, v1) to nearest, lo = their
// remainders to nearest (v = hi + lo to ~2^-22 relative, or 2^-25 absolute
// where lo falls below the FP16 normal range); v0 at the lower address
__device__ __forceinline__ void split_h2(float v0, float v1, uint32_t& hi, uint32_t& lo) {
    const __half2 h = __floats2half2_rn(v0, v1);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(v0 - hf.x, v1 - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Moments of one SFP_CHUNK of particles per warp; part[warp][d][c].
// Rounds of 32 particles: lane l computes the features of particle l once --
// T_d(x) for d < D by the three-term recurrence, and g_n (n >= 1) =
// p^e cos m phi, p^e sin m phi (e = m mod 2) from repeated multiplication of
// (x, y) / r -- splits each into an FP16 hi and lo part and writes them as
// row l of the warp's shared-memory tiles Th, Tl [32][D + 8] and Gh, Gl
// [32][GS] (row strides of 80 / 144 / 48 bytes put the eight 16-byte rows of
// a transposed 8 x 8 tile load on distinct banks).  ldmatrix .trans turns
// the particle-major rows into the fragments of M[d][n] = sum_k T_d(k) g_n(k)
// for mma.sync m16n8k16 (A = T, 16 d x 16 particles; B = g, 16 particles x 8
// columns), three products per hi/lo pair (hi hi, hi lo, lo hi), FP32
// accumulation over the chunk.  Column c = 0 (g_0 = 1) is the plain sum of
// T_d, one-signed for most d: on the tensor cores (a B fragment of ones in
// registers, products hi 1 and lo 1) it starts from zero in every round of
// 32 particles, whose sum (|.| <= 32) the tensor cores' FP32 accumulation
// keeps to ~2^-18, and the rounds are added on the CUDA cores (rounded to
// nearest).  Accumulated over a whole chunk in the tensor cores, this
// column's sums of ~1000 would lose ~1e-5 to the accumulation's truncation.
// The recurrences
// start from sw = 1 for particles inside the basis edge (p <= 1) and 0 for
// the rest, which makes every feature of an outside particle zero.
template <int MT, int NB>
__global__ void __launch_bounds__(256, MT == 2 ? 3 : 1) k_sfp_moments(const float* __restrict__ X,
                                                     const float* __restrict__ Y, int64_t n,
                                                     float inv_maxr, int maxm, int NCP,
                                                     float* __restrict__ part) {
    constexpr int D = MT * 16, TS = D + 8, GS = (NB == 3) ? 40 : 24;
    constexpr int WARP_HALVES = 2 * 32 * (TS + GS);
    static_assert(8 * NB <= GS, "g tile width");
    extern __shared__ __align__(16) __half sfh[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    __half* Th = sfh + (size_t)wib * WARP_HALVES;
    __half* Tl = Th + 32 * TS;
    __half* Gh = Tl + 32 * TS;
    __half* Gl = Gh + 32 * GS;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t base = wid * SFP_CHUNK;
    if (base >= n) return;
    // ldmatrix row addresses: lane = 8 j + i supplies row i of tile j
    const int li = lane & 7, lj = lane >> 3;
    // A tile (16 d x 16 particles) at d0 = 16 a, particles 16 kb: tile j holds
    // particles 8 (j >> 1) .. + 7 and d = 8 (j & 1) .. + 7
    const uint32_t aoff = (uint32_t)(((li + 8 * (lj >> 1)) * TS + 8 * (lj & 1)) * 2);
    // B tiles of column blocks u, u + 1: tile j holds particles 8 (j & 1) ..
    // + 7 and columns 8 u + 8 (j >> 1) .. + 7
    const uint32_t boff = (uint32_t)(((li + 8 * (lj & 1)) * GS + 8 * (lj >> 1)) * 2);
    const uint32_t sTh = (uint32_t)__cvta_generic_to_shared(Th), sTl = (uint32_t)__cvta_generic_to_shared(Tl);
    const uint32_t sGh = (uint32_t)__cvta_generic_to_shared(Gh), sGl = (uint32_t)__cvta_generic_to_shared(Gl);
    float acc[MT][NB][4];
#pragma unroll
    for (int a = 0; a < MT; a++)
#pragma unroll
        for (int u = 0; u < NB; u++)
#pragma unroll
            for (int i = 0; i < 4; i++) acc[a][u][i] = 0.f;
    float run0[MT][2];  // column 0, rows 16 a + q and 16 a + q + 8 (lanes with c4 = 0)
#pragma unroll
    for (int a = 0; a < MT; a++) run0[a][0] = run0[a][1] = 0.f;
    // B fragment of the column block (1, 0, ..., 0): b = B[2 c4 .. + 1][q], ones at q = 0
    const uint32_t ones[2] = {lane < 4 ? 0x3C003C00u : 0u, lane < 4 ? 0x3C003C00u : 0u};
    const int64_t end = min(base + (int64_t)SFP_CHUNK, n);
    // the coordinates of the next round are loaded one round ahead
    // (raw values: they are scaled where they are used, a round later)
    bool nin = base + lane < end;
    float nx = 0.f, ny = 0.f;
    if (nin) {
        nx = __ldg(X + base + lane);
        ny = __ldg(Y + base + lane);
    }
    for (int64_t r0 = base; r0 < end; r0 += 32) {
        // ---- features of particle r0 + lane, split into row lane of the tiles
        {
            // a lane past the end stands outside the basis edge: no contribution
            const float px = nin ? nx * inv_maxr : 2.f, py = nin ? ny * inv_maxr : 0.f;
            nin = r0 + 32 + lane < end;
            if (nin) {
                nx = __ldg(X + r0 + 32 + lane);
                ny = __ldg(Y + r0 + 32 + lane);
            }
            const float p2 = px * px + py * py;
            const bool act = p2 <= 1.0f;
            const float sw = act ? 1.f : 0.f;
            const float xc = act ? 2.f * p2 - 1.f : 0.f, x2 = 2.f * xc;
            // T_{d+2} = y2 T_d - T_{d-2} (y2 = 2 T_2(x)): the even and the odd
            // terms are two independent recurrences
            const float y2 = 2.f * fmaf(x2, xc, -1.f);
            float T[D];
            T[0] = sw;
            T[1] = sw * xc;
            T[2] = fmaf(x2, T[1], -T[0]);
            T[3] = fmaf(x2, T[2], -T[1]);
#pragma unroll
            for (int d = 4; d < D; d++) T[d] = fmaf(y2, T[d - 2], -T[d - 4]);
#pragma unroll
            for (int d = 0; d < D; d += 8) {
                uint4 h, l;
                split_h2(T[d], T[d + 1], h.x, l.x);
                split_h2(T[d + 2], T[d + 3], h.y, l.y);
                split_h2(T[d + 4], T[d + 5], h.z, l.z);
                split_h2(T[d + 6], T[d + 7], h.w, l.w);
                *reinterpret_cast<uint4*>(Th + lane * TS + d) = h;
                *reinterpret_cast<uint4*>(Tl + lane * TS + d) = l;
            }
            // |p| and the direction (x, y) / |p| from one reciprocal square root
            const float rs = (act && p2 > 0.f) ? rsqrtf(p2) : 0.f;
            const float pr = p2 * rs;
            const bool dir = rs > 0.f;
            const float cr = dir ? px * rs : 1.f, ci = dir ? py * rs : 0.f;
            float zr = sw, zi = 0.f;
#pragma unroll
            for (int u = 0; u < NB * 8; u += 8) {
                float g[8];
#pragma unroll
                for (int k = 0; k < 8; k += 2) {
                    const int m = (u + k) / 2 + 1;
                    float gc = 0.f, gs = 0.f;
                    if (m <= maxm) {
                        const float nr = zr * cr - zi * ci;
                        zi = zr * ci + zi * cr;
                        zr = nr;
                        gc = (m & 1) ? zr * pr : zr;
                        gs = (m & 1) ? zi * pr : zi;
                    }
                    g[k] = gc;
                    g[k + 1] = gs;
                }
                uint4 h, l;
                split_h2(g[0], g[1], h.x, l.x);
                split_h2(g[2], g[3], h.y, l.y);
                split_h2(g[4], g[5], h.z, l.z);
                split_h2(g[6], g[7], h.w, l.w);
                *reinterpret_cast<uint4*>(Gh + lane * GS + u) = h;
                *reinterpret_cast<uint4*>(Gl + lane * GS + u) = l;
            }
        }
        __syncwarp();
        // ---- columns 1 .. 8 NB on the tensor cores, 2 k-blocks of 16 particles
        float f0[MT][4];  // column 0 of this round
#pragma unroll
        for (int kb = 0; kb < 2; kb++) {
            uint32_t bh[NB][2], bl[NB][2];
            const uint32_t kbA = (uint32_t)(16 * kb * TS * 2), kbB = (uint32_t)(16 * kb * GS * 2);
#pragma unroll
            for (int u = 0; u < NB; u += 2) {
                if (u + 1 < NB) {
                    uint32_t r[4];
                    ldsm_t4(r, sGh + kbB + boff + 16 * u);
                    bh[u][0] = r[0]; bh[u][1] = r[1]; bh[u + 1][0] = r[2]; bh[u + 1][1] = r[3];
                    ldsm_t4(r, sGl + kbB + boff + 16 * u);
                    bl[u][0] = r[0]; bl[u][1] = r[1]; bl[u + 1][0] = r[2]; bl[u + 1][1] = r[3];
                } else {
                    ldsm_t2(bh[u], sGh + kbB + boff + 16 * u);
                    ldsm_t2(bl[u], sGl + kbB + boff + 16 * u);
                }
            }
            uint32_t ah[MT][4], al[MT][4];
#pragma unroll
            for (int a = 0; a < MT; a++) {
                ldsm_t4(ah[a], sTh + kbA + aoff + 32 * a);
                ldsm_t4(al[a], sTl + kbA + aoff + 32 * a);
            }
#pragma unroll
            for (int a = 0; a < MT; a++) {
                if (kb == 0) mma_f16_0(f0[a], ah[a], ones);
                else mma_f16(f0[a], ah[a], ones);
            }
#pragma unroll
            for (int a = 0; a < MT; a++)
#pragma unroll
                for (int u = 0; u < NB; u++) mma_f16(acc[a][u], al[a], bh[u]);
#pragma unroll
            for (int a = 0; a < MT; a++)
#pragma unroll
                for (int u = 0; u < NB; u++) mma_f16(acc[a][u], ah[a], bl[u]);
#pragma unroll
            for (int a = 0; a < MT; a++)
#pragma unroll
                for (int u = 0; u < NB; u++) mma_f16(acc[a][u], ah[a], bh[u]);
#pragma unroll
            for (int a = 0; a < MT; a++) mma_f16(f0[a], al[a], ones);
        }
#pragma unroll
        for (int a = 0; a < MT; a++) {
            run0[a][0] += f0[a][0];
            run0[a][1] += f0[a][2];
        }
        __syncwarp();
    }
    // c0 = D[q][2c4], c1 = D[q][2c4+1], c2 = D[q+8][2c4], c3 = D[q+8][2c4+1]; column
    // n of the product is feature column n + 1
    const int q = lane >> 2, c4 = lane & 3;
    float* dst = part + wid * (size_t)D * NCP;
#pragma unroll
    for (int a = 0; a < MT; a++)
#pragma unroll
        for (int u = 0; u < NB; u++) {
            const int rr = a * 16 + q, cc = u * 8 + 2 * c4 + 1;
            if (cc < NCP) {
                dst[rr * NCP + cc] = acc[a][u][0];
                dst[(rr + 8) * NCP + cc] = acc[a][u][2];
            }
            if (cc + 1 < NCP) {
                dst[rr * NCP + cc + 1] = acc[a][u][1];
                dst[(rr + 8) * NCP + cc + 1] = acc[a][u][3];
            }
        }
#pragma unroll
    for (int a = 0; a < MT; a++)
        if (c4 == 0) {
            dst[(a * 16 + q) * NCP] = run0[a][0];
            dst[(a * 16 + q + 8) * NCP] = run0[a][1];
        }
    // columns past the products
    for (int i = lane; i < D * (NCP - 1 - 8 * NB); i += 32) {
        const int d = i / (NCP - 1 - 8 * NB), c = 1 + 8 * NB + (i - d * (NCP - 1 - 8 * NB));
        dst[d * NCP + c] = 0.f;
    }
}

// FP64 sum of the per-warp partials: one block per moment, each thread a
// strided subset of the warps, then a fixed-shape tree (deterministic)
template <typename T>
__global__ void k_sfp_reduce(const T* __restrict__ part, int64_t nwarp, int nmom,
                             double* __restrict__ mom) {
    __shared__ double sh[256];
    const int i = blockIdx.x;
    double s = 0.0;
    for (int64_t w = threadIdx.x; w < nwarp; w += blockDim.x) s += (double)part[w * nmom + i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) mom[i] = sh[0];
}

// First stage of the coalesced FP64 sum of per-warp (or per-block) partial
// rows: block b sums rows [b rpb, (b + 1) rpb) of part[nrow][nmom] in a
// fixed order, each thread a set of moment columns (consecutive threads on
// consecutive columns); k_sfp_reduce then sums the nslab rows of out.
template <typename T>
__global__ void k_sfp_slab(const T* __restrict__ part, int64_t nrow, int nmom, int64_t rpb,
                           double* __restrict__ out) {
    const int64_t r0 = blockIdx.x * rpb, r1 = min(nrow, r0 + rpb);
    for (int i = threadIdx.x; i < nmom; i += blockDim.x) {
        double s0 = 0.0, s1 = 0.0;
        int64_t r = r0;
        for (; r + 1 < r1; r += 2) {
            s0 += (double)part[r * nmom + i];
            s1 += (double)part[(r + 1) * nmom + i];
        }
        if (r < r1) s0 += (double)part[r * nmom + i];
        out[blockIdx.x * (int64_t)nmom + i] = s0 + s1;
    }
}

// plain FP64 moments on CUDA cores: features staged per block, one thread
// per (d, c) moment summing over the block's particles, FP64 partial per block
__global__ void k_sfp_moments64(const float* __restrict__ X, const float* __restrict__ Y, int64_t n,
                                double inv_maxr, int maxm, int D, int NCP,
                                double* __restrict__ part) {
    extern __shared__ double fs[];  // [256][D + NCP]
    const int w = D + NCP;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double* f = fs + threadIdx.x * w;
    for (int k = 0; k < w; k++) f[k] = 0.0;
    if (i < n) {
        const double px = X[i] * inv_maxr, py = Y[i] * inv_maxr, p2 = px * px + py * py;
        if (p2 <= 1.0) {
            const double xc = 2.0 * p2 - 1.0;
            f[0] = 1.0;
            if (D > 1) f[1] = xc;
            for (int d = 2; d < D; d++) f[d] = 2.0 * xc * f[d - 1] - f[d - 2];
            const double pr = sqrt(p2);
            const double cr = pr > 0.0 ? px / pr : 1.0, ci = pr > 0.0 ? py / pr : 0.0;
            double zr = 1.0, zi = 0.0;
            f[D] = 1.0;
            for (int m = 1; m <= maxm; m++) {
                double nr = zr * cr - zi * ci;
                zi = zr * ci + zi * cr;
                zr = nr;
                const double e = (m & 1) ? pr : 1.0;
                f[D + 2 * m - 1] = zr * e;
                f[D + 2 * m] = zi * e;
            }
        }
    }
    __syncthreads();
    const int nb = min((int64_t)blockDim.x, n - blockIdx.x * (int64_t)blockDim.x);
    for (int mo = threadIdx.x; mo < D * NCP; mo += blockDim.x) {
        const int d = mo / NCP, c = mo - d * NCP;
        double s = 0.0;
        for (int p = 0; p < nb; p++) s += fs[p * w + d] * fs[p * w + D + c];
        part[blockIdx.x * (size_t)D * NCP + mo] = s;
    }
}

// sfpacc (sfpacc.f:41-112, 249-259) at (x, y) from the per-m Chebyshev
// series of the scaled coefficients: qc[(0/1)][m][d] (cosine / sine), FP64;
// zero outside the basis edge r > maxr
__device__ __forceinline__ void sfp_force(double x, double y, double maxr, int maxm, int D,
                                          const double* __restrict__ qs, double& ax, double& ay, double& ph) {
    const double rr = sqrt(x * x + y * y);
    double ar = 0, at = 0;
    ax = ay = ph = 0.0;
    if (rr > maxr) return;
    const double r = rr > 1e-5 ? rr : 1e-5;
    const double c1 = x / r, s1 = y / r;
    const double p = rr / maxr, xc = 2.0 * p * p - 1.0;
    double cm = 1.0, sm = 0.0;  // cos m phi, sin m phi
    for (int m = 0; m <= maxm; m++) {
        if (m > 0) {
            double nc = cm * c1 - sm * s1;
            sm = sm * c1 + cm * s1;
            cm = nc;
        }
        // Clenshaw for Q(x) and Q'(x) of both series
        double val[2], der[2];
        for (int h = 0; h < 2; h++) {
            const double* a = qs + ((size_t)h * (maxm + 1) + m) * D;
            double b1 = 0, b2 = 0, d1 = 0, d2 = 0;
            for (int d = D - 1; d >= 1; d--) {
                double bn = 2.0 * xc * b1 - b2 + a[d];
                double dn = 2.0 * xc * d1 - d2 + 2.0 * b1;
                b2 = b1;
                b1 = bn;
                d2 = d1;
                d1 = dn;
            }
            val[h] = xc * b1 - b2 + a[0];
            der[h] = xc * d1 - d2 + b1;
        }
        // f = p^e Q(x) (e = m mod 2), df/dp = e Q + p^e Q'(x) dx/dp, dx/dp = 4 p
        const double pe = (m & 1) ? p : 1.0, e = (double)(m & 1);
        const double fc = pe * val[0], fs = pe * val[1];
        const double dc = e * val[0] + pe * der[0] * 4.0 * p;
        const double ds = e * val[1] + pe * der[1] * 4.0 * p;
        if (m == 0) {
            ar += dc;
            ph -= fc;
        } else {
            ar += dc * cm + ds * sm;
            at += (double)m * (fs * cm - fc * sm);
            ph -= fc * cm + fs * sm;
        }
    }
    at = at * maxr / r;
    ax = ar * c1 - at * s1;
    ay = ar * s1 + at * c1;
}

__global__ void k_sfp_acc(const float* __restrict__ X, const float* __restrict__ Y, int64_t n,
                          double maxr, int maxm, int D, const double* __restrict__ qs,
                          float* __restrict__ acc, float* __restrict__ pot) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ax, ay, ph;
    sfp_force(X[i], Y[i], maxr, maxm, D, qs, ax, ay, ph);
    acc[2 * i] = (float)ax;
    acc[2 * i + 1] = (float)ay;
    if (pot) pot[i] = (float)ph;
}

// The time loop's force table, as the reference tabulates its basis
// (sfptab.f:43-78) and interpolates it (sfpval.f:24-52): per m the radial
// factors f_c, f_s = p^e Q(x) of the cosine and sine series and their
// p-derivatives, at SFP_NT radii p_i = i / (SFP_NT - 1), evaluated in FP64
// from the force series (Clenshaw, as sfp_force) and stored as FP32.
#define SFP_NT 1025
__global__ void k_sfp_ftab(int maxm, int D, const double* __restrict__ qs, float4* __restrict__ tab) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (maxm + 1) * SFP_NT) return;
    const int m = i / SFP_NT, j = i - m * SFP_NT;
    const double p = (double)j / (double)(SFP_NT - 1), xc = 2.0 * p * p - 1.0;
    double val[2], der[2];
    for (int h = 0; h < 2; h++) {
        const double* a = qs + ((size_t)h * (maxm + 1) + m) * D;
        double b1 = 0, b2 = 0, d1 = 0, d2 = 0;
        for (int d = D - 1; d >= 1; d--) {
            const double bn = 2.0 * xc * b1 - b2 + a[d];
            const double dn = 2.0 * xc * d1 - d2 + 2.0 * b1;
            b2 = b1;
            b1 = bn;
            d2 = d1;
            d1 = dn;
        }
        val[h] = xc * b1 - b2 + a[0];
        der[h] = xc * d1 - d2 + b1;
    }
    const double pe = (m & 1) ? p : 1.0, e = (double)(m & 1);
    tab[i] = make_float4((float)(pe * val[0]), (float)(pe * val[1]), (float)(e * val[0] + pe * der[0] * 4.0 * p),
                         (float)(e * val[1] + pe * der[1] * 4.0 * p));
}

// one leapfrog step in the SFP field (stpgrp.f:26-32 with the time step
// made explicit): v += a(x) dt, x += v dt, the force from the table by
// 4-point Lagrange interpolation in p (FP32; the interpolation error of the
// degree <= 63 series on 1025 radii is ~1e-7 of the force)
__global__ void k_sfp_kick(float* __restrict__ X, float* __restrict__ Y, float* __restrict__ VX,
                           float* __restrict__ VY, int64_t n, float maxr, int maxm,
                           const float4* __restrict__ tab, float dt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = X[i], y = Y[i];
    float ax = 0.f, ay = 0.f;
    const float rr = sqrtf(x * x + y * y);
    if (rr <= maxr) {
        const float r = fmaxf(rr, 1e-5f);
        const float c1 = x / r, s1 = y / r;
        const float u = rr / maxr * (float)(SFP_NT - 1);
        const int i0 = min(max((int)u - 1, 0), SFP_NT - 4);
        const float t = u - (float)i0;  // in [0, 3]: nodes i0 .. i0 + 3
        const float w0 = -(t - 1.f) * (t - 2.f) * (t - 3.f) * (1.f / 6.f);
        const float w1 = t * (t - 2.f) * (t - 3.f) * 0.5f;
        const float w2 = -t * (t - 1.f) * (t - 3.f) * 0.5f;
        const float w3 = t * (t - 1.f) * (t - 2.f) * (1.f / 6.f);
        float ar = 0.f, at = 0.f, cm = 1.f, sm = 0.f;
        for (int m = 0; m <= maxm; m++) {
            if (m > 0) {
                const float nc = cm * c1 - sm * s1;
                sm = sm * c1 + cm * s1;
                cm = nc;
            }
            const float4* q = tab + (size_t)m * SFP_NT + i0;
            const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
            const float fc = w0 * a.x + w1 * b.x + w2 * c.x + w3 * d.x;
            const float fs = w0 * a.y + w1 * b.y + w2 * c.y + w3 * d.y;
            const float dc = w0 * a.z + w1 * b.z + w2 * c.z + w3 * d.z;
            const float ds = w0 * a.w + w1 * b.w + w2 * c.w + w3 * d.w;
            if (m == 0) {
                ar += dc;
            } else {
                ar += dc * cm + ds * sm;
                at += (float)m * (fs * cm - fc * sm);
            }
        }
        at = at * maxr / r;
        ax = ar * c1 - at * s1;
        ay = ar * s1 + at * c1;
    }
    const float vx = VX[i] + ax * dt, vy = VY[i] + ay * dt;
    VX[i] = vx;
    VY[i] = vy;
    X[i] = x + vx * dt;
    Y[i] = y + vy * dt;
}

// ---------------------------------------------------------------------------
#define SFP_CUDA(s, call)                                                        \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            (s)->err = std::string(#call) + ": " + cudaGetErrorString(e_);       \
            return GX_ERR_CUDA;                                                  \
        }                                                                        \
    } while (0)

extern "C" int gx_sfp_init(const GxSfpBasis* b, double maxr, int device, GxSfp** out) {
    if (!b || !out || !(maxr > 0.0)) return g_sfp_err = "null argument or maxr <= 0", GX_ERR_ARG;
    *out = nullptr;
    if (b->minm < 0 || b->maxm < b->minm || b->minn < 0 || b->maxn < b->minn || b->nsect < 1 ||
        b->k < 0 || !b->xcoeff || (b->maxn > 0 && !b->roots))
        return g_sfp_err = "invalid basis selection", GX_ERR_ARG;
    if (b->maxm > 11) return g_sfp_err = "maxm > 11 not supported", GX_ERR_RANGE;
    // U_nm / p^(m mod 2) has degree n + k + (m - m mod 2) / 2 in x = 2 p^2 - 1:
    // that many Chebyshev terms plus one, 32 or 64
    const int deg = b->maxn + b->k + b->maxm / 2;
    if (deg + 1 > 64) return g_sfp_err = "maxn + k + maxm / 2 + 1 > 64 not supported", GX_ERR_RANGE;
    GxSfp* s = new GxSfp();
    s->b = *b;
    s->roots.assign(b->roots ? b->roots : b->xcoeff,
                    (b->roots ? b->roots : b->xcoeff) +
                        (b->roots ? (size_t)(b->maxm + 1) * (b->maxn + 1) * b->maxn : 0));
    s->xcoeff.assign(b->xcoeff, b->xcoeff + (size_t)(b->maxm + 1) * (b->maxn + 1) * (b->k + 1));
    s->b.roots = s->roots.data();
    s->b.xcoeff = s->xcoeff.data();
    s->maxr = maxr;
    for (int m = b->minm; m <= b->maxm; m += b->nsect)
        for (int n = b->minn; n <= b->maxn; n++) {
            s->msel.push_back(m);
            s->nsel.push_back(n);
        }
    s->nfun = (int)s->msel.size();
    s->D = (deg + 1 <= 32) ? 32 : 64;
    s->NC = 2 * b->maxm + 1;
    cheb_coeffs(s);
    s->dev = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->e1);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->mom, sizeof(double) * SFP_MAXMOM);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->upart, sizeof(double) * (size_t)s->nsm * SFP_MAXMOM);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->slab, sizeof(double) * (size_t)2 * s->nsm * SFP_MAXMOM);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->errword, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(s->errword, 0, sizeof(int32_t));
    if (e != cudaSuccess) {
        g_sfp_err = std::string("CUDA: ") + cudaGetErrorString(e);
        delete s;
        return GX_ERR_CUDA;
    }
    *out = s;
    return GX_OK;
}

extern "C" void gx_sfp_destroy(GxSfp* s) {
    if (!s) return;
    cudaSetDevice(s->dev);
    if (s->stream) cudaStreamSynchronize(s->stream);
    void* p[] = {s->xy, s->vel, s->ftab, s->part, s->mom, s->qc, s->upart, s->slab, s->errword};
    for (void* q : p)
        if (q) cudaFree(q);
    if (s->e0) cudaEventDestroy(s->e0);
    if (s->e1) cudaEventDestroy(s->e1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

extern "C" const char* gx_sfp_last_error(const GxSfp* s) { return s ? s->err.c_str() : g_sfp_err.c_str(); }

// records (x, y[, vx, vy], ...) -> SoA positions and velocities (zero when
// the records carry none)
__global__ void k_sfp_xy(const float* __restrict__ aos, int stride, int64_t n, int64_t cap,
                         float* __restrict__ xy, float* __restrict__ vel) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    xy[i] = aos[i * stride];
    xy[cap + i] = aos[i * stride + 1];
    vel[i] = stride >= 4 ? aos[i * stride + 2] : 0.f;
    vel[cap + i] = stride >= 4 ? aos[i * stride + 3] : 0.f;
}

// SoA -> records (x, y, vx, vy)
__global__ void k_sfp_unxy(const float* __restrict__ xy, const float* __restrict__ vel, int64_t n, int64_t cap,
                           float4* __restrict__ aos) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    aos[i] = make_float4(xy[i], xy[cap + i], vel[i], vel[cap + i]);
}

extern "C" int gx_sfp_load(GxSfp* s, const float* coords, int64_t n, int stride) {
    if (!s || n < 0 || stride < 2 || (n > 0 && !coords)) return GX_ERR_ARG;
    cudaSetDevice(s->dev);
    if (n > s->cap) {
        if (s->xy) cudaFree(s->xy);
        if (s->vel) cudaFree(s->vel);
        if (s->part) cudaFree(s->part);
        s->xy = nullptr;
        s->vel = nullptr;
        s->part = nullptr;
        s->cap = std::max<int64_t>(n, 1);
        SFP_CUDA(s, cudaMalloc((void**)&s->xy, sizeof(float) * 2 * s->cap));
        SFP_CUDA(s, cudaMalloc((void**)&s->vel, sizeof(float) * 2 * s->cap));
        const int64_t nw = (s->cap + SFP_CHUNK - 1) / SFP_CHUNK;
        const int64_t nb = (s->cap + 255) / 256;
        const size_t bytes = std::max(sizeof(float) * nw * 64 * 32, sizeof(double) * nb * 64 * 32);
        SFP_CUDA(s, cudaMalloc((void**)&s->part, bytes));
    }
    s->n = n;
    if (n == 0) return GX_OK;
    float* tmp = nullptr;
    SFP_CUDA(s, cudaMallocAsync((void**)&tmp, sizeof(float) * stride * n, s->stream));
    SFP_CUDA(s, cudaMemcpyAsync(tmp, coords, sizeof(float) * stride * n, cudaMemcpyHostToDevice, s->stream));
    k_sfp_xy<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(tmp, stride, n, s->cap, s->xy, s->vel);
    SFP_CUDA(s, cudaGetLastError());
    SFP_CUDA(s, cudaFreeAsync(tmp, s->stream));
    SFP_CUDA(s, cudaStreamSynchronize(s->stream));
    return GX_OK;
}

// ---------------------------------------------------------------------------
// Moments on the 5th-generation tensor cores (tcgen05, TMEM accumulator).
//
// One tcgen05.mma.cta_group::1.kind::f16 per 16 particles, M = 128, N = 48,
// K = 16, FP32 accumulation in TMEM, both operands MN-major in shared
// memory without swizzle, so that every particle's features are 16-byte
// row vectors (one st.shared.v4 per 8 values):
//   A rows  0..15  T_d hi (FP16) for even d = 2i, rows 16..31 for odd
//   d = 2i + 1; rows 32..63 the lo parts (T_d - hi) in the same order;
//   rows 64..127 are not used (the descriptor's M blocks 8..15 fall on the
//   next K-block, read by the MMA, never read back).
//   B columns 0..15 g_n hi (n = 1..16: cos m phi, sin m phi, m = 1..8,
//   times p for odd m), 16..31 the lo parts, 32 g_0 = 1, 33..47 zero.
// D[r][c] in TMEM then holds every product of the hi/lo split:
//   M[d][0] = D[h][32] + D[h + 32][32],
//   M[d][c] = D[h][c-1] + D[h][c+15] + D[h+32][c-1] + D[h+32][c+15]
// with h = d / 2 for even d and 16 + d / 2 for odd d (summed on the host).
// Canonical MN-major layout: a core matrix is 8 K-rows (particles) of 16
// bytes (8 consecutive M or N elements), 128 bytes contiguous; M / N blocks
// of 8 are SBO = 128 bytes apart, K-blocks of 8 particles LBO = 1024 (A) /
// 768 (B) bytes apart.  A warp's 32 particles write 4 K-blocks: the 8 lanes
// of a K-block fill one 128-byte core matrix, so the stores are conflict
// free.
// A CTA (one per SM) has 16 producer warps, two threads per particle: the
// "even" thread runs T_0, T_2, .. (T_{d+2} = 2 T_2 T_d - T_{d-2}) and g for
// m = 1..4, the "odd" thread T_1, T_3, .. and g for m = 5..8 (from z^4) and
// the column of ones.  Rounds of 256 particles, three stages; warp 18 waits
// for a stage, issues its 16 MMAs and commits them to the stage's empty
// barrier.  The accumulator alternates between two TMEM regions, one per
// group of UM_DRAIN rounds (1024 particles): after a group's last MMA the
// issuer commits to that region's barrier, and warps 16 and 17 (TMEM lanes
// 0..31 and 32..63) add it in FP64 into the CTA's partial rows in global
// memory, then release the region, while the MMAs of the next group run
// into the other one.  Waits are bounded; on time-out the CTA raises the
// error word, waits (bounded) for its issued MMAs and frees its TMEM.
#define UM_T 256                    // particles per round
#define UM_PROD 512                 // producer threads (two per particle)
#define UM_THREADS (UM_PROD + 96)   // + drain warps 16, 17 and the issue warp 18
#define UM_KB (UM_T / 8)            // K-blocks per round
#define UM_N 48
#define UM_AKB 1024                 // A bytes per K-block (8 blocks x 128)
#define UM_BKB 768                  // B bytes per K-block (6 blocks x 128)
#define UM_ABYTES (UM_KB * UM_AKB + UM_AKB)  // + M blocks 8..15 of the last K-block
#define UM_BUFBYTES (UM_ABYTES + UM_KB * UM_BKB)
#define UM_NBUF 3
#define UM_DRAIN 4                  // rounds per accumulator group
#define UM_TMEM_COLS 128            // two regions of UM_N columns, 64 apart
#define UM_NRAW (64 * UM_N)         // partial row entries per CTA
static_assert(UM_NRAW <= SFP_MAXMOM, "raw rows fit the moment buffers");
#define UM_SPIN (1u << 22)

__device__ __forceinline__ uint32_t um_smem(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
// shared-memory matrix descriptor: start, LBO (K-block stride), SBO (M / N
// block stride), in 16-byte units; version 1, base offset 0, no swizzle
__device__ __forceinline__ uint64_t um_desc(uint32_t saddr, uint32_t lbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((128u >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// instruction descriptor: D F32, A and B F16, both MN-major, N = 48, M = 128
#define UM_IDESC ((1u << 4) | (0u << 7) | (0u << 10) | (1u << 15) | (1u << 16) | \
                  ((uint32_t)(UM_N >> 3) << 17) | (8u << 24))

__device__ __forceinline__ void um_mma(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %4, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(ad), "l"(bd), "r"(accumulate), "r"(UM_IDESC), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void um_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     um_smem(mbar))
                 : "memory");
}
__device__ __forceinline__ bool um_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(um_smem(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool um_wait(uint64_t* b, uint32_t parity) {
    for (uint32_t i = 0; i < UM_SPIN; i++)
        if (um_try(b, parity)) return true;
    return false;
}
// the same for the issue and drain warps, which wait most of the time: a
// short sleep between tries leaves the issue slots to the producers
__device__ __forceinline__ bool um_wait_idle(uint64_t* b, uint32_t parity) {
    for (uint32_t i = 0; i < UM_SPIN; i++) {
        if (um_try(b, parity)) return true;
        __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void um_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(um_smem(b)) : "memory");
}
__device__ __forceinline__ void um_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void um_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// 8 consecutive FP32 columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void um_ld8(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
// hi / lo halves of eight values into two 16-byte row vectors
__device__ __forceinline__ void um_split8(const float* v, uint4& h, uint4& l) {
    split_h2(v[0], v[1], h.x, l.x);
    split_h2(v[2], v[3], h.y, l.y);
    split_h2(v[4], v[5], h.z, l.z);
    split_h2(v[6], v[7], h.w, l.w);
}

__global__ void __launch_bounds__(UM_THREADS, 1) k_sfp_umma(const float* __restrict__ X,
                                                            const float* __restrict__ Y, int64_t n,
                                                            float inv_maxr, int maxm,
                                                            double* __restrict__ raw,
                                                            int32_t* __restrict__ errword) {
    extern __shared__ __align__(1024) unsigned char um_sm[];
    __shared__ __align__(8) uint64_t full[UM_NBUF], empty[UM_NBUF], accfull[2], drained[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int DW0 = UM_PROD / 32, ISW = DW0 + 2;  // drain warps DW0, DW0 + 1; issue warp
    static_assert(DW0 % 4 == 0, "the drain warps read TMEM lanes 0..31 and 32..63");
    if (tid == 0) {
        for (int b = 0; b < UM_NBUF; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(um_smem(&full[b])), "r"(UM_PROD / 32)
                         : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(um_smem(&empty[b])) : "memory");
        }
        for (int a = 0; a < 2; a++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(um_smem(&accfull[a])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(um_smem(&drained[a])) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // zero every stage once (B columns 33..47, the rows past the last K-block)
    for (int i = tid; i < UM_NBUF * UM_BUFBYTES / 16; i += UM_THREADS)
        reinterpret_cast<uint4*>(um_sm)[i] = make_uint4(0u, 0u, 0u, 0u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == ISW) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(um_smem(&tmem_slot)),
                     "r"(UM_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    um_fence_before();
    __syncthreads();
    um_fence_after();
    const uint32_t tmem = tmem_slot;
    const int64_t rounds_total = (n + UM_T - 1) / UM_T;
    const int64_t my_rounds = (blockIdx.x < rounds_total) ? (rounds_total - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int64_t ngroups = (my_rounds + UM_DRAIN - 1) / UM_DRAIN;

    if (warp < DW0) {
        // ------------------------------------------------------------ producers
        const int pt = tid & (UM_T - 1), odd = tid / UM_T;  // particle of the round, its half
        const int kb = pt >> 3, r = pt & 7;
        float nx = 0.f, ny = 0.f;
        bool nv = false;
        if (my_rounds > 0) {
            const int64_t i = (int64_t)blockIdx.x * UM_T + pt;
            if (i < n) {
                nx = __ldg(X + i);
                ny = __ldg(Y + i);
                nv = true;
            }
        }
        for (int64_t li = 0; li < my_rounds; li++) {
            const int64_t rnd = blockIdx.x + li * gridDim.x;
            // a slot past the last particle sits outside the basis edge
            const float px = nv ? nx * inv_maxr : 2.f, py = nv ? ny * inv_maxr : 0.f;
            {
                const int64_t i = (rnd + gridDim.x) * UM_T + pt;
                nv = false;
                if (li + 1 < my_rounds && i < n) {
                    nx = __ldg(X + i);
                    ny = __ldg(Y + i);
                    nv = true;
                }
            }
            const float p2 = px * px + py * py;
            const bool act = p2 <= 1.0f;
            const float sw = act ? 1.f : 0.f;
            const float xc = act ? 2.f * p2 - 1.f : 0.f, x2 = 2.f * xc;
            const float y2 = 2.f * fmaf(x2, xc, -1.f);  // 2 T_2(x)
            // |p| and the direction (x, y) / |p| from one reciprocal square root
            const float rs = (act && p2 > 0.f) ? rsqrtf(p2) : 0.f;
            const float pr = p2 * rs;
            const bool dir = rs > 0.f;
            const float cr = dir ? px * rs : 1.f, ci = dir ? py * rs : 0.f;
            // T_{odd + 2j}, j = 0..15 (seeded with sw: zero outside the edge)
            float t[16];
            t[0] = odd ? sw * xc : sw;
            t[1] = odd ? fmaf(x2, fmaf(x2, sw * xc, -sw), -sw * xc) : fmaf(x2, sw * xc, -sw);
#pragma unroll
            for (int j = 2; j < 16; j++) t[j] = fmaf(y2, t[j - 1], -t[j - 2]);
            // g for m = 1..4 (even half) or 5..8 (odd half)
            float g[8];
            {
                float zr = sw, zi = 0.f;
                if (odd) {  // z^4
                    const float ar = cr * cr - ci * ci, ai = 2.f * cr * ci;
                    zr = sw * (ar * ar - ai * ai);
                    zi = sw * (2.f * ar * ai);
                }
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int m = 4 * odd + k + 1;
                    const float nr = zr * cr - zi * ci;
                    zi = zr * ci + zi * cr;
                    zr = nr;
                    const bool on = m <= maxm;
                    const float f = (m & 1) ? pr : 1.f;
                    g[2 * k] = on ? zr * f : 0.f;
                    g[2 * k + 1] = on ? zi * f : 0.f;
                }
            }
            const int b = (int)(li % UM_NBUF);
            // warp-uniform: a lane that timed out takes its whole warp out
            if (li >= UM_NBUF &&
                !__all_sync(0xffffffffu, um_wait(&empty[b], (uint32_t)(((li / UM_NBUF) - 1) & 1)))) {
                if (lane == 0) atomicExch(errword, 5);
                break;
            }
            unsigned char* A = um_sm + (size_t)b * UM_BUFBYTES + kb * UM_AKB + r * 16;
            unsigned char* B = um_sm + (size_t)b * UM_BUFBYTES + UM_ABYTES + kb * UM_BKB + r * 16;
            uint4 h, l;
            um_split8(t, h, l);  // d = odd + 0, 2, .., 14: M block 2 odd (hi), 4 + 2 odd (lo)
            *reinterpret_cast<uint4*>(A + (2 * odd) * 128) = h;
            *reinterpret_cast<uint4*>(A + (4 + 2 * odd) * 128) = l;
            um_split8(t + 8, h, l);  // d = odd + 16, .., 30
            *reinterpret_cast<uint4*>(A + (2 * odd + 1) * 128) = h;
            *reinterpret_cast<uint4*>(A + (5 + 2 * odd) * 128) = l;
            um_split8(g, h, l);  // columns 8 odd .. + 7: N block odd (hi), 2 + odd (lo)
            *reinterpret_cast<uint4*>(B + odd * 128) = h;
            *reinterpret_cast<uint4*>(B + (2 + odd) * 128) = l;
            if (odd) *reinterpret_cast<uint4*>(B + 4 * 128) = make_uint4(act ? 0x3C00u : 0u, 0u, 0u, 0u);
            // generic-proxy stores -> async proxy (the tensor core reads shared memory)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) um_arrive(&full[b]);
        }
    } else if (warp == ISW) {
        // ------------------------------------------------------------ MMA issue
        bool ok = true;
        int64_t last = -1;  // last round whose MMAs were committed
        for (int64_t li = 0; li < my_rounds && ok; li++) {
            const int b = (int)(li % UM_NBUF);
            const int64_t grp = li / UM_DRAIN;
            const int acc = (int)(grp & 1);
            const bool first = (li % UM_DRAIN) == 0;
            const bool lastr = (li % UM_DRAIN) == UM_DRAIN - 1 || li + 1 == my_rounds;
            if (first && grp >= 2) ok = __all_sync(0xffffffffu, um_wait_idle(&drained[acc], (uint32_t)(((grp / 2) - 1) & 1)));
            if (ok) ok = __all_sync(0xffffffffu, um_wait_idle(&full[b], (uint32_t)((li / UM_NBUF) & 1)));
            if (!ok) {
                if (lane == 0) atomicExch(errword, 5);
                break;
            }
            um_fence_after();
            if (lane == 0) {
                const uint32_t a0 = um_smem(um_sm + (size_t)b * UM_BUFBYTES), b0 = a0 + UM_ABYTES;
                const uint32_t td = tmem + (uint32_t)(64 * acc);
#pragma unroll 1
                for (int k = 0; k < UM_KB / 2; k++)
                    um_mma(td, um_desc(a0 + k * 2 * UM_AKB, UM_AKB), um_desc(b0 + k * 2 * UM_BKB, UM_BKB),
                           (first && k == 0) ? 0u : 1u);
                um_commit(&empty[b]);
                if (lastr) um_commit(&accfull[acc]);
            }
            __syncwarp();
            last = li;
        }
        if (last >= 0 && lane == 0)  // every issued MMA has completed (bounded)
            um_wait(&empty[(int)(last % UM_NBUF)], (uint32_t)((last / UM_NBUF) & 1));
        __syncwarp();
    } else {
        // ------------------------------------------------- drain (TMEM -> FP64)
        const int q = warp - DW0;  // TMEM lanes 32 q .. 32 q + 31
        double* row = raw + ((size_t)blockIdx.x * 64 + 32 * q + lane) * UM_N;
        if (ngroups == 0)
            for (int c = 0; c < UM_N; c++) row[c] = 0.0;
        for (int64_t grp = 0; grp < ngroups; grp++) {
            const int acc = (int)(grp & 1);
            if (!__all_sync(0xffffffffu, um_wait_idle(&accfull[acc], (uint32_t)((grp / 2) & 1)))) {
                if (lane == 0) atomicExch(errword, 5);
                break;
            }
            um_fence_after();
            float v[UM_N];
#pragma unroll
            for (int c = 0; c < UM_N; c += 8)
                um_ld8(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(64 * acc + c), v + c);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            um_fence_before();
            __syncwarp();
            if (lane == 0) um_arrive(&drained[acc]);
#pragma unroll
            for (int c = 0; c < UM_N; c += 2) {
                double2 s = make_double2((double)v[c], (double)v[c + 1]);
                if (grp > 0) {
                    const double2 o = *reinterpret_cast<const double2*>(row + c);
                    s.x += o.x;
                    s.y += o.y;
                }
                *reinterpret_cast<double2*>(row + c) = s;
            }
        }
    }
    um_fence_before();
    __syncthreads();
    um_fence_after();
    if (warp == ISW)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UM_TMEM_COLS)
                     : "memory");
}

// mom = the FP64 sum of the nrow partial rows part[nrow][nmom]: slabs of
// rows summed coalesced (at most 2 per SM), then the slab sums
template <typename T>
static int sfp_sum_rows(GxSfp* s, const T* part, int64_t nrow, int nmom) {
    const int64_t nslab = std::min<int64_t>(nrow, 2 * (int64_t)s->nsm);
    const int64_t rpb = (nrow + nslab - 1) / nslab;
    const int nsl = (int)((nrow + rpb - 1) / rpb);
    k_sfp_slab<T><<<nsl, 256, 0, s->stream>>>(part, nrow, nmom, rpb, s->slab);
    SFP_CUDA(s, cudaGetLastError());
    k_sfp_reduce<double><<<nmom, 256, 0, s->stream>>>(s->slab, nsl, nmom, s->mom);
    SFP_CUDA(s, cudaGetLastError());
    s->launches += 2;
    return GX_OK;
}

// moments on the device (precision GX_PREC_MIXED: tensor cores; GX_PREC_FP64: CUDA cores)
static int sfp_moments(GxSfp* s, int precision) {
    const int D = s->D, NCP = (s->NC + 7) / 8 * 8, nmom = D * NCP;
    const int64_t n = s->n;
    if (precision == GX_PREC_FP64) {
        const int64_t nb = (n + 255) / 256;
        const size_t sm = sizeof(double) * 256 * (D + NCP);
        SFP_CUDA(s, cudaFuncSetAttribute(k_sfp_moments64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_sfp_moments64<<<(unsigned)nb, 256, sm, s->stream>>>(s->xy, s->xy + s->cap, n, 1.0 / s->maxr,
                                                              s->b.maxm, D, NCP, (double*)s->part);
        SFP_CUDA(s, cudaGetLastError());
        s->launches += 1;
        return sfp_sum_rows<double>(s, (const double*)s->part, nb, nmom);
    }
    const float inv = (float)(1.0 / s->maxr);
    if (precision == GX_PREC_MIXED_TC05) {
        if (D != 32 || s->NC > 17)
            return s->err = "the tcgen05 path takes at most 32 Chebyshev terms and maxm <= 8", GX_ERR_RANGE;
        // tcgen05: one CTA per SM (at most), FP64 partial rows [64][UM_N] per CTA
        const int64_t rounds = (n + UM_T - 1) / UM_T;
        const int grid = (int)std::min<int64_t>(rounds, s->nsm);
        // (+ 4 KB past the stages: no descriptor-addressed read can leave the allocation)
        const size_t sm = (size_t)UM_NBUF * UM_BUFBYTES + 4096;
        SFP_CUDA(s, cudaFuncSetAttribute(k_sfp_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_sfp_umma<<<grid, UM_THREADS, sm, s->stream>>>(s->xy, s->xy + s->cap, n, inv, s->b.maxm, s->upart,
                                                         s->errword);
        SFP_CUDA(s, cudaGetLastError());
        s->launches += 1;
        return sfp_sum_rows<double>(s, s->upart, grid, UM_NRAW);
    }
    const int64_t nw = (n + SFP_CHUNK - 1) / SFP_CHUNK;
    const unsigned grid = (unsigned)((nw * 32 + 255) / 256);
    // feature columns 1 .. NC - 1 in blocks of 8
    const int NB = (s->NC - 1 + 7) / 8;
    if (NB > 3) return s->err = "more than 11 harmonics on the tensor-core path", GX_ERR_RANGE;
    const size_t sm = sizeof(__half) * 8 * 2 * 32 * ((size_t)(D + 8) + (NB == 3 ? 40 : 24));
    auto k = (D == 32) ? ((NB <= 1) ? k_sfp_moments<2, 1> : (NB == 2) ? k_sfp_moments<2, 2> : k_sfp_moments<2, 3>)
                       : ((NB <= 1) ? k_sfp_moments<4, 1> : (NB == 2) ? k_sfp_moments<4, 2> : k_sfp_moments<4, 3>);
    SFP_CUDA(s, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k<<<grid, 256, sm, s->stream>>>(s->xy, s->xy + s->cap, n, inv, s->b.maxm, NCP, s->part);
    SFP_CUDA(s, cudaGetLastError());
    s->launches += 1;
    return sfp_sum_rows<float>(s, s->part, nw, nmom);
}

// sfpsum + scaled: coeff[n * (2 maxm + 1) + m + maxm] (cosine +m, sine -m)
static int sfp_coeff(GxSfp* s, int precision, double pmass, double* coeff) {
    const int D = s->D, NCP = (s->NC + 7) / 8 * 8;
    const int ngx = 2 * s->b.maxm + 1, maxm = s->b.maxm;
    std::vector<double> mom((size_t)D * NCP, 0.0);
    s->launches = 0;
    SFP_CUDA(s, cudaEventRecord(s->e0, s->stream));
    if (s->n > 0) {
        int rc = sfp_moments(s, precision);
        if (rc) return rc;
    }
    SFP_CUDA(s, cudaEventRecord(s->e1, s->stream));
    std::vector<double> raw;
    if (s->n > 0 && precision == GX_PREC_MIXED_TC05) {
        raw.resize(UM_NRAW);
        SFP_CUDA(s, cudaMemcpyAsync(raw.data(), s->mom, sizeof(double) * UM_NRAW, cudaMemcpyDeviceToHost, s->stream));
    } else if (s->n > 0)
        SFP_CUDA(s, cudaMemcpyAsync(mom.data(), s->mom, sizeof(double) * D * NCP, cudaMemcpyDeviceToHost, s->stream));
    SFP_CUDA(s, cudaStreamSynchronize(s->stream));
    if (!raw.empty()) {
        // the tcgen05 rows: T_d hi at row h (h = d / 2 for even d, 16 + d / 2
        // for odd d), lo at h + 32; columns g hi 0..15, g lo 16..31, ones 32
        for (int d = 0; d < D; d++) {
            const double* rh = raw.data() + (size_t)((d & 1) ? 16 + d / 2 : d / 2) * UM_N;
            const double* rl = rh + 32 * UM_N;
            mom[(size_t)d * NCP] = rh[32] + rl[32];
            for (int c = 1; c < NCP; c++)
                mom[(size_t)d * NCP + c] = (c <= 16) ? rh[c - 1] + rh[c + 15] + rl[c - 1] + rl[c + 15] : 0.0;
        }
    }
    SFP_CUDA(s, cudaEventElapsedTime(&s->last_ms, s->e0, s->e1));
    {
        int32_t ew = 0;
        SFP_CUDA(s, cudaMemcpy(&ew, s->errword, sizeof ew, cudaMemcpyDeviceToHost));
        if (ew) {
            cudaMemset(s->errword, 0, sizeof ew);
            return s->err = "device check raised the error word", GX_ERR_DEVICE;
        }
    }
    memset(coeff, 0, sizeof(double) * (size_t)(s->b.maxn + 1) * ngx);
    const double fac = pmass / (s->maxr * s->maxr);
    for (int f = 0; f < s->nfun; f++) {
        const int m = s->msel[f], n = s->nsel[f];
        const double* a = s->acheb.data() + (size_t)f * D;
        const int cc = (m == 0) ? 0 : 2 * m - 1, cs = 2 * m;
        double vc = 0, vs = 0;
        for (int d = 0; d < D; d++) {
            vc += a[d] * mom[(size_t)d * NCP + cc];
            if (m > 0) vs += a[d] * mom[(size_t)d * NCP + cs];
        }
        const int k = n * ngx + maxm;
        coeff[k + m] = vc * fac;
        if (m > 0) coeff[k - m] = vs * fac;
    }
    return GX_OK;
}

extern "C" int gx_sfp_sum(GxSfp* s, int precision, double pmass, double* coeff) {
    if (!s || !coeff) return GX_ERR_ARG;
    if (precision != GX_PREC_MIXED && precision != GX_PREC_FP64 && precision != GX_PREC_MIXED_TC05)
        return GX_ERR_ARG;
    cudaSetDevice(s->dev);
    return sfp_coeff(s, precision, pmass, coeff);
}

// the per-m Chebyshev series of the force evaluation from scaled
// coefficients, uploaded to s->qc (stream-ordered)
static int sfp_series(GxSfp* s, const double* coeff) {
    const int D = s->D, maxm = s->b.maxm, ngx = 2 * maxm + 1;
    // the previous upload from this buffer has completed (every caller syncs the stream)
    s->qs_h.assign((size_t)2 * (maxm + 1) * D, 0.0);
    for (int f = 0; f < s->nfun; f++) {
        const int m = s->msel[f], n = s->nsel[f];
        const double* a = s->acheb.data() + (size_t)f * D;
        const int l = n * ngx + maxm;
        const double cr = coeff[l + m], ci = (m > 0) ? coeff[l - m] : 0.0;
        for (int d = 0; d < D; d++) {
            s->qs_h[((size_t)0 * (maxm + 1) + m) * D + d] += cr * a[d];
            s->qs_h[((size_t)1 * (maxm + 1) + m) * D + d] += ci * a[d];
        }
    }
    if (!s->qc) SFP_CUDA(s, cudaMalloc((void**)&s->qc, sizeof(double) * 2 * 12 * 64));
    SFP_CUDA(s, cudaMemcpyAsync(s->qc, s->qs_h.data(), sizeof(double) * s->qs_h.size(), cudaMemcpyHostToDevice,
                                s->stream));
    return GX_OK;
}

// sfpacc for the loaded particles from scaled coefficients; acc [n][2], pot [n]
extern "C" int gx_sfp_acc(GxSfp* s, const double* coeff, float* acc, float* pot) {
    if (!s || !coeff || (!acc && s->n > 0)) return GX_ERR_ARG;
    cudaSetDevice(s->dev);
    const int D = s->D, maxm = s->b.maxm;
    int rc = sfp_series(s, coeff);
    if (rc) return rc;
    const int64_t n = s->n;
    if (n > 0) {
        float *dacc = nullptr, *dpot = nullptr;
        SFP_CUDA(s, cudaMallocAsync((void**)&dacc, sizeof(float) * 2 * n, s->stream));
        SFP_CUDA(s, cudaMallocAsync((void**)&dpot, sizeof(float) * n, s->stream));
        k_sfp_acc<<<(unsigned)((n + 127) / 128), 128, 0, s->stream>>>(s->xy, s->xy + s->cap, n, s->maxr,
                                                                    maxm, D, s->qc, dacc, dpot);
        SFP_CUDA(s, cudaGetLastError());
        SFP_CUDA(s, cudaMemcpyAsync(acc, dacc, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, s->stream));
        if (pot) SFP_CUDA(s, cudaMemcpyAsync(pot, dpot, sizeof(float) * n, cudaMemcpyDeviceToHost, s->stream));
        SFP_CUDA(s, cudaFreeAsync(dacc, s->stream));
        SFP_CUDA(s, cudaFreeAsync(dpot, s->stream));
    }
    SFP_CUDA(s, cudaStreamSynchronize(s->stream));
    return GX_OK;
}

// The SFP-driven time loop (the sf2d code's step, step.f:135-290: getacc
// -> sfpacc, stpgrp, massgn -> sfpadd, then sfpsum at step.f:250): per
// step the coefficients of the current positions (gx_sfp_sum's arithmetic
// at `precision`), then one kernel that evaluates the force at each
// particle and moves it, v += a dt, x += v dt.  The particles stay on the
// device; coeff_out (may be NULL) receives the coefficients of the final
// positions.
extern "C" int gx_sfp_step(GxSfp* s, int nsteps, double dt, int precision, double pmass, double* coeff_out) {
    if (!s || nsteps < 0) return GX_ERR_ARG;
    if (precision != GX_PREC_MIXED && precision != GX_PREC_FP64 && precision != GX_PREC_MIXED_TC05)
        return GX_ERR_ARG;
    cudaSetDevice(s->dev);
    const int ngx = 2 * s->b.maxm + 1;
    std::vector<double> coeff((size_t)(s->b.maxn + 1) * ngx);
    const int64_t n = s->n;
    if (!s->ftab) SFP_CUDA(s, cudaMalloc((void**)&s->ftab, sizeof(float4) * 12 * SFP_NT));
    for (int k = 0; k < nsteps; k++) {
        int rc = sfp_coeff(s, precision, pmass, coeff.data());
        if (rc) return rc;
        rc = sfp_series(s, coeff.data());
        if (rc) return rc;
        if (n > 0) {
            const int nt = (s->b.maxm + 1) * SFP_NT;
            k_sfp_ftab<<<(unsigned)((nt + 127) / 128), 128, 0, s->stream>>>(s->b.maxm, s->D, s->qc, s->ftab);
            SFP_CUDA(s, cudaGetLastError());
            k_sfp_kick<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(
                s->xy, s->xy + s->cap, s->vel, s->vel + s->cap, n, (float)s->maxr, s->b.maxm, s->ftab, (float)dt);
            SFP_CUDA(s, cudaGetLastError());
        }
    }
    if (coeff_out) {
        int rc = sfp_coeff(s, precision, pmass, coeff_out);
        if (rc) return rc;
    }
    SFP_CUDA(s, cudaStreamSynchronize(s->stream));
    return GX_OK;
}

// the loaded particles back as records (x, y, vx, vy)
extern "C" int gx_sfp_unload(GxSfp* s, float* coords) {
    if (!s || (s->n > 0 && !coords)) return GX_ERR_ARG;
    cudaSetDevice(s->dev);
    const int64_t n = s->n;
    if (n == 0) return GX_OK;
    float4* tmp = nullptr;
    SFP_CUDA(s, cudaMallocAsync((void**)&tmp, sizeof(float4) * n, s->stream));
    k_sfp_unxy<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(s->xy, s->vel, n, s->cap, tmp);
    SFP_CUDA(s, cudaGetLastError());
    SFP_CUDA(s, cudaMemcpyAsync(coords, tmp, sizeof(float4) * n, cudaMemcpyDeviceToHost, s->stream));
    SFP_CUDA(s, cudaFreeAsync(tmp, s->stream));
    SFP_CUDA(s, cudaStreamSynchronize(s->stream));
    return GX_OK;
}

extern "C" int gx_sfp_last_ms(const GxSfp* s, float* ms, int64_t* launches) {
    if (!s || !ms) return GX_ERR_ARG;
    *ms = s->last_ms;
    if (launches) *launches = s->launches;
    return GX_OK;
}
