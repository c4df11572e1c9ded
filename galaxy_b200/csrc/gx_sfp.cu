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
// (particles): it runs on the tensor cores with mma.sync m16n8k8 TF32,
// each operand split hi + lo (three products, FP32 accumulate per warp over
// a chunk of particles, chunks summed in FP64).  The fragments are formed
// in registers from each lane's particles: no shared-memory staging of
// per-particle features, which would otherwise bound the kernel.
// a_nmd are formed once on the host in FP64 from the roots and
// coefficients of the basis (Chebyshev interpolation at 64 nodes).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "gx_common.cuh"

#define SFP_CHUNK 1024  // particles per warp-chunk (FP32 accumulation span)

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
    float* part = nullptr;      // per-warp partial moments
    double* mom = nullptr;      // [D][NCP] FP64 moments
    double* qc = nullptr;       // device force series [2][maxm+1][D]
    double* upart = nullptr;    // per-CTA FP64 partial moments of the tcgen05 path
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

__device__ __forceinline__ void mma_tf32(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Moments of one SFP_CHUNK of particles per warp; part[warp][d][c].
// Rounds of 32 particles: lane l computes the features of particle l once --
// T_d(x) for d < D by the three-term recurrence, and g_n (n >= 1) =
// p^e cos m phi, p^e sin m phi (e = m mod 2) from repeated multiplication of
// (x, y) / r -- into the warp's shared-memory tiles Ts[32][D + 8] and
// Gs[32][GSTR] (padded so that the fragment loads below hit 32 distinct
// banks).  Column c = 0 (g_0 = 1) is the plain sum of T_d, taken on the CUDA
// cores (lane d); columns 1 .. NB*8 come from mma.sync m16n8k8 TF32 with the
// operands split hi/lo (3 products), FP32 accumulation over the chunk.
#define SFP_GSTR 24  // >= 8 NB, and 24 p mod 32 spreads c4 over banks
template <int MT, int NB>
__global__ void __launch_bounds__(256) k_sfp_moments(const float* __restrict__ X,
                                                     const float* __restrict__ Y, int64_t n,
                                                     float inv_maxr, int maxm, int NCP,
                                                     float* __restrict__ part) {
    constexpr int D = MT * 16, TSTR = D + 8;
    extern __shared__ __align__(16) float sfs[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    float* Ts = sfs + (size_t)wib * 32 * (TSTR + SFP_GSTR);
    float* Gs = Ts + 32 * TSTR;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t base = wid * SFP_CHUNK;
    if (base >= n) return;
    const int q = lane >> 2, c4 = lane & 3;
    float acc[MT][NB][4];
#pragma unroll
    for (int a = 0; a < MT; a++)
#pragma unroll
        for (int u = 0; u < NB; u++)
#pragma unroll
            for (int i = 0; i < 4; i++) acc[a][u][i] = 0.f;
    float col0[MT / 2 > 0 ? MT / 2 : 1];  // lane d (+32): sum of T_d
#pragma unroll
    for (int h = 0; h < (MT / 2 > 0 ? MT / 2 : 1); h++) col0[h] = 0.f;
    const int64_t end = min(base + (int64_t)SFP_CHUNK, n);
    for (int64_t r0 = base; r0 < end; r0 += 32) {
        // ---- features of particle r0 + lane
        {
            const int64_t i = r0 + lane;
            float px = 2.f, py = 0.f;  // outside the basis edge: no contribution
            if (i < end) {
                px = __ldg(X + i) * inv_maxr;
                py = __ldg(Y + i) * inv_maxr;
            }
            const float p2 = px * px + py * py;
            const bool act = p2 <= 1.0f;
            const float xc = 2.f * p2 - 1.f;
            float* tr = Ts + lane * TSTR;
            float tm2 = 1.f, tm1 = xc;
            float4 v;
#pragma unroll
            for (int d = 0; d < D; d += 4) {
                float t4[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int dd = d + k;
                    float t;
                    if (dd == 0) t = 1.f;
                    else if (dd == 1) t = xc;
                    else {
                        t = 2.f * xc * tm1 - tm2;
                        tm2 = tm1;
                        tm1 = t;
                    }
                    t4[k] = act ? t : 0.f;
                }
                v = make_float4(t4[0], t4[1], t4[2], t4[3]);
                *reinterpret_cast<float4*>(tr + d) = v;
            }
            const float pr = sqrtf(p2);
            const float cr = pr > 0.f ? px / pr : 1.f, ci = pr > 0.f ? py / pr : 0.f;
            float* gr = Gs + lane * SFP_GSTR;
            float zr = 1.f, zi = 0.f;
#pragma unroll
            for (int u = 0; u < NB * 8; u += 2) {
                const int m = u / 2 + 1;
                float gc = 0.f, gs = 0.f;
                if (m <= maxm) {
                    const float nr = zr * cr - zi * ci;
                    zi = zr * ci + zi * cr;
                    zr = nr;
                    const float f = (m & 1) ? pr : 1.f;
                    gc = act ? zr * f : 0.f;
                    gs = act ? zi * f : 0.f;
                }
                gr[u] = gc;
                gr[u + 1] = gs;
            }
        }
        __syncwarp();
        // ---- column 0 on the CUDA cores
#pragma unroll 8
        for (int pp = 0; pp < 32; pp++) {
#pragma unroll
            for (int h = 0; h < (MT / 2 > 0 ? MT / 2 : 1); h++) col0[h] += Ts[pp * TSTR + lane + 32 * h];
        }
        // ---- columns 1 .. 8 NB on the tensor cores, 4 k-blocks of 8 particles
#pragma unroll
        for (int kb = 0; kb < 4; kb++) {
            const float* t0 = Ts + (8 * kb + c4) * TSTR;
            const float* t1 = t0 + 4 * TSTR;
            const float* g0 = Gs + (8 * kb + c4) * SFP_GSTR;
            const float* g1 = g0 + 4 * SFP_GSTR;
            uint32_t bh[NB][2], bl[NB][2];
#pragma unroll
            for (int u = 0; u < NB; u++) {
                const float v0 = g0[8 * u + q], v1 = g1[8 * u + q];
                bh[u][0] = f2tf32(v0);
                bl[u][0] = f2tf32(v0 - __uint_as_float(bh[u][0]));
                bh[u][1] = f2tf32(v1);
                bl[u][1] = f2tf32(v1 - __uint_as_float(bh[u][1]));
            }
#pragma unroll
            for (int a = 0; a < MT; a++) {
                // a0 = A[q][c4], a1 = A[q+8][c4], a2 = A[q][c4+4], a3 = A[q+8][c4+4]
                const float v[4] = {t0[16 * a + q], t0[16 * a + q + 8], t1[16 * a + q], t1[16 * a + q + 8]};
                uint32_t ah[4], al[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    ah[i] = f2tf32(v[i]);
                    al[i] = f2tf32(v[i] - __uint_as_float(ah[i]));
                }
#pragma unroll
                for (int u = 0; u < NB; u++) {
                    mma_tf32(acc[a][u], al, bh[u]);
                    mma_tf32(acc[a][u], ah, bl[u]);
                    mma_tf32(acc[a][u], ah, bh[u]);
                }
            }
        }
        __syncwarp();
    }
    // c0 = D[q][2c4], c1 = D[q][2c4+1], c2 = D[q+8][2c4], c3 = D[q+8][2c4+1]; column
    // n of the product is feature column n + 1
    float* dst = part + wid * (size_t)D * NCP;
#pragma unroll
    for (int a = 0; a < MT; a++)
#pragma unroll
        for (int u = 0; u < NB; u++) {
            const int r0 = a * 16 + q, cc = u * 8 + 2 * c4 + 1;
            if (cc < NCP) {
                dst[r0 * NCP + cc] = acc[a][u][0];
                dst[(r0 + 8) * NCP + cc] = acc[a][u][2];
            }
            if (cc + 1 < NCP) {
                dst[r0 * NCP + cc + 1] = acc[a][u][1];
                dst[(r0 + 8) * NCP + cc + 1] = acc[a][u][3];
            }
        }
#pragma unroll
    for (int h = 0; h < (MT / 2 > 0 ? MT / 2 : 1); h++)
        if (lane + 32 * h < D) dst[(lane + 32 * h) * NCP] = col0[h];
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

// sfpacc (sfpacc.f:41-112, 249-259) from the per-m Chebyshev series of the
// scaled coefficients: qc[(0/1)][m][d] (cosine / sine), FP64
__global__ void k_sfp_acc(const float* __restrict__ X, const float* __restrict__ Y, int64_t n,
                          double maxr, int maxm, int D, const double* __restrict__ qs,
                          float* __restrict__ acc, float* __restrict__ pot) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = X[i], y = Y[i];
    double rr = sqrt(x * x + y * y);
    double ar = 0, at = 0, ph = 0;
    if (rr <= maxr) {
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
        acc[2 * i] = (float)(ar * c1 - at * s1);
        acc[2 * i + 1] = (float)(ar * s1 + at * c1);
    } else {
        acc[2 * i] = acc[2 * i + 1] = 0.f;
    }
    if (pot) pot[i] = (float)ph;
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
    if (b->maxn + b->k + 1 > 64) return g_sfp_err = "maxn + k + 1 > 64 not supported", GX_ERR_RANGE;
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
    s->D = (b->maxn + b->k + 1 <= 32) ? 32 : 64;
    s->NC = 2 * b->maxm + 1;
    cheb_coeffs(s);
    s->dev = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->e1);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->mom, sizeof(double) * 64 * 32);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->upart, sizeof(double) * (size_t)s->nsm * 32 * 32);
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
    void* p[] = {s->xy, s->part, s->mom, s->qc, s->upart, s->errword};
    for (void* q : p)
        if (q) cudaFree(q);
    if (s->e0) cudaEventDestroy(s->e0);
    if (s->e1) cudaEventDestroy(s->e1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

extern "C" const char* gx_sfp_last_error(const GxSfp* s) { return s ? s->err.c_str() : g_sfp_err.c_str(); }

__global__ void k_sfp_xy(const float* __restrict__ aos, int stride, int64_t n, int64_t cap,
                         float* __restrict__ xy) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    xy[i] = aos[i * stride];
    xy[cap + i] = aos[i * stride + 1];
}

extern "C" int gx_sfp_load(GxSfp* s, const float* coords, int64_t n, int stride) {
    if (!s || n < 0 || stride < 2 || (n > 0 && !coords)) return GX_ERR_ARG;
    cudaSetDevice(s->dev);
    if (n > s->cap) {
        if (s->xy) cudaFree(s->xy);
        if (s->part) cudaFree(s->part);
        s->xy = nullptr;
        s->part = nullptr;
        s->cap = std::max<int64_t>(n, 1);
        SFP_CUDA(s, cudaMalloc((void**)&s->xy, sizeof(float) * 2 * s->cap));
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
    k_sfp_xy<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(tmp, stride, n, s->cap, s->xy);
    SFP_CUDA(s, cudaGetLastError());
    SFP_CUDA(s, cudaFreeAsync(tmp, s->stream));
    SFP_CUDA(s, cudaStreamSynchronize(s->stream));
    return GX_OK;
}

// ---------------------------------------------------------------------------
// Moments on the 5th-generation tensor cores (tcgen05, TMEM accumulator).
//
// One tcgen05.mma.cta_group::1.kind::tf32 per 8 particles, M = 128, N = 40,
// K = 8, both operands K-major in shared memory without swizzle:
//   A rows 0..31   T_d hi (TF32 part of T_d(x_p)), rows 32..63 T_d lo
//   (T_d - hi); rows 64..127 are not used (the tile of the next K-block,
//   read by the MMA, never read back).
//   B rows  0      g_0 = 1, rows 1..16 g_n hi, rows 17..32 g_n lo, 33..39 0.
// D[m][n] in TMEM then holds every product of the hi/lo split:
//   M[d][0] = D[d][0] + D[d+32][0],
//   M[d][c] = D[d][c] + D[d][c+16] + D[d+32][c] + D[d+32][c+16]  (c = 1..16).
// Layout of a K-block tile (UMMA canonical K-major, no swizzle): core
// matrices of 8 rows x 16 bytes; the two 16-byte halves of K are LBO = 144
// bytes apart, 8-row groups SBO = 288 bytes apart; consecutive K-blocks of a
// round are 2336 (A) / 1440 (B) bytes apart.  These strides put the 32
// scalar stores of a warp (4 K-blocks x 8 particles) on 32 distinct banks.
// A CTA of 256 threads takes rounds of 128 particles (two threads per
// particle: one writes its T rows, the other its g rows),
// triple-buffered; one thread issues the 16 MMAs of a round and commits
// them to the buffer's mbarrier.  Every UM_DRAIN rounds the accumulator is
// drained into FP64 shared memory (warps 0 and 1 read TMEM lanes 0..63)
// and the next MMA starts it afresh.  Waits are bounded; on time-out the
// CTA raises the error word, waits (bounded) for its MMAs, frees its TMEM.
#define UM_T 128          // particles per round
#define UM_THREADS 256    // threads 0..127 write the T rows, 128..255 the g rows
#define UM_KB (UM_T / 8)  // K-blocks per round
#define UM_N 40
#define UM_LBO 144
#define UM_SBO 288
#define UM_SA 2336        // A bytes per K-block (8 groups x 288 + 32)
#define UM_SB 1440        // B bytes per K-block (5 groups x 288)
#define UM_ABYTES (UM_KB * UM_SA + 8 * UM_SBO)  // + the rows 64..127 of the last K-block
#define UM_BUFBYTES (UM_ABYTES + UM_KB * UM_SB)
#define UM_NBUF 3
#define UM_DRAIN 8
#define UM_TMEM_COLS 64
#define UM_SPIN (1u << 22)

__device__ __forceinline__ uint32_t um_smem(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t um_off(int r, int k) {
    return (uint32_t)((r >> 3) * UM_SBO + (k >> 2) * UM_LBO + (r & 7) * 16 + (k & 3) * 4);
}
// shared-memory matrix descriptor: start, LBO, SBO (16-byte units), version 1
__device__ __forceinline__ uint64_t um_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((UM_LBO >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((UM_SBO >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // version
    return d;                // base offset 0, legacy LBO mode, no swizzle
}
// instruction descriptor: D F32, A and B TF32, both K-major, N = 40, M = 128
#define UM_IDESC ((1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(UM_N >> 3) << 17) | (8u << 24))

__device__ __forceinline__ void um_mma(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %4, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
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

__global__ void __launch_bounds__(UM_THREADS + 64, 1) k_sfp_umma(const float* __restrict__ X,
                                                                  const float* __restrict__ Y, int64_t n,
                                                                  float inv_maxr, int maxm,
                                                                  double* __restrict__ part, int NCP,
                                                                  int32_t* __restrict__ errword) {
    extern __shared__ __align__(1024) unsigned char um_sm[];
    __shared__ __align__(8) uint64_t full[UM_NBUF], empty[UM_NBUF];
    __shared__ uint32_t tmem_slot;
    unsigned char* buf0 = um_sm;
    double* drain = reinterpret_cast<double*>(um_sm + UM_NBUF * UM_BUFBYTES);  // [64][UM_N]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NG = 2 * maxm;  // harmonic columns g_1 .. g_NG
    const int nthr = UM_THREADS + 64;
    const int MMAW = UM_THREADS / 32;  // warps MMAW (issue + lanes 0..31), MMAW + 1 (lanes 32..63)
    if (tid == 0) {
        for (int b = 0; b < UM_NBUF; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(um_smem(&full[b])), "r"(UM_THREADS / 32)
                         : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(um_smem(&empty[b])) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 64 * UM_N; i += nthr) drain[i] = 0.0;
    // zero every buffer once (B rows past the harmonics, the padding rows)
    for (int i = tid; i < UM_NBUF * UM_BUFBYTES / 4; i += nthr) reinterpret_cast<float*>(um_sm)[i] = 0.f;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == MMAW) {
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

    if (warp < MMAW) {
        // ------------------------------------------------------------ producers
        const int pt = tid & (UM_T - 1), role = tid / UM_T;  // particle of the round, rows written
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
            const float cx = nx, cy = ny;
            const bool cv = nv;
            {
                const int64_t i = (rnd + gridDim.x) * UM_T + pt;
                nv = false;
                if (li + 1 < my_rounds && i < n) {
                    nx = __ldg(X + i);
                    ny = __ldg(Y + i);
                    nv = true;
                }
            }
            const int b = (int)(li % UM_NBUF);
            if (li >= UM_NBUF && !um_wait(&empty[b], (uint32_t)(((li / UM_NBUF) - 1) & 1))) {
                atomicExch(errword, 5);
                break;
            }
            unsigned char* A = buf0 + (size_t)b * UM_BUFBYTES;
            unsigned char* B = A + UM_ABYTES;
            // a slot past the last particle sits outside the basis edge
            const float px = cv ? cx * inv_maxr : 2.f;
            const float py = cv ? cy * inv_maxr : 0.f;
            const float p2 = px * px + py * py;
            const bool act = p2 <= 1.0f;
            const float xc = 2.f * p2 - 1.f;
            const int kb = pt >> 3, k = pt & 7;
            if (role == 0) {
                unsigned char* a = A + kb * UM_SA;
                float tm2 = 1.f, tm1 = xc;
#pragma unroll
                for (int d = 0; d < 32; d++) {
                    float t;
                    if (d == 0) t = 1.f;
                    else if (d == 1) t = xc;
                    else {
                        t = 2.f * xc * tm1 - tm2;
                        tm2 = tm1;
                        tm1 = t;
                    }
                    t = act ? t : 0.f;
                    const float hi = __uint_as_float(f2tf32(t));
                    *reinterpret_cast<float*>(a + um_off(d, k)) = hi;
                    *reinterpret_cast<float*>(a + um_off(d + 32, k)) = t - hi;
                }
            } else {
                unsigned char* bb = B + kb * UM_SB;
                *reinterpret_cast<float*>(bb + um_off(0, k)) = act ? 1.f : 0.f;
                const float pr = sqrtf(p2);
                const float cr = pr > 0.f ? px / pr : 1.f, ci = pr > 0.f ? py / pr : 0.f;
                float zr = 1.f, zi = 0.f;
#pragma unroll
                for (int u = 0; u < 16; u += 2) {
                    const int m = u / 2 + 1;
                    float gc = 0.f, gs = 0.f;
                    if (u < NG) {
                        const float nr = zr * cr - zi * ci;
                        zi = zr * ci + zi * cr;
                        zr = nr;
                        const float f = (m & 1) ? pr : 1.f;
                        gc = act ? zr * f : 0.f;
                        gs = act ? zi * f : 0.f;
                    }
                    const float hc = __uint_as_float(f2tf32(gc)), hs = __uint_as_float(f2tf32(gs));
                    *reinterpret_cast<float*>(bb + um_off(1 + u, k)) = hc;
                    *reinterpret_cast<float*>(bb + um_off(2 + u, k)) = hs;
                    *reinterpret_cast<float*>(bb + um_off(17 + u, k)) = gc - hc;
                    *reinterpret_cast<float*>(bb + um_off(18 + u, k)) = gs - hs;
                }
            }
            // generic-proxy stores -> async proxy (the tensor core reads shared memory)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(um_smem(&full[b])) : "memory");
        }
    } else {
        // ------------------------------------------------- MMA issue and drain
        // both warps take every iteration and every named barrier; after a
        // failed wait a warp only skips work (never the barrier)
        const bool issuer = (warp == MMAW);
        bool ok = true;
        int since = 0;
        for (int64_t li = 0; li < my_rounds; li++) {
            const int b = (int)(li % UM_NBUF);
            if (issuer && ok) {
                if (!um_wait(&full[b], (uint32_t)((li / UM_NBUF) & 1))) {
                    atomicExch(errword, 5);
                    ok = false;
                }
                um_fence_after();
                if (ok && lane == 0) {
                    const uint32_t a0 = um_smem(buf0 + (size_t)b * UM_BUFBYTES), b0 = a0 + UM_ABYTES;
#pragma unroll 1
                    for (int kb = 0; kb < UM_KB; kb++)
                        um_mma(tmem, um_desc(a0 + kb * UM_SA), um_desc(b0 + kb * UM_SB),
                               (since == 0 && kb == 0) ? 0u : 1u);
                    um_commit(&empty[b]);
                }
                __syncwarp();
            }
            since++;
            if (since == UM_DRAIN || li + 1 == my_rounds) {
                // both drain warps meet once the issuer has committed this round
                // (a parity wait must not start more than one phase early), then
                // wait for its MMAs (and all before)
                asm volatile("bar.sync 1, 64;" ::: "memory");
                if (ok && !um_wait(&empty[b], (uint32_t)((li / UM_NBUF) & 1))) {
                    atomicExch(errword, 5);
                    ok = false;
                }
                um_fence_after();
                if (ok) {
                    float v[UM_N];
                    const int q = warp - MMAW;  // TMEM lanes 32 q .. 32 q + 31
#pragma unroll
                    for (int c = 0; c < UM_N; c += 8) um_ld8(tmem + ((uint32_t)(32 * q) << 16) + c, v + c);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    double* dr = drain + (32 * q + lane) * UM_N;
#pragma unroll
                    for (int c = 0; c < UM_N; c++) dr[c] += (double)v[c];
                }
                um_fence_before();
                asm volatile("bar.sync 1, 64;" ::: "memory");  // the next MMA may overwrite
                um_fence_after();
                since = 0;
            }
        }
        if (!ok && issuer && lane == 0 && my_rounds > 0) {
            // wait (bounded) for whatever was committed before freeing TMEM
            for (int bb = 0; bb < UM_NBUF; bb++) um_wait(&empty[bb], 0u);
        }
    }
    um_fence_before();
    __syncthreads();
    um_fence_after();
    if (warp == MMAW)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UM_TMEM_COLS)
                     : "memory");
    // combine the hi/lo quadrants: part[cta][d][c], c < NCP
    double* dst = part + (size_t)blockIdx.x * 32 * NCP;
    for (int i = tid; i < 32 * NCP; i += nthr) {
        const int d = i / NCP, c = i - d * NCP;
        double v = 0.0;
        if (c == 0) v = drain[d * UM_N] + drain[(d + 32) * UM_N];
        else if (c <= NG && c <= 16)
            v = drain[d * UM_N + c] + drain[d * UM_N + c + 16] + drain[(d + 32) * UM_N + c] +
                drain[(d + 32) * UM_N + c + 16];
        dst[i] = v;
    }
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
        k_sfp_reduce<double><<<nmom, 256, 0, s->stream>>>((double*)s->part, nb, nmom, s->mom);
        SFP_CUDA(s, cudaGetLastError());
        s->launches += 2;
        return GX_OK;
    }
    const float inv = (float)(1.0 / s->maxr);
    if (precision == GX_PREC_MIXED_TC05) {
        if (D != 32 || s->NC > 17)
            return s->err = "the tcgen05 path takes at most 32 Chebyshev terms and maxm <= 8", GX_ERR_RANGE;
        // tcgen05: one CTA per SM (at most), FP64 partial per CTA
        const int64_t rounds = (n + UM_T - 1) / UM_T;
        const int grid = (int)std::min<int64_t>(rounds, s->nsm);
        const size_t sm = (size_t)UM_NBUF * UM_BUFBYTES + sizeof(double) * 64 * UM_N;
        SFP_CUDA(s, cudaFuncSetAttribute(k_sfp_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_sfp_umma<<<grid, UM_THREADS + 64, sm, s->stream>>>(s->xy, s->xy + s->cap, n, inv, s->b.maxm, s->upart, NCP,
                                                  s->errword);
        SFP_CUDA(s, cudaGetLastError());
        k_sfp_reduce<double><<<32 * NCP, 256, 0, s->stream>>>(s->upart, grid, 32 * NCP, s->mom);
        SFP_CUDA(s, cudaGetLastError());
        s->launches += 2;
        return GX_OK;
    }
    const int64_t nw = (n + SFP_CHUNK - 1) / SFP_CHUNK;
    const unsigned grid = (unsigned)((nw * 32 + 255) / 256);
    // feature columns 1 .. NC - 1 in blocks of 8
    const int NB = (s->NC - 1 + 7) / 8;
    if (NB > 3) return s->err = "more than 11 harmonics on the tensor-core path", GX_ERR_RANGE;
    const size_t sm = sizeof(float) * 8 * 32 * ((size_t)(D + 8) + SFP_GSTR);
    auto k = (D == 32) ? ((NB <= 1) ? k_sfp_moments<2, 1> : (NB == 2) ? k_sfp_moments<2, 2> : k_sfp_moments<2, 3>)
                       : ((NB <= 1) ? k_sfp_moments<4, 1> : (NB == 2) ? k_sfp_moments<4, 2> : k_sfp_moments<4, 3>);
    SFP_CUDA(s, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k<<<grid, 256, sm, s->stream>>>(s->xy, s->xy + s->cap, n, inv, s->b.maxm, NCP, s->part);
    SFP_CUDA(s, cudaGetLastError());
    k_sfp_reduce<float><<<nmom, 256, 0, s->stream>>>(s->part, nw, nmom, s->mom);
    SFP_CUDA(s, cudaGetLastError());
    s->launches += 2;
    return GX_OK;
}

// sfpsum + scaled: coeff[n * (2 maxm + 1) + m + maxm] (cosine +m, sine -m)
extern "C" int gx_sfp_sum(GxSfp* s, int precision, double pmass, double* coeff) {
    if (!s || !coeff) return GX_ERR_ARG;
    if (precision != GX_PREC_MIXED && precision != GX_PREC_FP64 && precision != GX_PREC_MIXED_TC05)
        return GX_ERR_ARG;
    cudaSetDevice(s->dev);
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
    if (s->n > 0)
        SFP_CUDA(s, cudaMemcpyAsync(mom.data(), s->mom, sizeof(double) * D * NCP, cudaMemcpyDeviceToHost, s->stream));
    SFP_CUDA(s, cudaStreamSynchronize(s->stream));
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

// sfpacc for the loaded particles from scaled coefficients; acc [n][2], pot [n]
extern "C" int gx_sfp_acc(GxSfp* s, const double* coeff, float* acc, float* pot) {
    if (!s || !coeff || (!acc && s->n > 0)) return GX_ERR_ARG;
    cudaSetDevice(s->dev);
    const int D = s->D, maxm = s->b.maxm, ngx = 2 * maxm + 1;
    std::vector<double> qs((size_t)2 * (maxm + 1) * D, 0.0);
    for (int f = 0; f < s->nfun; f++) {
        const int m = s->msel[f], n = s->nsel[f];
        const double* a = s->acheb.data() + (size_t)f * D;
        const int l = n * ngx + maxm;
        const double cr = coeff[l + m], ci = (m > 0) ? coeff[l - m] : 0.0;
        for (int d = 0; d < D; d++) {
            qs[((size_t)0 * (maxm + 1) + m) * D + d] += cr * a[d];
            qs[((size_t)1 * (maxm + 1) + m) * D + d] += ci * a[d];
        }
    }
    if (!s->qc) SFP_CUDA(s, cudaMalloc((void**)&s->qc, sizeof(double) * 2 * 12 * 64));
    SFP_CUDA(s, cudaMemcpyAsync(s->qc, qs.data(), sizeof(double) * qs.size(), cudaMemcpyHostToDevice, s->stream));
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

extern "C" int gx_sfp_last_ms(const GxSfp* s, float* ms, int64_t* launches) {
    if (!s || !ms) return GX_ERR_ARG;
    *ms = s->last_ms;
    if (launches) *launches = s->launches;
    return GX_OK;
}
