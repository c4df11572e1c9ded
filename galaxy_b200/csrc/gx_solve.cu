// gx_solve.cu -- field solve of the mixed-precision path (findf).
//
//   k_fwd_ring (3D)   p3manl.f:62-109: the azimuthal and vertical DFTs of
//                     one ring per CTA, the ring's planes and the tables
//                     bulk-copied into shared memory (grids whose ring data
//                     fit, unless GX_FLAG_ROWBLOCK_TRANSFORMS);
//   k_fwd_az, k_fwd_z (3D) / k_fwd2 (2D)   p3manl.f:62-109 / p2manl.f:32-45:
//                     the azimuthal real DFT of every ring-plane row
//                     restricted to the active harmonics (the m = 0 term
//                     summed in FP64), then (3D) per ring the zero-padded
//                     length-2 ngz vertical DFT.  Both are small GEMMs
//                     against twiddle tables staged in shared memory, with
//                     the K sum split over lanes; only the active harmonics
//                     are formed.
//   k_conv            p3conv.f:137-230 / p2conv.f:114-181 (2D, and 3D grids
//                     that gx_conv.cu's bulk-copy kernel does not take): for every
//                     (harmonic, vertical wavenumber) the dense radial
//                     contraction with the FP32 Green table of each field
//                     type, the Green matrix streamed from HBM once per step.
//   synthesis         p3fsyn.f / p2fsyn.f fused with polcat: gx_synth.cu.
// FFTPACK conventions (SRC/utils/sfftpack): forward a_m = sum x cos,
// b_m = -sum x sin; backward x_j = a_0 + (-1)^j a_N + 2 sum (a cos - b sin).
#include <algorithm>

#include "gx_bulk.cuh"
#include "gx_common.cuh"


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

// C[M][N] = A[M][K] * B[K][N] in shared memory, 4x4 register tiles with the
// K sum split over KS adjacent lanes (lane ks takes k = ks, ks + KS, ...) and
// reduced by shuffles; epi(r0, c0, acc) runs on the lane with ks == 0.  The
// tile loop has the same trip count on every thread (the shuffles need the
// whole warp); blockDim.x must be a multiple of 32.
template <int KS, class Epi>
__device__ __forceinline__ void sgemm44_sk(int M, int N, int K, const float* A, int lda,
                                           const float* B, int ldb, Epi epi) {
    const int tilesN = (N + 3) >> 2, tilesM = (M + 3) >> 2, nt = tilesM * tilesN;
    const int per = blockDim.x / KS, ks = threadIdx.x % KS;
    for (int t0 = 0; t0 < nt; t0 += per) {
        const int t = t0 + threadIdx.x / KS;
        const bool act = t < nt;
        const int tm = act ? t / tilesN : 0, tn = act ? t - tm * tilesN : 0;
        const int r0 = tm * 4, c0 = tn * 4;
        float acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
        if (act) {
            const float* ap = A + (size_t)r0 * lda;
            const float* bp = B + c0;
#pragma unroll 4
            for (int k = ks; k < K; k += KS) {
                const float4 b = *reinterpret_cast<const float4*>(bp + (size_t)k * ldb);
                const float a0 = ap[k], a1 = ap[lda + k], a2 = ap[2 * lda + k], a3 = ap[3 * lda + k];
                acc[0][0] += a0 * b.x; acc[0][1] += a0 * b.y; acc[0][2] += a0 * b.z; acc[0][3] += a0 * b.w;
                acc[1][0] += a1 * b.x; acc[1][1] += a1 * b.y; acc[1][2] += a1 * b.z; acc[1][3] += a1 * b.w;
                acc[2][0] += a2 * b.x; acc[2][1] += a2 * b.y; acc[2][2] += a2 * b.z; acc[2][3] += a2 * b.w;
                acc[3][0] += a3 * b.x; acc[3][1] += a3 * b.y; acc[3][2] += a3 * b.z; acc[3][3] += a3 * b.w;
            }
        }
#pragma unroll
        for (int o = 1; o < KS; o <<= 1)
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] += __shfl_xor_sync(0xffffffffu, acc[i][j], o);
        if (act && ks == 0) epi(r0, c0, acc);
    }
}

// sgemm44_sk with A stored transposed: A(r, k) = At[k * ldat + r] (ldat % 4
// == 0, rows up to ru4(M) addressable), so each k takes one float4 of A.
// The products and their order are those of sgemm44_sk on the same matrix.
template <int KS, class Epi>
__device__ __forceinline__ void sgemm44_skT(int M, int N, int K, const float* At, int ldat,
                                            const float* B, int ldb, Epi epi) {
    const int tilesN = (N + 3) >> 2, tilesM = (M + 3) >> 2, nt = tilesM * tilesN;
    const int per = blockDim.x / KS, ks = threadIdx.x % KS;
    for (int t0 = 0; t0 < nt; t0 += per) {
        const int t = t0 + threadIdx.x / KS;
        const bool act = t < nt;
        const int tm = act ? t / tilesN : 0, tn = act ? t - tm * tilesN : 0;
        const int r0 = tm * 4, c0 = tn * 4;
        float acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
        if (act) {
            const float* ap = At + r0;
            const float* bp = B + c0;
#pragma unroll 4
            for (int k = ks; k < K; k += KS) {
                const float4 b = *reinterpret_cast<const float4*>(bp + (size_t)k * ldb);
                const float4 a = *reinterpret_cast<const float4*>(ap + (size_t)k * ldat);
                acc[0][0] += a.x * b.x; acc[0][1] += a.x * b.y; acc[0][2] += a.x * b.z; acc[0][3] += a.x * b.w;
                acc[1][0] += a.y * b.x; acc[1][1] += a.y * b.y; acc[1][2] += a.y * b.z; acc[1][3] += a.y * b.w;
                acc[2][0] += a.z * b.x; acc[2][1] += a.z * b.y; acc[2][2] += a.z * b.z; acc[2][3] += a.z * b.w;
                acc[3][0] += a.w * b.x; acc[3][1] += a.w * b.y; acc[3][2] += a.w * b.z; acc[3][3] += a.w * b.w;
            }
        }
#pragma unroll
        for (int o = 1; o < KS; o <<= 1)
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] += __shfl_xor_sync(0xffffffffu, acc[i][j], o);
        if (act && ks == 0) epi(r0, c0, acc);
    }
}

// forward twiddle tables, built once per context:
//   Taz[j][2a] = cos(2 pi m_a j / na), Taz[j][2a+1] = -sin(...)   [na][ncp]
//   Tz[2k][z] = cos(pi k z / ngz), Tz[2k+1][z] = -sin(...)       [ru4(2 nkz)][ngz]
//   TzT[z][r] = Tz[r][z]                                         [ngz][ru4(2 nkz)]
//   Tf[j][c] = Taz[j][c + cb], c < 2 nact - cb, else 0           [na][ncpf]
__global__ void k_fwdtab(DevGeo g, int nact, int ncp, float* __restrict__ Taz, float* __restrict__ Tz,
                         float* __restrict__ TzT, float* __restrict__ Tf, int cb, int ncpf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int na = g.na, ngz = g.ngz, nkz = g.nkz;
    if (i < na * ncp) {
        const int j = i / ncp, c = i - j * ncp;
        float v = 0.f;
        if (c < 2 * nact) {
            const int m = g.act[c >> 1];
            const int idx = (int)(((int64_t)m * j) % na);
            float sn, co;
            sincospif(2.0f * (float)idx / (float)na, &sn, &co);
            v = (c & 1) ? -sn : co;
        }
        Taz[i] = v;
        if (Tf && c >= cb && c - cb < ncpf) Tf[(size_t)j * ncpf + (c - cb)] = v;
    }
    if (g.ndim == 3 && i < ru4(2 * nkz) * ngz) {
        const int r = i / ngz, z = i - r * ngz, k = r >> 1;
        float v = 0.f;
        if (k < nkz) {
            const int idx = (int)(((int64_t)k * z) % (2 * ngz));
            float sn, co;
            sincospif((float)idx / (float)ngz, &sn, &co);
            v = (r & 1) ? -sn : co;
        }
        Tz[i] = v;
        TzT[(size_t)z * ru4(2 * nkz) + r] = v;
    }
}

// 3D forward, azimuthal part (p3manl.f:62-83): the active-harmonic DFT of
// FWD_RB ring-plane rows per CTA, C1[row][2a, 2a+1] = (a_m, b_m); the m = 0
// column summed in FP64.  Rows of rings without mass are skipped (the
// vertical part zeroes their spectrum).
#define FWD_RB 32
__global__ void __launch_bounds__(288) k_fwd_az(DevGeo g, int ncp, const int32_t* __restrict__ jrk,
                                                const int32_t* __restrict__ zr,
                                                const float* __restrict__ mass,
                                                const float* __restrict__ Taz,
                                                float* __restrict__ C1) {
    extern __shared__ __align__(16) float sm[];
    const int na = g.na, ngz = g.ngz, nr = g.nr;
    const int row0 = blockIdx.x * FWD_RB;
    const int rlo = (max(jrk[0], 1) - 1) * ngz, rhi = min(jrk[1], nr) * ngz;  // active rows [rlo, rhi)
    if (row0 + FWD_RB <= rlo || row0 >= rhi) return;
    const int nrows = min(FWD_RB, g.nrow - row0);
    if (zr) {
        // only blocks with a row in the planes the vertical part sums (the
        // planes holding mass, the first rounded down to a multiple of 4)
        const int zs = zr[0] & ~3, ze = zr[1];
        int in = 0;
        if ((int)threadIdx.x < nrows) {
            const int iz = (row0 + (int)threadIdx.x) % ngz;
            in = iz >= zs && iz <= ze;
        }
        if (!__syncthreads_or(in)) return;
    }
    const int ldx = na + 1;
    float* X = sm;                 // [FWD_RB][na + 1]
    float* T = X + FWD_RB * ldx;   // [na][ncp]
    // several loads in flight per thread: the prologue is latency-bound
    for (int b = threadIdx.x; b < FWD_RB * na; b += 4 * blockDim.x) {
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = b + u * blockDim.x, r = i / na;
            v[u] = (i < FWD_RB * na && r < nrows) ? __ldg(mass + (size_t)row0 * na + i) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = b + u * blockDim.x;
            if (i < FWD_RB * na) {
                const int r = i / na, j = i - r * na;
                X[r * ldx + j] = v[u];
            }
        }
    }
    {
        const int n4 = na * ncp / 4;
        const float4* src = reinterpret_cast<const float4*>(Taz);
        float4* dst = reinterpret_cast<float4*>(T);
        for (int b = threadIdx.x; b < n4; b += 8 * blockDim.x) {
            float4 v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int i = b + u * blockDim.x;
                if (i < n4) v[u] = __ldg(src + i);
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int i = b + u * blockDim.x;
                if (i < n4) dst[i] = v[u];
            }
        }
    }
    __syncthreads();
    sgemm44_sk<4>(FWD_RB, ncp, na, X, ldx, T, ncp, [&](int r0, int c0, float (&acc)[4][4]) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (r0 + i >= nrows) continue;
            *reinterpret_cast<float4*>(C1 + (size_t)(row0 + r0 + i) * ncp + c0) =
                make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
        }
    });
    if (g.act[0] == 0) {
        __syncthreads();  // column 0 of the GEMM is written before the FP64 sum replaces it
        // 8 lanes per row, FP64 partial sums over na / 8 points each
        const int r = threadIdx.x >> 3, q = threadIdx.x & 7;
        double s = 0.0;
        if (r < FWD_RB)
            for (int j = q; j < na; j += 8) s += (double)X[r * ldx + j];
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (r < nrows && q == 0) C1[(size_t)(row0 + r) * ncp] = (float)s;
    }
}

// 3D forward, vertical part (p3manl.f:84-109): per ring, the zero-padded
// length-2 ngz DFT of the azimuthal spectra, FWD_KR output rows (2 per kz)
// per CTA.  S[(a nkz + k) nr + ir] = (A_c, B_c, A_s, B_s).
#define FWD_KR 32
__global__ void __launch_bounds__(288) k_fwd_z(DevGeo g, int nact, int ncp,
                                               const int32_t* __restrict__ jrk,
                                               const int32_t* __restrict__ zr,
                                               const float* __restrict__ C1,
                                               const float* __restrict__ Tz, float4* __restrict__ S) {
    extern __shared__ __align__(16) float sm[];
    const int ngz = g.ngz, nkz = g.nkz, nr = g.nr;
    // the planes summed: all, or those holding mass with the first rounded
    // down to a multiple of 4, so that every lane of the K split below sums
    // the same planes in the same order as over the whole grid (the others
    // add exact zeros): the spectrum is bitwise the whole-grid one
    const int zs = zr ? (zr[0] & ~3) : 0;
    const int nzs = zr ? max(zr[1] - zs + 1, 0) : ngz;
    const int ir = blockIdx.x, kr0 = blockIdx.y * FWD_KR;   // first output row (2 kz0)
    const int nrow_out = min(FWD_KR, 2 * nkz - kr0);
    if (ir < jrk[0] - 1 || ir > min(jrk[1], nr) - 1) {
        // only the rings that hold mass are transformed (p3fndf.f:44-57); the
        // others get a zero spectrum so that the sum over ranks stays exact
        for (int i = threadIdx.x; i < nact * (nrow_out / 2); i += blockDim.x) {
            const int a = i / (nrow_out / 2), k = kr0 / 2 + (i - a * (nrow_out / 2));
            S[((size_t)a * nkz + k) * nr + ir] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        return;
    }
    float* B = sm;                      // [nzs][ncp]
    float* Tk = B + ngz * ncp;          // [FWD_KR][nzs]
    // several loads in flight per thread: the prologue is latency-bound
    {
        const float4* src = reinterpret_cast<const float4*>(C1 + ((size_t)ir * ngz + zs) * ncp);
        float4* dst = reinterpret_cast<float4*>(B);
        const int n4 = nzs * ncp / 4;
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
    for (int b = threadIdx.x; b < FWD_KR * nzs; b += 4 * blockDim.x) {
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = b + u * blockDim.x, r = i / max(nzs, 1), z = i - r * nzs;
            v[u] = (i < nrow_out * nzs) ? __ldg(Tz + (size_t)(kr0 + r) * ngz + zs + z) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = b + u * blockDim.x;
            if (i < FWD_KR * nzs) Tk[i] = v[u];
        }
    }
    __syncthreads();
    sgemm44_sk<4>(nrow_out, ncp, nzs, Tk, nzs, B, ncp, [&](int r0, int c0, float (&acc)[4][4]) {
        // rows r0 = 2k, 2k+1, 2k+2, 2k+3 (relative to kr0); cols c0 = 2a .. 2a+3
#pragma unroll
        for (int dk = 0; dk < 2; dk++) {
            const int k = (kr0 + r0) / 2 + dk;
            if (k >= nkz || r0 + 2 * dk >= nrow_out) continue;
#pragma unroll
            for (int da = 0; da < 2; da++) {
                const int a = (c0 >> 1) + da;
                if (a >= nact) continue;
                S[((size_t)a * nkz + k) * nr + ir] =
                    make_float4(acc[2 * dk][2 * da], acc[2 * dk + 1][2 * da], acc[2 * dk][2 * da + 1],
                                acc[2 * dk + 1][2 * da + 1]);
            }
        }
    });
}

// 3D forward transform of one ring per CTA (p3manl.f:62-109): the
// azimuthal and vertical DFTs of k_fwd_az and k_fwd_z in one launch, with
// the ring's planes, the twiddle tables and the intermediate spectra in
// shared memory.  One thread issues bulk copies of the azimuthal table and
// of the ring's plane rows (only the planes summed: those holding mass, the
// first rounded down to a multiple of 4) on one mbarrier; the azimuthal DFT
// of up to FWR_XR rows at a time goes into C1 [plane][ncpf] in shared
// memory; then the block of the transposed vertical table for those planes
// replaces the first two and the vertical DFT writes S.
//
// Both DFTs are FP32 GEMMs on 4 x 4 register tiles whose operands are
// float4 loads from shared memory.  A warp takes 4 row groups x 8 column
// quads, so that each operand load is 4 or 8 distinct 16-byte words (one
// shared-memory wavefront).  Thread rows are interleaved (rows tm + RG i) so
// that the 4 row groups of a warp fall on different banks.  The azimuthal
// sum over spokes is split over warps in contiguous ranges and the partial
// tiles are added in warp order; the vertical sum runs over the planes in
// order, so a sum over the planes holding mass equals the sum over all
// planes bit for bit (the others add exact zeros).  The m = 0 column is not
// in the GEMMs: its azimuthal sum is formed in FP64 (8 lanes per row), its
// vertical DFT by 4 lanes per kz (planes by residue mod 4), and its sine
// part is zero.
#define FWR_THREADS 512
#define FWR_WARPS (FWR_THREADS / 32)
#define FWR_XR 48
__global__ void __launch_bounds__(FWR_THREADS) k_fwd_ring(DevGeo g, int nact, int ncpf, int cb,
                                                          const int32_t* __restrict__ jrk,
                                                          const int32_t* __restrict__ zr,
                                                          const float* __restrict__ mass,
                                                          const float* __restrict__ Tf,
                                                          const float* __restrict__ TzT, float4* __restrict__ S,
                                                          int32_t* __restrict__ errword) {
    extern __shared__ __align__(128) float sm[];
    __shared__ uint64_t bar;
    const int na = g.na, ngz = g.ngz, nkz = g.nkz, nr = g.nr;
    const int ir = blockIdx.x;
    if (ir < jrk[0] - 1 || ir > min(jrk[1], nr) - 1) {
        // a ring without mass: zero spectrum (p3fndf.f:44-57)
        for (int i = threadIdx.x; i < nact * nkz; i += blockDim.x)
            S[(size_t)i * nr + ir] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const int zs = zr ? (zr[0] & ~3) : 0;
    const int nzs = zr ? max(zr[1] - zs + 1, 0) : ngz;
    const int ldx = na + 4, ldt = ru4(2 * nkz), tnN = ncpf >> 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tml = lane >> 3, tnl = lane & 7;
    float* C1 = sm;                            // [ru4(ngz)][ncpf]   harmonics m > 0 (or all)
    float* C0 = C1 + (size_t)ru4(ngz) * ncpf;  // [ru4(ngz)]         m = 0 (FP64 sums)
    float* P = C0 + ru4(ngz);                  // [FWR_WARPS][16][32] partial tiles
    float* T = P + FWR_WARPS * 16 * 32;        // [na][ncpf]         (azimuthal part)
    float* X = T + (size_t)na * ncpf;          // [FWR_XR][na + 4]   (azimuthal part)
    float* Tt = T;                             // [nzs][ldt]         (vertical part)
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    uint32_t ph = 0;
    for (int c0 = 0; c0 < nzs; c0 += FWR_XR) {
        const int nx = min(FWR_XR, nzs - c0);
        if (threadIdx.x == 0) {
            const uint32_t rowb = (uint32_t)na * 4u, tabb = c0 == 0 ? (uint32_t)(na * ncpf) * 4u : 0u;
            mbar_expect_tx(&bar, tabb + (uint32_t)nx * rowb);
            if (tabb) bulk_g2s(T, Tf, tabb, &bar);
            const float* src = mass + ((size_t)ir * ngz + zs + c0) * na;
            for (int r = 0; r < nx; r++) bulk_g2s(X + (size_t)r * ldx, src + (size_t)r * na, rowb, &bar);
        }
        if (!__syncthreads_and(mbar_wait(&bar, ph))) {
            if (threadIdx.x == 0) {
                atomicExch(errword, 5);
                mbar_wait(&bar, ph);  // the copies in flight land before the CTA leaves
            }
            return;
        }
        ph ^= 1;
        if (cb) {
            // m = 0: FP64 sum of each row, 8 lanes per row, na / 8 points each
            const int r = threadIdx.x >> 3, q = threadIdx.x & 7;
            double s = 0.0;
            if (r < nx)
                for (int j = q; j < na; j += 8) s += (double)X[r * ldx + j];
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (r < nx && q == 0) C0[c0 + r] = (float)s;
        }
        // C1[c0 + r][c] = sum_j X[r][j] Tf[j][c]; thread rows tm + RG i
        // the split of the spoke sum depends on the columns alone (not on the
        // chunk's rows), so that every row's sum is formed the same way
        // whichever planes are transformed
        const int RG = (nx + 3) >> 2;
        const int WTN = (tnN + 7) >> 3, WT = ((RG + 3) >> 2) * WTN;
        const int KG = max(1, FWR_WARPS / (((FWR_XR / 4 + 3) >> 2) * WTN));
        const int kc = (na + 4 * KG - 1) / (4 * KG) * 4;
        for (int wi = warp; wi < WT * KG; wi += FWR_WARPS) {
            const int wt = wi % WT, kg = wi / WT;
            const int tm = (wt / WTN) * 4 + tml, tn = (wt % WTN) * 8 + tnl;
            const int tmc = min(tm, RG - 1), tnc = min(tn, tnN - 1);
            float acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[i][c] = 0.f;
            const int j1 = min(na, (kg + 1) * kc);
            const float* xa = X + (size_t)tmc * ldx;
            const float* tb = T + 4 * tnc;
#pragma unroll 1
            for (int j = kg * kc; j < j1; j += 4) {
                float4 a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; i++) a[i] = *reinterpret_cast<const float4*>(xa + (size_t)i * RG * ldx + j);
#pragma unroll
                for (int q = 0; q < 4; q++) b[q] = *reinterpret_cast<const float4*>(tb + (size_t)(j + q) * ncpf);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float av[4] = {a[i].x, a[i].y, a[i].z, a[i].w};
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        acc[i][0] += av[q] * b[q].x;
                        acc[i][1] += av[q] * b[q].y;
                        acc[i][2] += av[q] * b[q].z;
                        acc[i][3] += av[q] * b[q].w;
                    }
                }
            }
            if (KG == 1) {
                if (tm < RG && tn < tnN) {
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const int r = tm + RG * i;
                        if (r < nx)
                            *reinterpret_cast<float4*>(C1 + (size_t)(c0 + r) * ncpf + 4 * tn) =
                                make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
                    }
                }
            } else {
#pragma unroll
                for (int e = 0; e < 16; e++) P[(warp * 16 + e) * 32 + lane] = acc[e >> 2][e & 3];
            }
        }
        if (KG > 1) {
            __syncthreads();
            // add the KG partial tiles of each warp tile in warp order
            for (int idx = threadIdx.x; idx < WT * 16 * 32; idx += blockDim.x) {
                const int ln = idx & 31, e = (idx >> 5) & 15, wt = idx >> 9;
                const int tm = (wt / WTN) * 4 + (ln >> 3), tn = (wt % WTN) * 8 + (ln & 7);
                const int r = tm + RG * (e >> 2);
                if (tm >= RG || tn >= tnN || r >= nx) continue;
                float v = P[((0 * WT + wt) * 16 + e) * 32 + ln];
                for (int kg = 1; kg < KG; kg++) v += P[((kg * WT + wt) * 16 + e) * 32 + ln];
                C1[(size_t)(c0 + r) * ncpf + 4 * tn + (e & 3)] = v;
            }
        }
        __syncthreads();  // X, T and P are free again
    }
    if (nzs > 0) {
        if (threadIdx.x == 0) {
            const uint32_t b = (uint32_t)nzs * (uint32_t)ldt * 4u;
            mbar_expect_tx(&bar, b);
            bulk_g2s(Tt, TzT + (size_t)zs * ldt, b, &bar);
        }
        if (!__syncthreads_and(mbar_wait(&bar, ph))) {
            if (threadIdx.x == 0) {
                atomicExch(errword, 5);
                mbar_wait(&bar, ph);
            }
            return;
        }
    }
    // S[a][k][ir] from rows 2k, 2k+1 (cos, -sin kz) x columns 2a, 2a+1 (a_m, b_m)
    {
        const int tmN = ldt >> 2, WTN = (tnN + 7) >> 3, WT = ((tmN + 3) >> 2) * WTN;
        for (int wt = warp; wt < WT; wt += FWR_WARPS) {
            const int tm = (wt / WTN) * 4 + tml, tn = (wt % WTN) * 8 + tnl;
            const int tmc = min(tm, tmN - 1), tnc = min(tn, tnN - 1);
            float acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[i][c] = 0.f;
            const float* ta = Tt + 4 * tmc;
            const float* cbp = C1 + 4 * tnc;
#pragma unroll 4
            for (int z = 0; z < nzs; z++) {
                const float4 a = *reinterpret_cast<const float4*>(ta + (size_t)z * ldt);
                const float4 b = *reinterpret_cast<const float4*>(cbp + (size_t)z * ncpf);
                const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    acc[i][0] += av[i] * b.x;
                    acc[i][1] += av[i] * b.y;
                    acc[i][2] += av[i] * b.z;
                    acc[i][3] += av[i] * b.w;
                }
            }
            if (tm < tmN && tn < tnN) {
#pragma unroll
                for (int dk = 0; dk < 2; dk++) {
                    const int k = 2 * tm + dk;
                    if (k >= nkz) continue;
#pragma unroll
                    for (int da = 0; da < 2; da++) {
                        const int a = (4 * tn + cb) / 2 + da;
                        if (a >= nact) continue;
                        S[((size_t)a * nkz + k) * nr + ir] =
                            make_float4(acc[2 * dk][2 * da], acc[2 * dk + 1][2 * da], acc[2 * dk][2 * da + 1],
                                        acc[2 * dk + 1][2 * da + 1]);
                    }
                }
            }
        }
        if (cb) {
            // m = 0: 4 lanes per kz, lane q sums the planes z = zs + q (mod 4)
            const int q = threadIdx.x & 3;
            for (int kb = 0; kb < nkz; kb += FWR_THREADS / 4) {
                const int k = kb + (threadIdx.x >> 2);
                float ac = 0.f, bc = 0.f;
                if (k < nkz)
                    for (int z = q; z < nzs; z += 4) {
                        const float2 t = *reinterpret_cast<const float2*>(Tt + (size_t)z * ldt + 2 * k);
                        ac += t.x * C0[z];
                        bc += t.y * C0[z];
                    }
#pragma unroll
                for (int o = 1; o < 4; o <<= 1) {
                    ac += __shfl_xor_sync(0xffffffffu, ac, o);
                    bc += __shfl_xor_sync(0xffffffffu, bc, o);
                }
                if (k < nkz && q == 0) S[(size_t)k * nr + ir] = make_float4(ac, bc, 0.f, 0.f);
            }
        }
    }
}

// the column layout of k_fwd_ring's azimuthal table: with m = 0 active its
// two columns are left out (cb = 2)
static inline int fwd_ring_cb(const Spec& sp) { return (sp.nact > 0 && sp.m[0] == 0) ? 2 : 0; }
static inline int fwd_ring_ncpf(const Spec& sp) { return ru4(2 * sp.nact - fwd_ring_cb(sp)); }

// shared memory of k_fwd_ring, bytes; 0 when the geometry does not fit
static size_t fwd_ring_smem(const DevGeo& g, const Spec& sp) {
    if (g.na % 4) return 0;
    const int ncpf = fwd_ring_ncpf(sp);
    if (ncpf == 0) return 0;
    const size_t az = (size_t)g.na * ncpf + (size_t)FWR_XR * (g.na + 4);
    const size_t vz = (size_t)g.ngz * ru4(2 * g.nkz);
    const size_t b = sizeof(float) * ((size_t)ru4(g.ngz) * (ncpf + 1) + FWR_WARPS * 16 * 32 + std::max(az, vz));
    return b <= 200 * 1024 ? b : 0;
}

// 2D forward (p2manl.f:32-45), one ring per CTA of F2_THREADS: thread
// (a, q) sums harmonic a (of a block of F2_H) over the spokes j = q (mod
// F2_Q) in spoke order, the twiddles read through L1 (the context's table,
// k_fwdtab); the F2_Q partials are added in q order.  The m = 0 column is
// summed in FP64 over a warp.  S[a nr + ir] = (a_m, 0, b_m, 0).
#define F2_H 16
#define F2_Q 16
#define F2_THREADS (F2_H * F2_Q)
__global__ void __launch_bounds__(F2_THREADS) k_fwd2(DevGeo g, int nact, int ncp, const float* __restrict__ mass,
                                                     const float* __restrict__ Taz, float4* __restrict__ S) {
    extern __shared__ __align__(16) float sm[];
    __shared__ float2 part[F2_Q][F2_H];
    const int na = g.na, nr = g.nr, ir = blockIdx.x;
    float* x = sm;  // [na]
    for (int j = threadIdx.x; j < na; j += blockDim.x) x[j] = __ldg(mass + (size_t)ir * na + j);
    __syncthreads();
    const int h = threadIdx.x % F2_H, q = threadIdx.x / F2_H;
    for (int a0 = 0; a0 < nact; a0 += F2_H) {
        const int a = a0 + h;
        float sc = 0.f, ss = 0.f;
        if (a < nact) {
#pragma unroll 4
            for (int j = q; j < na; j += F2_Q) {
                const float xv = x[j];
                const float2 t = __ldg(reinterpret_cast<const float2*>(Taz + (size_t)j * ncp + 2 * a));
                sc += xv * t.x;
                ss += xv * t.y;
            }
        }
        part[q][h] = make_float2(sc, ss);
        __syncthreads();
        if (threadIdx.x < F2_H && a0 + (int)threadIdx.x < nact) {
            const int aa = a0 + threadIdx.x;
            float2 v = part[0][threadIdx.x];
            for (int k = 1; k < F2_Q; k++) {
                v.x += part[k][threadIdx.x].x;
                v.y += part[k][threadIdx.x].y;
            }
            if (!(aa == 0 && g.act[0] == 0)) S[(size_t)aa * nr + ir] = make_float4(v.x, 0.f, v.y, 0.f);
        }
        __syncthreads();
    }
    if (g.act[0] == 0 && threadIdx.x < 32) {
        double s0 = 0.0;
        for (int j = threadIdx.x; j < na; j += 32) s0 += (double)x[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        if (threadIdx.x == 0) S[ir] = make_float4((float)s0, 0.f, 0.f, 0.f);
    }
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
    const int a = blockIdx.x, k = blockIdx.y, m = g.act[a];
    float4* Sin = sh4;              // [nr]
    float4* part = sh4 + nr;        // [8][nr]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < nr; i += blockDim.x)
        Sin[i] = (i >= js && i <= ks) ? S[((size_t)a * nkz + k) * nr + i] : make_float4(0, 0, 0, 0);
    __syncthreads();
    {
        // one field type per CTA (blockIdx.z)
        const int t = blockIdx.z;
        if (!((tmask >> t) & 1)) return;
        bool valid = true;
        if (t == 1) valid = (m >= 1) && (m <= min(ng, mmax - 1) - 1);
        if (t == 2) valid = (g.ndim == 3) && (k >= 1) && (k <= ngz - 1);
        // ring-major output [t][ir][kz][a] (read as one block per ring by the synthesis)
        const size_t ost = (size_t)nkz * nact;
        float4* out = O + ((size_t)t * nr * nkz + k) * nact + a;
        if (!valid) {
            for (int i = threadIdx.x; i < nr; i += blockDim.x) out[i * ost] = make_float4(0, 0, 0, 0);
            return;
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
            out[i * ost] = s;
        }
        __syncthreads();
    }
}

bool gx_conv_bulk_ok(const DevGeo& g);
int gx_conv_bulk(GxCtx* c, int nact, int tmask);

// ---------------------------------------------------------------------------
// findf for the mixed path: mass -> field (and optional polar copy)
int gx_mixed_findf(GxCtx* c, int lpot, bool polcat_only_field, const int32_t* frk, const int32_t* zr) {
    const DevGeo& g = c->g;
    const int nact = c->spec.nact;
    if (nact == 0) return c->err = "no active harmonics", GX_ERR_ARG;
    const int ncp = ru4(2 * nact);
    int rc = GX_OK;
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
    if (g.ndim != 3) zr = nullptr;
    if (zr) {
        rc = gx_comm_reduce_planes(c, const_cast<int32_t*>(zr));
        if (rc) return rc;
    }
    if (g.ndim == 3) {
        const size_t ntaz = (size_t)g.na * ncp, ntz = (size_t)ru4(2 * g.nkz) * g.ngz;
        const int cb = fwd_ring_cb(c->spec), ncpf = fwd_ring_ncpf(c->spec);
        float* TzT = c->fwdtab ? c->fwdtab + ntaz + ntz : nullptr;
        float* Tf = c->fwdtab ? TzT + ntz : nullptr;
        if (!c->fwdtab) {
            // [Taz][Tz][TzT][Tf]
            GX_CUDA(c, cudaMalloc((void**)&c->fwdtab, sizeof(float) * (2 * ntaz + 2 * ntz)));
            TzT = c->fwdtab + ntaz + ntz;
            Tf = TzT + ntz;
            const size_t mx = std::max(ntaz, ntz);
            k_fwdtab<<<(unsigned)((mx + 255) / 256), 256, 0, c->stream>>>(g, nact, ncp, c->fwdtab,
                                                                          c->fwdtab + ntaz, TzT, Tf, cb, ncpf);
            GX_LAUNCHED(c);
        }
        const size_t smr = (c->cfg.flags & GX_FLAG_ROWBLOCK_TRANSFORMS) ? 0 : fwd_ring_smem(g, c->spec);
        if (smr) {
            GX_CUDA(c, cudaFuncSetAttribute(k_fwd_ring, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr));
            k_fwd_ring<<<g.nr, FWR_THREADS, smr, c->stream>>>(g, nact, ncpf, cb, c->jrk_d, zr, c->mass, Tf, TzT,
                                                              c->specS, c->errword);
            GX_LAUNCHED(c);
        } else {
            if (!c->fwdC1) GX_CUDA(c, cudaMalloc((void**)&c->fwdC1, sizeof(float) * (size_t)g.nrow * ncp));
            size_t sm = sizeof(float) * ((size_t)FWD_RB * (g.na + 1) + ntaz);
            GX_CUDA(c, cudaFuncSetAttribute(k_fwd_az, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            k_fwd_az<<<(g.nrow + FWD_RB - 1) / FWD_RB, 288, sm, c->stream>>>(g, ncp, c->jrk_d, zr, c->mass,
                                                                             c->fwdtab, c->fwdC1);
            GX_LAUNCHED(c);
            sm = sizeof(float) * ((size_t)g.ngz * ncp + (size_t)FWD_KR * g.ngz);
            GX_CUDA(c, cudaFuncSetAttribute(k_fwd_z, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            dim3 gz(g.nr, (2 * g.nkz + FWD_KR - 1) / FWD_KR);
            k_fwd_z<<<gz, 288, sm, c->stream>>>(g, nact, ncp, c->jrk_d, zr, c->fwdC1, c->fwdtab + ntaz,
                                                c->specS);
            GX_LAUNCHED(c);
        }
    } else {
        const size_t ntaz = (size_t)g.na * ncp;
        if (!c->fwdtab) {
            GX_CUDA(c, cudaMalloc((void**)&c->fwdtab, sizeof(float) * ntaz));
            k_fwdtab<<<(unsigned)((ntaz + 255) / 256), 256, 0, c->stream>>>(g, nact, ncp, c->fwdtab, nullptr,
                                                                            nullptr, nullptr, 0, 0);
            GX_LAUNCHED(c);
        }
        const size_t sm = sizeof(float) * (size_t)g.na;
        GX_CUDA(c, cudaFuncSetAttribute(k_fwd2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_fwd2<<<g.nr, F2_THREADS, sm, c->stream>>>(g, nact, ncp, c->mass, c->fwdtab, c->specS);
        GX_LAUNCHED(c);
    }
    rc = gx_comm_reduce_spectrum(c);
    if (rc) return rc;
    rc = gx_phase_mark(c, PH_CONV);
    if (rc) return rc;
    if (gx_conv_bulk_ok(g)) {
        rc = gx_conv_bulk(c, nact, tmask);
        if (rc) return rc;
        if (gx_plane_split(c)) {
            rc = gx_comm_reduce_conv(c);
            if (rc) return rc;
        }
    } else {
        size_t sm = sizeof(float4) * (size_t)g.nr * 9;
        dim3 grid(nact, g.nkz, 4);
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
    rc = gx_synthesis(c, tmask, polar, frk, zr);
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
    c->zr_valid = false;
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
    c->zones_ready = false;  // the zone arrays no longer describe the mass
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
