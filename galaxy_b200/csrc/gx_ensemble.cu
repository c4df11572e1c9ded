// gx_ensemble.cu -- an ensemble of independent 2D discs on one polar grid
// geometry, advanced together: one persistent cooperative launch per step,
// the launches of a batch of steps replayed from a CUDA graph.
//
// Each disc is the run the single-disc path makes of it (SRC/progs/galaxy.f
// time loop: findf, getacc + stpgrp, massgn): same cell keys and weights
// (gx_cell, weight.f:61-101), the same integer fixed-point deposit
// (massgn.f:68-89; 2^-20 of a particle mass, summed as integers, so the
// mass array is the same integers), the same forward / contraction /
// synthesis arithmetic (p2manl.f:32-45, p2conv.f:99-187, p2fsyn.f:34-56,
// polcat.f:22-41) with FP32 sums, the m = 0 forward sum in FP64.
//
// One step launch:
//   solve   CTA d (d < ndisc, strided) turns disc d's integer mass into its
//           (fx, fy) field grid: forward DFT of the active harmonics per
//           ring, radial contraction with the shared Green table (read from
//           L2), synthesis + polcat; it then zeroes the integer mass and
//           publishes the field with a ready flag (the launch's epoch).
//   push    every CTA takes chunks of particles (one disc each); it waits
//           (bounded) for the disc's ready flag, stages the disc's field in
//           shared memory, and for each particle interpolates (grdacc),
//           kicks and drifts (stpgrp), and deposits the new position into a
//           shared-memory copy of the disc's integer mass grid, flushed
//           with integer atomics (order-free, deterministic).  The particle
//           sums of the m = 2 amplitude go to a per-chunk slot.
//   close   the last CTA to finish sums the chunk slots of every disc in
//           chunk order (deterministic FP64) into the A2 series and
//           advances the step counter.
// The deposit-only launch (mode 0) makes the initial mass (masset) and A2 at
// step 0.
#include <algorithm>
#include <vector>

#include "gx_common.cuh"

#define ENS_FIXQ 1048576.0f  // 2^20
#define ENS_MAXACT 64
#define ENS_SPIN (1u << 24)
#define ENS_TUNE_REPS 3
// series entries past max_steps that the tuner's trial steps may write
#define ENS_SPARE (2 + ENS_TUNE_REPS + 1)

struct GxEnsemble {
    GxCtx* ctx = nullptr;  // geometry, Green table, active harmonics, stream
    std::string err;
    int ndisc = 0;
    int64_t ntot = 0;
    std::vector<int64_t> off;  // disc offsets [ndisc + 1]
    int max_steps = 0;
    int64_t steps_done = 0;
    float* P = nullptr;                  // SoA [4][ntot]: x, y, vx, vy
    float* pm = nullptr;                 // particle mass of each disc
    unsigned long long* mass64 = nullptr;  // [ndisc][mesh] fixed point
    float2* field = nullptr;             // [ndisc][mesh] (fx, fy)
    int32_t* chunks = nullptr;           // [nchunks][3]: disc, start, end
    int32_t* dchunk = nullptr;           // [ndisc + 1] first chunk of each disc
    double* a2part = nullptr;            // [nchunks][3]: sum cos 2phi, sum sin 2phi, count
    double* series = nullptr;            // [max_steps + ENS_SPARE][ndisc][2]
    uint32_t* ctl = nullptr;             // [0] entries recorded, [1] CTAs done, [2 + d] ready epoch
    float* tw = nullptr;                 // twiddle tables (ens_tables)
    // tuning and launch
    int threads = 512, chunk = 16384, nchunks = 0, grid = 0, nchunks_cap = 0;
    size_t smem = 0;
    cudaGraphExec_t gexec = nullptr;
    int gsteps = 0;
    bool use_graph = true;
    float last_ms = 0.f;
    int64_t launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

struct EnsArgs {
    DevGeo g;
    int ndisc, nact, nchunks, mode, tmask;
    float* P;
    int64_t ntot;
    const float* pm;
    unsigned long long* mass64;
    float2* field;
    const int32_t* chunks;
    const int32_t* dchunk;
    double* a2part;
    double* series;
    uint32_t* ctl;
    int32_t* errword;
    const float* green;
    const float* tw;
    int act_m[ENS_MAXACT];
};

// twiddle tables [4][nact][na]: forward cos, forward -sin (p2manl's FFTPACK
// signs), synthesis cosine and sine weights scaled by 1/na (p2fsyn.f)
__global__ void k_ens_tables(DevGeo g, int nact, const int* __restrict__ mlist, float* __restrict__ tw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int na = g.na;
    if (i >= nact * na) return;
    const int a = i / na, j = i - a * na, m = mlist[a];
    const int idx = (int)(((int64_t)m * j) % na);
    float sn, cs;
    sincospif(2.0f * (float)idx / (float)na, &sn, &cs);
    const float scale = 1.0f / (float)na;
    float tc, ts;
    if (m == 0) {
        tc = 1.f;
        ts = 0.f;
    } else if (m == g.mmax - 1) {
        tc = (j & 1) ? -1.f : 1.f;
        ts = 0.f;
    } else {
        tc = 2.f * cs;
        ts = -2.f * sn;
    }
    const size_t pl = (size_t)nact * na;
    tw[i] = cs;
    tw[pl + i] = -sn;
    tw[2 * pl + i] = tc * scale;
    tw[3 * pl + i] = ts * scale;
}

// ---------------------------------------------------------------------------
// field solve of disc d by the whole CTA (p2fndf.f:25-66 with polcat)
__device__ void ens_solve(const EnsArgs& A, int d, float* sm) {
    const DevGeo& g = A.g;
    const int nr = g.nr, na = g.na, nact = A.nact, mesh = g.mesh;
    const int ldm = na + 1;
    const size_t pl = (size_t)nact * na;
    float* M = sm;                                   // [nr][na + 1]
    float* Tw = M + (size_t)nr * ldm;                // [4][nact][na]
    // float2 arrays start on a 16-byte boundary
    float2* S = reinterpret_cast<float2*>(M + ((nr * ldm + 4 * pl + 3) & ~(size_t)3));  // [nact][nr]: (a_m, b_m)
    float2* O = S + (size_t)nact * nr;               // [2][nact][nr]: (W_c, W_s) of fr, ftheta
    unsigned long long* m64 = A.mass64 + (size_t)d * mesh;
    const float pmass = A.pm[d];
    // integer mass -> FP32 x pmass (scaled.f:89-92); the integers are cleared
    // for the deposit of this step
    for (int i = threadIdx.x; i < mesh; i += blockDim.x) {
        const long long v = (long long)m64[i];
        m64[i] = 0ull;
        M[(i / na) * ldm + (i % na)] = (float)((double)v * (1.0 / (double)ENS_FIXQ)) * pmass;
    }
    for (int i = threadIdx.x; i < 4 * (int)pl; i += blockDim.x) Tw[i] = A.tw[i];
    __syncthreads();
    // forward transform per ring (p2manl.f:32-45): a_m = sum x cos, b_m = -sum x sin
    for (int o = threadIdx.x; o < nact * nr; o += blockDim.x) {
        const int a = o / nr, ir = o - a * nr;
        const float* row = M + (size_t)ir * ldm;
        float2 r;
        if (A.act_m[a] == 0) {
            double s = 0.0;
            for (int j = 0; j < na; j++) s += (double)row[j];
            r = make_float2((float)s, 0.f);
        } else {
            const float* tc = Tw + (size_t)a * na;
            const float* ts = Tw + pl + (size_t)a * na;
            float ca = 0.f, sa = 0.f;
            for (int j = 0; j < na; j++) {
                ca = fmaf(row[j], tc[j], ca);
                sa = fmaf(row[j], ts[j], sa);
            }
            r = make_float2(ca, sa);
        }
        S[o] = r;
    }
    __syncthreads();
    // radial contraction (p2conv.f:114-181): fr uses (G.M_c, G.M_s), ftheta
    // (+G.M_s, -G.M_c); Green rows of source ring is, columns of field ring ir
    for (int o = threadIdx.x; o < 2 * nact * nr; o += blockDim.x) {
        const int t = o / (nact * nr), rem = o - t * nact * nr, a = rem / nr, ir = rem - a * nr;
        const int m = A.act_m[a];
        float2 w = make_float2(0.f, 0.f);
        const bool valid = ((A.tmask >> t) & 1) && (t == 0 || ((m >= 1) && (m <= min(g.ng, g.mmax - 1) - 1)));
        if (valid) {
            const float* G = A.green + (((size_t)t * g.ng + m) * g.nkz) * nr * (size_t)nr + ir;
            const float2* Sa = S + (size_t)a * nr;
            float wc = 0.f, ws = 0.f;
            for (int is = 0; is < nr; is++) {
                const float gv = __ldg(G + (size_t)is * nr);
                const float2 sv = Sa[is];
                wc = fmaf(gv, sv.x, wc);
                ws = fmaf(gv, sv.y, ws);
            }
            w = (t == 0) ? make_float2(wc, ws) : make_float2(ws, -wc);
        }
        O[o] = w;
    }
    __syncthreads();
    // synthesis (p2fsyn.f:34-56, 1/na) and polcat (polcat.f:22-41):
    // f(j) = C + S, f(na - j) = C - S
    const float* TC = Tw + 2 * pl;
    const float* TS = Tw + 3 * pl;
    const int half = na / 2, nj = half + 1;
    float2* F = A.field + (size_t)d * mesh;
    for (int o = threadIdx.x; o < nr * nj; o += blockDim.x) {
        const int ir = o / nj, j = o - ir * nj;
        float c0 = 0.f, s0 = 0.f, c1 = 0.f, s1 = 0.f;
        for (int a = 0; a < nact; a++) {
            const float tc = TC[(size_t)a * na + j], ts = TS[(size_t)a * na + j];
            const float2 w0 = O[(size_t)a * nr + ir], w1 = O[(size_t)(nact + a) * nr + ir];
            c0 = fmaf(w0.x, tc, c0);
            s0 = fmaf(w0.y, ts, s0);
            c1 = fmaf(w1.x, tc, c1);
            s1 = fmaf(w1.y, ts, s1);
        }
        float sn, cs;
        sincospif(2.0f * (float)j / (float)na, &sn, &cs);
        {
            const float fr = c0 + s0, ft = c1 + s1;
            F[(size_t)ir * na + j] = make_float2(fr * cs - ft * sn, fr * sn + ft * cs);
        }
        if (j > 0 && j < half) {
            const float fr = c0 - s0, ft = c1 - s1;
            F[(size_t)ir * na + (na - j)] = make_float2(fr * cs + ft * sn, -fr * sn + ft * cs);
        }
    }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ens_ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void ens_st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// mode 0: deposit at the current positions (masset) and A2; mode 1: one step
__global__ void __launch_bounds__(1024) k_ens_step(EnsArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ uint32_t s_epoch;
    __shared__ int s_last;
    __shared__ double red[3][32];
    const DevGeo& g = A.g;
    const int mesh = g.mesh;
    if (threadIdx.x == 0) s_epoch = ens_ld_acquire(&A.ctl[0]) + 1u;
    __syncthreads();
    const uint32_t epoch = s_epoch;

    // ---- field solve of the discs of this CTA, each published by its flag
    if (A.mode == 1) {
        for (int d = blockIdx.x; d < A.ndisc; d += gridDim.x) {
            ens_solve(A, d, reinterpret_cast<float*>(smraw));
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                ens_st_release(&A.ctl[2 + d], epoch);
            }
            __syncthreads();
        }
    }

    // ---- particle chunks
    float2* F = reinterpret_cast<float2*>(smraw);                              // [mesh]
    unsigned long long* bins = reinterpret_cast<unsigned long long*>(F + mesh);  // [mesh]
    float* X = A.P;
    float* Y = A.P + A.ntot;
    float* VX = A.P + 2 * A.ntot;
    float* VY = A.P + 3 * A.ntot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int c = blockIdx.x; c < A.nchunks; c += gridDim.x) {
        const int d = A.chunks[3 * c], s0 = A.chunks[3 * c + 1], s1 = A.chunks[3 * c + 2];
        if (A.mode == 1) {
            if (threadIdx.x == 0) {
                uint32_t it = 0;
                while (ens_ld_acquire(&A.ctl[2 + d]) != epoch) {
                    if (++it > ENS_SPIN) {
                        atomicExch(A.errword, 4);
                        break;
                    }
                    __nanosleep(100);
                }
            }
            __syncthreads();
            const float4* src = reinterpret_cast<const float4*>(A.field + (size_t)d * mesh);
            for (int i = threadIdx.x; i < mesh / 2; i += blockDim.x)
                reinterpret_cast<float4*>(F)[i] = __ldcg(src + i);
        }
        for (int i = threadIdx.x; i < mesh; i += blockDim.x) bins[i] = 0ull;
        __syncthreads();
        double sc = 0.0, ss = 0.0, sn = 0.0;
        for (int p = s0 + threadIdx.x; p < s1; p += blockDim.x) {
            float x = X[p], y = Y[p];
            if (A.mode == 1) {
                float vx = VX[p], vy = VY[p];
                // grdacc.f:40-84 at the old position, halo (frhalo.f:55-56);
                // the interpolation cell from the fast FP32 arithmetic, as the
                // single-disc pass forms it (the field is continuous across a
                // cell boundary, so a cell off by rounding changes nothing)
                const CellW cw = gx_cell_t<false, 2>(g, x, y, 0.f, true);
                float ax = 0.f, ay = 0.f;
                if (cw.key >= 0) {
                    float w[8];
                    int ic[8];
                    gx_weights(g, cw, w);
                    gx_corners(g, cw.key, ic);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        if (ic[k] < 0) continue;
                        const float2 f = F[ic[k]];
                        ax += f.x * w[k];
                        ay += f.y * w[k];
                    }
                }
                if (g.halo == 1 && cw.key >= 0) {
                    const float r2 = x * x + y * y;
                    const float rr = sqrtf(r2);
                    float fr = -g.halo_v2 * rr / (r2 + g.halo_rc2);
                    if (fr != 0.f) {
                        fr = fr / rr;
                        ax += fr * x;
                        ay += fr * y;
                    }
                } else if (g.halo == 2 && cw.key >= 0) {
                    float az_ = 0.f, ph_ = 0.f;
                    gx_disc_force(g, x, y, 0.f, ax, ay, az_, ph_);
                }
                // stpgrp.f:26-32
                vx += ax;
                vy += ay;
                x += vx;
                y += vy;
                X[p] = x;
                Y[p] = y;
                VX[p] = vx;
                VY[p] = vy;
            }
            // massgn.f:68-89 at the new position
            const CellW cn = gx_cell(g, x, y, 0.f, false);
            if (cn.key >= 0) {
                float w[8];
                int ic[8];
                gx_weights(g, cn, w);
                gx_corners(g, cn.key, ic);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (ic[k] >= 0) {
                        // round(w 2^20), ties to even, by one FMA with 1.5 2^23
                        const int v = __float_as_int(fmaf(w[k], ENS_FIXQ, 12582912.0f)) - 0x4B400000;
                        atomicAdd(&bins[ic[k]], (unsigned long long)(long long)v);
                    }
                const double xd = x, yd = y, r2 = xd * xd + yd * yd;
                if (r2 > 0.0) {
                    const double inv = 1.0 / r2;
                    sc += (xd * xd - yd * yd) * inv;
                    ss += 2.0 * xd * yd * inv;
                }
                sn += 1.0;
            }
        }
        // chunk sums of the m = 2 amplitude (fixed order: deterministic)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sc += __shfl_down_sync(0xffffffffu, sc, o);
            ss += __shfl_down_sync(0xffffffffu, ss, o);
            sn += __shfl_down_sync(0xffffffffu, sn, o);
        }
        if (lane == 0) {
            red[0][warp] = sc;
            red[1][warp] = ss;
            red[2][warp] = sn;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, b = 0.0, n = 0.0;
            for (int w = 0; w < nw; w++) {
                a += red[0][w];
                b += red[1][w];
                n += red[2][w];
            }
            A.a2part[3 * c] = a;
            A.a2part[3 * c + 1] = b;
            A.a2part[3 * c + 2] = n;
        }
        // flush the chunk's integer mass (integer atomics: order-free)
        unsigned long long* m64 = A.mass64 + (size_t)d * mesh;
        for (int i = threadIdx.x; i < mesh; i += blockDim.x) {
            const unsigned long long v = bins[i];
            if (v) atomicAdd(&m64[i], v);
        }
        __syncthreads();
    }

    // ---- the last CTA to finish records the A2 series entry
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(&A.ctl[1], 1u);
        s_last = (prev == gridDim.x - 1) ? 1 : 0;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double* out = A.series + (size_t)(epoch - 1) * A.ndisc * 2;
        for (int d = threadIdx.x; d < A.ndisc; d += blockDim.x) {
            double a = 0.0, b = 0.0, n = 0.0;
            for (int c = A.dchunk[d]; c < A.dchunk[d + 1]; c++) {
                a += __ldcg(&A.a2part[3 * c]);
                b += __ldcg(&A.a2part[3 * c + 1]);
                n += __ldcg(&A.a2part[3 * c + 2]);
            }
            out[2 * d] = (n > 0.0) ? a / n : 0.0;
            out[2 * d + 1] = (n > 0.0) ? b / n : 0.0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            A.ctl[1] = 0u;
            __threadfence();
            ens_st_release(&A.ctl[0], epoch);
        }
    }
}

// ---------------------------------------------------------------------------
// host side
#define ENS_CUDA(e, call)                                                    \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) {                                             \
            (e)->err = std::string(#call) + ": " + cudaGetErrorString(e_);   \
            return GX_ERR_CUDA;                                              \
        }                                                                    \
    } while (0)

static std::string g_ens_err;

__global__ void k_ens_aos_to_soa(const float* __restrict__ aos, float* __restrict__ P, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 4; k++) P[k * n + i] = aos[4 * i + k];
}
__global__ void k_ens_soa_to_aos(const float* __restrict__ P, float* __restrict__ aos, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 4; k++) aos[4 * i + k] = P[k * n + i];
}

// chunk table for the current chunk size, launch geometry for the current
// block size
static int ens_configure(GxEnsemble* e, int threads, int chunk) {
    GxCtx* c = e->ctx;
    std::vector<int32_t> ch;
    std::vector<int32_t> dc(e->ndisc + 1);
    for (int d = 0; d < e->ndisc; d++) {
        dc[d] = (int32_t)(ch.size() / 3);
        for (int64_t s = e->off[d]; s < e->off[d + 1]; s += chunk) {
            ch.push_back(d);
            ch.push_back((int32_t)s);
            ch.push_back((int32_t)std::min<int64_t>(s + chunk, e->off[d + 1]));
        }
    }
    dc[e->ndisc] = (int32_t)(ch.size() / 3);
    const int nch = (int)(ch.size() / 3);
    if (nch > e->nchunks_cap) {
        if (e->chunks) cudaFree(e->chunks);
        if (e->a2part) cudaFree(e->a2part);
        e->chunks = nullptr;
        e->a2part = nullptr;
        ENS_CUDA(e, cudaMalloc((void**)&e->chunks, sizeof(int32_t) * 3 * std::max(nch, 1)));
        ENS_CUDA(e, cudaMalloc((void**)&e->a2part, sizeof(double) * 3 * std::max(nch, 1)));
        e->nchunks_cap = nch;
    }
    if (nch > 0)
        ENS_CUDA(e, cudaMemcpyAsync(e->chunks, ch.data(), sizeof(int32_t) * ch.size(), cudaMemcpyHostToDevice,
                                    c->stream));
    ENS_CUDA(e, cudaMemcpyAsync(e->dchunk, dc.data(), sizeof(int32_t) * dc.size(), cudaMemcpyHostToDevice,
                                c->stream));
    ENS_CUDA(e, cudaStreamSynchronize(c->stream));
    e->nchunks = nch;
    e->threads = threads;
    e->chunk = chunk;
    const DevGeo& g = c->g;
    const size_t pl = (size_t)c->spec.nact * g.na;
    const size_t solve = sizeof(float) * (((size_t)g.nr * (g.na + 1) + 4 * pl + 3) & ~(size_t)3) +
                         sizeof(float2) * 3 * (size_t)c->spec.nact * g.nr;
    const size_t push = (sizeof(float2) + sizeof(unsigned long long)) * (size_t)g.mesh;
    e->smem = std::max(solve, push);
    ENS_CUDA(e, cudaFuncSetAttribute(k_ens_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e->smem));
    int per_sm = 0, sms = 0;
    ENS_CUDA(e, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_step, threads, e->smem));
    ENS_CUDA(e, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev));
    if (per_sm < 1) return e->err = "ensemble step kernel does not fit on an SM", GX_ERR_RANGE;
    e->grid = per_sm * sms;
    if (e->gexec) {
        cudaGraphExecDestroy(e->gexec);
        e->gexec = nullptr;
        e->gsteps = 0;
    }
    return GX_OK;
}

static EnsArgs ens_args(GxEnsemble* e, int mode) {
    GxCtx* c = e->ctx;
    EnsArgs A;
    A.g = c->g;
    A.ndisc = e->ndisc;
    A.nact = c->spec.nact;
    A.nchunks = e->nchunks;
    A.mode = mode;
    A.tmask = 1 | (c->g.ng > 1 ? 2 : 0);
    A.P = e->P;
    A.ntot = e->ntot;
    A.pm = e->pm;
    A.mass64 = e->mass64;
    A.field = e->field;
    A.chunks = e->chunks;
    A.dchunk = e->dchunk;
    A.a2part = e->a2part;
    A.series = e->series;
    A.ctl = e->ctl;
    A.errword = c->errword;
    A.green = c->green32;
    A.tw = e->tw;
    for (int a = 0; a < ENS_MAXACT; a++) A.act_m[a] = (a < c->spec.nact) ? c->spec.m[a] : 0;
    return A;
}

// one cooperative launch (all CTAs resident: the flag waits always end)
static int ens_launch(GxEnsemble* e, int mode) {
    EnsArgs A = ens_args(e, mode);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)e->grid);
    cfg.blockDim = dim3((unsigned)e->threads);
    cfg.dynamicSmemBytes = e->smem;
    cfg.stream = e->ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    ENS_CUDA(e, cudaLaunchKernelEx(&cfg, k_ens_step, A));
    e->launches++;
    return GX_OK;
}

static int ens_check(GxEnsemble* e) {
    int32_t ew = 0;
    ENS_CUDA(e, cudaMemcpy(&ew, e->ctx->errword, sizeof ew, cudaMemcpyDeviceToHost));
    if (ew) {
        char b[96];
        snprintf(b, sizeof b, "device check raised error word %d", ew);
        e->err = b;
        return GX_ERR_DEVICE;
    }
    return GX_OK;
}

extern "C" {

void gx_ensemble_destroy(GxEnsemble* e) {
    if (!e) return;
    if (e->ctx) {
        cudaSetDevice(e->ctx->dev);
        cudaStreamSynchronize(e->ctx->stream);
    }
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    void* ptrs[] = {e->P, e->pm, e->mass64, e->field, e->chunks, e->dchunk, e->a2part, e->series, e->ctl, e->tw};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->ctx) gx_destroy(e->ctx);
    delete e;
}

const char* gx_ensemble_last_error(const GxEnsemble* e) { return e ? e->err.c_str() : g_ens_err.c_str(); }

int gx_ensemble_create(const GxConfig* cfg, int ndisc, const int64_t* counts, const float* pmass,
                       const float* coords, int max_steps, GxEnsemble** out) {
    if (!cfg || !counts || !pmass || !out || ndisc < 1 || max_steps < 0) {
        g_ens_err = "null argument or ndisc < 1";
        return GX_ERR_ARG;
    }
    *out = nullptr;
    if (cfg->ndim != 2 || cfg->precision != GX_PREC_MIXED) {
        g_ens_err = "the ensemble runs 2D grids on the mixed path";
        return GX_ERR_ARG;
    }
    int64_t ntot = 0;
    for (int d = 0; d < ndisc; d++) {
        if (counts[d] < 0) {
            g_ens_err = "negative particle count";
            return GX_ERR_ARG;
        }
        ntot += counts[d];
    }
    if (ntot > (int64_t)INT32_MAX - 1) {
        g_ens_err = "more than 2^31 - 2 particles";
        return GX_ERR_RANGE;
    }
    if (ntot > 0 && !coords) {
        g_ens_err = "null coords";
        return GX_ERR_ARG;
    }
    GxEnsemble* e = new GxEnsemble();
    GxConfig c1 = *cfg;
    c1.pmass = 1.0f;
    int rc = gx_grdset(&c1, &e->ctx);
    if (rc) {
        g_ens_err = gx_last_error(nullptr);
        delete e;
        return rc;
    }
    GxCtx* c = e->ctx;
    const DevGeo& g = c->g;
    auto fail = [&](int code) {
        g_ens_err = e->err.empty() ? c->err : e->err;
        gx_ensemble_destroy(e);
        return code;
    };
    if (c->spec.nact > ENS_MAXACT) {
        e->err = "more than 64 active harmonics";
        return fail(GX_ERR_RANGE);
    }
    if ((size_t)g.mesh * (sizeof(float2) + sizeof(unsigned long long)) > 200 * 1024 || (g.mesh & 1)) {
        e->err = "grid too large for the ensemble (16 B per cell of shared memory, 200 KB at most)";
        return fail(GX_ERR_RANGE);
    }
    rc = gx_greenm(c);
    if (rc) return fail(rc);
    e->ndisc = ndisc;
    e->ntot = ntot;
    e->max_steps = max_steps;
    e->off.assign(ndisc + 1, 0);
    for (int d = 0; d < ndisc; d++) e->off[d + 1] = e->off[d] + counts[d];
    cudaStream_t st = c->stream;
    rc = [&]() -> int {
        ENS_CUDA(e, cudaMalloc((void**)&e->P, sizeof(float) * 4 * std::max<int64_t>(ntot, 1)));
        ENS_CUDA(e, cudaMalloc((void**)&e->pm, sizeof(float) * ndisc));
        ENS_CUDA(e, cudaMalloc((void**)&e->mass64, sizeof(unsigned long long) * ndisc * (size_t)g.mesh));
        ENS_CUDA(e, cudaMalloc((void**)&e->field, sizeof(float2) * ndisc * (size_t)g.mesh));
        ENS_CUDA(e, cudaMalloc((void**)&e->dchunk, sizeof(int32_t) * (ndisc + 1)));
        ENS_CUDA(e, cudaMalloc((void**)&e->series, sizeof(double) * 2 * ndisc * ((size_t)max_steps + ENS_SPARE)));
        ENS_CUDA(e, cudaMalloc((void**)&e->ctl, sizeof(uint32_t) * (2 + ndisc)));
        ENS_CUDA(e, cudaMalloc((void**)&e->tw, sizeof(float) * 4 * (size_t)c->spec.nact * g.na));
        ENS_CUDA(e, cudaEventCreate(&e->ev0));
        ENS_CUDA(e, cudaEventCreate(&e->ev1));
        ENS_CUDA(e, cudaMemcpyAsync(e->pm, pmass, sizeof(float) * ndisc, cudaMemcpyHostToDevice, st));
        ENS_CUDA(e, cudaMemsetAsync(e->mass64, 0, sizeof(unsigned long long) * ndisc * (size_t)g.mesh, st));
        ENS_CUDA(e, cudaMemsetAsync(e->ctl, 0, sizeof(uint32_t) * (2 + ndisc), st));
        ENS_CUDA(e, cudaMemsetAsync(e->series, 0, sizeof(double) * 2 * ndisc * ((size_t)max_steps + ENS_SPARE), st));
        int* mlist = nullptr;
        ENS_CUDA(e, cudaMallocAsync((void**)&mlist, sizeof(int) * c->spec.nact, st));
        ENS_CUDA(e, cudaMemcpyAsync(mlist, c->spec.m, sizeof(int) * c->spec.nact, cudaMemcpyHostToDevice, st));
        const int nt = c->spec.nact * g.na;
        k_ens_tables<<<(nt + 255) / 256, 256, 0, st>>>(g, c->spec.nact, mlist, e->tw);
        ENS_CUDA(e, cudaGetLastError());
        ENS_CUDA(e, cudaFreeAsync(mlist, st));
        if (ntot > 0) {
            float* stage = nullptr;
            ENS_CUDA(e, cudaMallocAsync((void**)&stage, sizeof(float) * 4 * ntot, st));
            ENS_CUDA(e, cudaMemcpyAsync(stage, coords, sizeof(float) * 4 * ntot, cudaMemcpyHostToDevice, st));
            k_ens_aos_to_soa<<<(unsigned)((ntot + 255) / 256), 256, 0, st>>>(stage, e->P, ntot);
            ENS_CUDA(e, cudaGetLastError());
            ENS_CUDA(e, cudaFreeAsync(stage, st));
        }
        return GX_OK;
    }();
    if (rc) return fail(rc);
    rc = ens_configure(e, 512, 16384);
    if (rc) return fail(rc);
    // masset: the initial integer mass and A2 at step 0
    rc = ens_launch(e, 0);
    if (rc) return fail(rc);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        e->err = "initial deposit failed";
        return fail(GX_ERR_CUDA);
    }
    rc = ens_check(e);
    if (rc) return fail(rc);
    *out = e;
    return GX_OK;
}

// nsteps steps; the launches of a batch of steps are captured once into a
// CUDA graph and replayed (when capture of the cooperative launch is
// refused, the steps are launched directly and use_graph turns off)
int gx_ensemble_step(GxEnsemble* e, int nsteps) {
    if (!e || nsteps < 0) return GX_ERR_ARG;
    if (e->steps_done + nsteps > e->max_steps) return e->err = "more steps than max_steps", GX_ERR_RANGE;
    GxCtx* c = e->ctx;
    cudaSetDevice(c->dev);
    cudaStream_t st = c->stream;
    e->launches = 0;
    ENS_CUDA(e, cudaEventRecord(e->ev0, st));
    int left = nsteps;
    const int G = 16;
    if (e->use_graph && left >= G) {
        if (!e->gexec || e->gsteps != G) {
            if (e->gexec) cudaGraphExecDestroy(e->gexec);
            e->gexec = nullptr;
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            for (int k = 0; ok && k < G; k++) {
                EnsArgs A = ens_args(e, 1);
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)e->grid);
                cfg.blockDim = dim3((unsigned)e->threads);
                cfg.dynamicSmemBytes = e->smem;
                cfg.stream = st;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeCooperative;
                at[0].val.cooperative = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                ok = cudaLaunchKernelEx(&cfg, k_ens_step, A) == cudaSuccess;
            }
            cudaError_t ec = cudaStreamEndCapture(st, &graph);
            ok = ok && ec == cudaSuccess && graph;
            if (ok) ok = cudaGraphInstantiate(&e->gexec, graph, 0) == cudaSuccess;
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            if (ok) {
                e->gsteps = G;
            } else {
                e->gexec = nullptr;
                e->use_graph = false;
            }
        }
        while (e->gexec && left >= G) {
            ENS_CUDA(e, cudaGraphLaunch(e->gexec, st));
            e->launches += G;
            left -= G;
        }
    }
    for (; left > 0; left--) {
        int rc = ens_launch(e, 1);
        if (rc) return rc;
    }
    ENS_CUDA(e, cudaEventRecord(e->ev1, st));
    ENS_CUDA(e, cudaEventSynchronize(e->ev1));
    ENS_CUDA(e, cudaEventElapsedTime(&e->last_ms, e->ev0, e->ev1));
    e->steps_done += nsteps;
    return ens_check(e);
}

// autotuner: times each (threads, chunk) candidate over a few steps from a
// snapshot of the state, restores the state, keeps the fastest
int gx_ensemble_tune(GxEnsemble* e, int* threads_out, int* chunk_out) {
    if (!e) return GX_ERR_ARG;
    GxCtx* c = e->ctx;
    cudaSetDevice(c->dev);
    cudaStream_t st = c->stream;
    const DevGeo& g = c->g;
    const size_t pbytes = sizeof(float) * 4 * std::max<int64_t>(e->ntot, 1);
    const size_t mbytes = sizeof(unsigned long long) * e->ndisc * (size_t)g.mesh;
    const size_t cbytes = sizeof(uint32_t) * (2 + e->ndisc);
    char *sp = nullptr, *sm = nullptr, *sc = nullptr;
    ENS_CUDA(e, cudaMalloc((void**)&sp, pbytes));
    ENS_CUDA(e, cudaMalloc((void**)&sm, mbytes));
    ENS_CUDA(e, cudaMalloc((void**)&sc, cbytes));
    ENS_CUDA(e, cudaMemcpyAsync(sp, e->P, pbytes, cudaMemcpyDeviceToDevice, st));
    ENS_CUDA(e, cudaMemcpyAsync(sm, e->mass64, mbytes, cudaMemcpyDeviceToDevice, st));
    ENS_CUDA(e, cudaMemcpyAsync(sc, e->ctl, cbytes, cudaMemcpyDeviceToDevice, st));
    const int cand_t[3] = {256, 512, 1024};
    const int cand_c[4] = {4096, 8192, 16384, 32768};
    float best = 1e30f;
    int bt = e->threads, bc = e->chunk;
    int rc = GX_OK;
    const int reps = ENS_TUNE_REPS;
    for (int it = 0; it < 3 && rc == GX_OK; it++) {
        for (int ic = 0; ic < 4 && rc == GX_OK; ic++) {
            rc = ens_configure(e, cand_t[it], cand_c[ic]);
            if (rc) break;
            // warm-up step, then the timed steps; the series entries they
            // write (at most ENS_TUNE_REPS + 1 past the recorded ones, inside
            // the ENS_SPARE spare entries) are rewritten by later steps
            rc = ens_launch(e, 1);
            if (rc) break;
            ENS_CUDA(e, cudaEventRecord(e->ev0, st));
            for (int r = 0; r < reps && rc == GX_OK; r++) rc = ens_launch(e, 1);
            ENS_CUDA(e, cudaEventRecord(e->ev1, st));
            if (rc) break;
            ENS_CUDA(e, cudaEventSynchronize(e->ev1));
            float ms = 0.f;
            ENS_CUDA(e, cudaEventElapsedTime(&ms, e->ev0, e->ev1));
            if (ms < best) {
                best = ms;
                bt = cand_t[it];
                bc = cand_c[ic];
            }
            ENS_CUDA(e, cudaMemcpyAsync(e->P, sp, pbytes, cudaMemcpyDeviceToDevice, st));
            ENS_CUDA(e, cudaMemcpyAsync(e->mass64, sm, mbytes, cudaMemcpyDeviceToDevice, st));
            ENS_CUDA(e, cudaMemcpyAsync(e->ctl, sc, cbytes, cudaMemcpyDeviceToDevice, st));
        }
    }
    ENS_CUDA(e, cudaStreamSynchronize(st));
    cudaFree(sp);
    cudaFree(sm);
    cudaFree(sc);
    if (rc) return rc;
    rc = ens_configure(e, bt, bc);
    if (rc) return rc;
    if (threads_out) *threads_out = bt;
    if (chunk_out) *chunk_out = bc;
    return ens_check(e);
}

int gx_ensemble_config(const GxEnsemble* e, int* threads, int* chunk, int* grid, int* graph) {
    if (!e) return GX_ERR_ARG;
    if (threads) *threads = e->threads;
    if (chunk) *chunk = e->chunk;
    if (grid) *grid = e->grid;
    if (graph) *graph = e->use_graph ? 1 : 0;
    return GX_OK;
}

int gx_ensemble_steps_done(const GxEnsemble* e, int64_t* n) {
    if (!e || !n) return GX_ERR_ARG;
    *n = e->steps_done;
    return GX_OK;
}

int gx_ensemble_a2(GxEnsemble* e, double* out, int64_t cap) {
    if (!e || !out) return GX_ERR_ARG;
    const int64_t need = (e->steps_done + 1) * 2 * (int64_t)e->ndisc;
    if (cap < need) return e->err = "output smaller than (steps_done + 1) * ndisc * 2", GX_ERR_RANGE;
    cudaSetDevice(e->ctx->dev);
    ENS_CUDA(e, cudaMemcpy(out, e->series, sizeof(double) * need, cudaMemcpyDeviceToHost));
    return GX_OK;
}

int gx_ensemble_unload(GxEnsemble* e, float* coords) {
    if (!e || (e->ntot > 0 && !coords)) return GX_ERR_ARG;
    if (e->ntot == 0) return GX_OK;
    GxCtx* c = e->ctx;
    cudaSetDevice(c->dev);
    float* stage = nullptr;
    ENS_CUDA(e, cudaMallocAsync((void**)&stage, sizeof(float) * 4 * e->ntot, c->stream));
    k_ens_soa_to_aos<<<(unsigned)((e->ntot + 255) / 256), 256, 0, c->stream>>>(e->P, stage, e->ntot);
    ENS_CUDA(e, cudaGetLastError());
    ENS_CUDA(e, cudaMemcpyAsync(coords, stage, sizeof(float) * 4 * e->ntot, cudaMemcpyDeviceToHost, c->stream));
    ENS_CUDA(e, cudaFreeAsync(stage, c->stream));
    ENS_CUDA(e, cudaStreamSynchronize(c->stream));
    return GX_OK;
}

int gx_ensemble_last_ms(const GxEnsemble* e, float* ms, int64_t* launches) {
    if (!e) return GX_ERR_ARG;
    if (ms) *ms = e->last_ms;
    if (launches) *launches = e->launches;
    return GX_OK;
}

}  // extern "C"
