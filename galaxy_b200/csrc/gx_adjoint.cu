// gx_adjoint.cu -- adjoint of the 2D mixed-path step for the objective
// J = |A2(x_T)|, A2 = (1/n) sum_p e^{2 i phi_p} over all particles.
//
// Forward: nsteps of massgn, findf (+ polcat), getacc with the ISOT halo,
// stpgrp (the arithmetic of gx_step on particles kept in load order), with
// a checkpoint of (x, v) every ckpt_every steps.  Reverse sweep, from the
// final state: the trajectory is recomputed backwards by time reversal,
// x_s = x_{s+1} - v_{s+1}, v_s = v_{s+1} - a(x_s), and reset to the
// checkpoint at every checkpoint step; at each step, with
// mu = lambda_v + lambda_x:
//   lambda_v <- mu
//   lambda_x <- lambda_x + sum_c grad W_c(x) (F_c . mu)        (k_adj_a)
//               + halo Jacobian . mu
//               + pmass sum_c grad W_c(x) psi_c                   (k_adj_b)
// with psi = K^T Q, Q_c = sum_p W_c(x_p) mu_p (FP64 atomics into the mesh)
// and K the linear map mass -> (fx, fy): forward DFT of the active
// harmonics (p2manl.f:32-45), radial contraction (p2conv.f:114-181),
// synthesis (p2fsyn.f:34-56), polcat (polcat.f:22-41); K^T runs those
// steps transposed in reverse order (k_adjt_syn, k_adjt_conv, k_adjt_fwd).
// dJ/d(halo_rc, halo_v2) accumulate the halo's parameter derivatives . mu
// per block in FP64.
#include <algorithm>
#include <vector>

#include "gx_common.cuh"

#define ADJ_BS 256

// cell, weights and weight gradients at (x, y) (weight.f:61-101); 2D, one sector
__device__ __forceinline__ bool adj_wgrad(const DevGeo& g, float x, float y, int& key, float* w,
                                          float (*dw)[2]) {
    const CellW cw = gx_cell(g, x, y, 0.f, true);
    key = cw.key;
    if (cw.key < 0) return false;
    gx_weights(g, cw, w);
    const float r2 = x * x + y * y;
    if (!(r2 > 0.f)) {
        for (int k = 0; k < 4; k++) dw[k][0] = dw[k][1] = 0.f;
        return true;
    }
    const float rr = sqrtf(r2);
    const float dudr = (g.rmap == GX_RMAP_STDPOL) ? g.inv_ua / (1.f + rr) : g.inv_ua / rr;
    const float gu[2] = {dudr * x / rr, dudr * y / rr};
    const float ts = g.t_scale / r2;
    const float gt[2] = {-y * ts, x * ts};
    const float du = cw.du, dt = cw.dt;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        dw[0][i] = -(1.f - dt) * gu[i] - (1.f - du) * gt[i];
        dw[1][i] = -dt * gu[i] + (1.f - du) * gt[i];
        dw[2][i] = (1.f - dt) * gu[i] - du * gt[i];
        dw[3][i] = dt * gu[i] + du * gt[i];
    }
    return true;
}

// acceleration at (x, y) from the Cartesian field and the halo (grdacc + halfrc)
__device__ __forceinline__ void adj_accel(const DevGeo& g, const float4* __restrict__ F, int key,
                                          const float* w, float x, float y, float& ax, float& ay) {
    ax = ay = 0.f;
    if (key < 0) return;
    int ic[8];
    gx_corners(g, key, ic);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (ic[k] < 0) continue;
        const float4 f = __ldg(F + ic[k]);
        ax += f.x * w[k];
        ay += f.y * w[k];
    }
    if (g.halo == 1) {
        const float r2 = x * x + y * y, rr = sqrtf(r2);
        float fr = -g.halo_v2 * rr / (r2 + g.halo_rc2);
        if (fr != 0.f) {
            fr = fr / rr;
            ax += fr * x;
            ay += fr * y;
        }
    }
}

// particles in load order from the context's storage order
__global__ void k_adj_gather(const float* __restrict__ Pc, int64_t cap, int64_t n,
                             const int32_t* __restrict__ origin, float* __restrict__ S) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t o = origin[i];
    for (int k = 0; k < 4; k++) S[k * n + o] = Pc[k * cap + i];
}

// forward step of particles in load order: v += a(x); x += v (stpgrp.f:26-32)
__global__ void k_adj_fwd(DevGeo g, float* __restrict__ S, int64_t n, const float4* __restrict__ F) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = S[i], y = S[n + i], vx = S[2 * n + i], vy = S[3 * n + i];
    const CellW cw = gx_cell(g, x, y, 0.f, true);
    float w[8];
    if (cw.key >= 0) gx_weights(g, cw, w);
    float ax, ay;
    adj_accel(g, F, cw.key, w, x, y, ax, ay);
    vx += ax;
    vy += ay;
    S[i] = x + vx;
    S[n + i] = y + vy;
    S[2 * n + i] = vx;
    S[3 * n + i] = vy;
}

// reverse drift x_s = x_{s+1} - v_{s+1}
__global__ void k_adj_rdrift(float* __restrict__ S, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    S[i] -= S[2 * n + i];
    S[n + i] -= S[3 * n + i];
}

// largest |difference| between the reversed state and its checkpoint (max of
// non-negative floats as ordered integers: order-free)
__global__ void k_adj_drift(const float* __restrict__ S, const float* __restrict__ C, int64_t n4,
                            unsigned int* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n4) return;
    const float d = fabsf(S[i] - C[i]);
    if (d > 0.f) atomicMax(out, __float_as_uint(d));
}

// per-block FP64 sums of e^{2 i phi} over all particles
__global__ void k_adj_a2(const float* __restrict__ S, int64_t n, double* __restrict__ part) {
    __shared__ double sh[2][ADJ_BS / 32];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double c = 0.0, s = 0.0;
    if (i < n) {
        const double x = S[i], y = S[n + i], r2 = x * x + y * y;
        if (r2 > 0.0) {
            c = (x * x - y * y) / r2;
            s = 2.0 * x * y / r2;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, o);
        s += __shfl_down_sync(0xffffffffu, s, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][warp] = c;
        sh[1][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < ADJ_BS / 32; w++) {
            a += sh[0][w];
            b += sh[1][w];
        }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

// lambda_x at the final time: dJ/dx_T; lambda_v = 0
__global__ void k_adj_init(const float* __restrict__ S, int64_t n, double a2r, double a2i, double J,
                           float* __restrict__ L) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gx = 0.f, gy = 0.f;
    const double x = S[i], y = S[n + i], r2 = x * x + y * y;
    if (r2 > 0.0 && J > 0.0) {
        const double fr = (x * x - y * y) / r2, fi = 2.0 * x * y / r2, inv = 1.0 / (double)n;
        // dA2/dx = -2 i f y / (n r2), dA2/dy = 2 i f x / (n r2); dJ = Re(conj(A2) dA2) / J
        const double dxr = 2.0 * fi * y / r2 * inv, dxi = -2.0 * fr * y / r2 * inv;
        const double dyr = -2.0 * fi * x / r2 * inv, dyi = 2.0 * fr * x / r2 * inv;
        gx = (float)((a2r * dxr + a2i * dxi) / J);
        gy = (float)((a2r * dyr + a2i * dyi) / J);
    }
    L[i] = gx;
    L[n + i] = gy;
    L[2 * n + i] = 0.f;
    L[3 * n + i] = 0.f;
}

// reverse step, first particle pass at x_s: reverse kick (unless the state
// came from a checkpoint), mu, lambda_v <- mu, lambda_x += interpolation
// slope . (F . mu) + halo Jacobian . mu, Q += W mu, halo parameter terms
__global__ void __launch_bounds__(ADJ_BS) k_adj_a(DevGeo g, float* __restrict__ S, float* __restrict__ L,
                                                  int64_t n, const float4* __restrict__ F, int kick,
                                                  double* __restrict__ Q, double* __restrict__ tpart) {
    __shared__ double sh[2][ADJ_BS / 32];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t mesh = g.mesh;
    double drc = 0.0, dv2 = 0.0;
    if (i < n) {
        const float x = S[i], y = S[n + i];
        int key;
        float w[8], dw[4][2];
        const bool on = adj_wgrad(g, x, y, key, w, dw);
        if (kick) {
            float ax, ay;
            adj_accel(g, F, on ? key : -1, w, x, y, ax, ay);
            S[2 * n + i] -= ax;
            S[3 * n + i] -= ay;
        }
        float lx = L[i], ly = L[n + i];
        const float m0 = L[2 * n + i] + lx, m1 = L[3 * n + i] + ly;
        L[2 * n + i] = m0;
        L[3 * n + i] = m1;
        if (on) {
            int ic[8];
            gx_corners(g, key, ic);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (ic[k] < 0) continue;
                const float4 f = __ldg(F + ic[k]);
                const float fdot = f.x * m0 + f.y * m1;
                lx += dw[k][0] * fdot;
                ly += dw[k][1] * fdot;
                atomicAdd(&Q[ic[k]], (double)(w[k] * m0));
                atomicAdd(&Q[mesh + ic[k]], (double)(w[k] * m1));
            }
            if (g.halo == 1) {
                // h = -v2 x / d, d = r^2 + rc^2: Jacobian -v2 (I / d - 2 x x^T / d^2)
                const float d = x * x + y * y + g.halo_rc2, v2 = g.halo_v2;
                const float hxx = -v2 * (1.f / d - 2.f * x * x / (d * d));
                const float hyy = -v2 * (1.f / d - 2.f * y * y / (d * d));
                const float hxy = v2 * 2.f * x * y / (d * d);
                lx += hxx * m0 + hxy * m1;
                ly += hxy * m0 + hyy * m1;
                const double xm = (double)x * m0 + (double)y * m1;
                dv2 = -xm / (double)d;
                drc = (double)v2 * 2.0 * sqrt((double)g.halo_rc2) * xm / ((double)d * d);
            }
        }
        L[i] = lx;
        L[n + i] = ly;
    }
    for (int o = 16; o > 0; o >>= 1) {
        drc += __shfl_down_sync(0xffffffffu, drc, o);
        dv2 += __shfl_down_sync(0xffffffffu, dv2, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][warp] = drc;
        sh[1][warp] = dv2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < ADJ_BS / 32; w++) {
            a += sh[0][w];
            b += sh[1][w];
        }
        // each block owns its slot and the steps run in order: deterministic
        tpart[2 * blockIdx.x] += a;
        tpart[2 * blockIdx.x + 1] += b;
    }
}

// second particle pass: lambda_x += pmass sum_c grad W_c(x) psi_c
__global__ void k_adj_b(DevGeo g, const float* __restrict__ S, float* __restrict__ L, int64_t n,
                        const float* __restrict__ psi, float pmass) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int key;
    float w[8], dw[4][2];
    if (!adj_wgrad(g, S[i], S[n + i], key, w, dw)) return;
    int ic[8];
    gx_corners(g, key, ic);
    float gx = 0.f, gy = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (ic[k] < 0) continue;
        const float p = psi[ic[k]];
        gx += dw[k][0] * p;
        gy += dw[k][1] * p;
    }
    L[i] += pmass * gx;
    L[n + i] += pmass * gy;
}

// ---------------------------------------------------------------------------
// K^T.  Synthesis weights of harmonic m at spoke j: c_m(j) = 1 (m = 0),
// (-1)^j (m = na/2), 2 cos(2 pi m j / na) otherwise; s_m(j) = -2 sin(...)
// (0 for m = 0, na/2); scale 1/na (p2fsyn.f:42-53).
struct AdjAct {
    int m[64];
};

// polcat^T and synthesis^T: V[t][a][ir] = scale sum_j g_t(ir, j) (c_m(j), s_m(j))
__global__ void k_adjt_syn(DevGeo g, AdjAct act, int nact, const double* __restrict__ Q,
                           float2* __restrict__ V) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    const int nr = g.nr, na = g.na;
    if (o >= 2 * nact * nr) return;
    const int t = o / (nact * nr), rem = o - t * nact * nr, a = rem / nr, ir = rem - a * nr;
    const int m = act.m[a];
    const int64_t mesh = g.mesh;
    float sa = 0.f, sb = 0.f;
    for (int j = 0; j < na; j++) {
        const int64_t l = (int64_t)ir * na + j;
        const float qx = (float)Q[l], qy = (float)Q[mesh + l];
        float sn, cs;
        sincospif(2.0f * (float)j / (float)na, &sn, &cs);
        const float gv = (t == 0) ? (qx * cs + qy * sn) : (-qx * sn + qy * cs);
        if (m == 0) {
            sa += gv;
        } else if (m == g.mmax - 1) {
            sa += (j & 1) ? -gv : gv;
        } else {
            float sm, cm;
            sincospif(2.0f * (float)(((int64_t)m * j) % na) / (float)na, &sm, &cm);
            sa += 2.f * gv * cm;
            sb -= 2.f * gv * sm;
        }
    }
    const float scale = 1.0f / (float)na;
    V[o] = make_float2(scale * sa, scale * sb);
}

// radial contraction^T: per (a, is) one warp over ir
__global__ void k_adjt_conv(DevGeo g, AdjAct act, int nact, const float* __restrict__ G,
                            const float2* __restrict__ V, float2* __restrict__ AB) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nr = g.nr;
    if (wid >= nact * nr) return;
    const int a = wid / nr, is = wid - a * nr, m = act.m[a];
    const bool hasb = (m > 0 && m < g.mmax - 1);
    const bool ft = (g.ng > 1) && (m >= 1) && (m <= min(g.ng, g.mmax - 1) - 1);
    const float* G0 = G + ((size_t)(0 * g.ng + m) * g.nkz) * nr * (size_t)nr + (size_t)is * nr;
    const float* G1 = G + ((size_t)(1 * g.ng + m) * g.nkz) * nr * (size_t)nr + (size_t)is * nr;
    const float2* V0 = V + (size_t)a * nr;
    const float2* V1 = V + ((size_t)nact + a) * nr;
    float sa = 0.f, sb = 0.f;
    for (int ir = lane; ir < nr; ir += 32) {
        const float g0 = __ldg(G0 + ir);
        const float2 v0 = V0[ir];
        sa += g0 * v0.x;
        if (hasb) sb += g0 * v0.y;
        if (ft) {
            const float g1 = __ldg(G1 + ir);
            const float2 v1 = V1[ir];
            sb += g1 * v1.x;
            sa -= g1 * v1.y;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sa += __shfl_down_sync(0xffffffffu, sa, o);
        sb += __shfl_down_sync(0xffffffffu, sb, o);
    }
    if (lane == 0) AB[wid] = make_float2(sa, hasb ? sb : 0.f);
}

// forward DFT^T: psi(ir, j) = sum_a A cos(2 pi m j / na) - B sin(...)
__global__ void k_adjt_fwd(DevGeo g, AdjAct act, int nact, const float2* __restrict__ AB,
                           float* __restrict__ psi) {
    const int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (l >= g.mesh) return;
    const int na = g.na, nr = g.nr;
    const int ir = (int)(l / na), j = (int)(l - (int64_t)ir * na);
    float s = 0.f;
    for (int a = 0; a < nact; a++) {
        const float2 ab = AB[(size_t)a * nr + ir];
        float sm, cm;
        sincospif(2.0f * (float)(((int64_t)act.m[a] * j) % na) / (float)na, &sm, &cm);
        s += ab.x * cm - ab.y * sm;
    }
    psi[l] = s;
}

// ---------------------------------------------------------------------------
__global__ void k_adj_scatter(const float* __restrict__ S, int64_t n, float* __restrict__ Pc, int64_t cap,
                              int32_t* __restrict__ origin, int32_t* __restrict__ perm) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 4; k++) Pc[k * cap + i] = S[k * n + i];
    origin[i] = (int32_t)i;
    perm[i] = (int32_t)i;
}

namespace {
struct AdjBuf {
    float *S = nullptr, *L = nullptr, *ck = nullptr, *psi = nullptr;
    double *Q = nullptr, *part = nullptr, *tpart = nullptr;
    float2 *V = nullptr, *AB = nullptr;
    unsigned int* drift = nullptr;
    ~AdjBuf() {
        void* p[] = {S, L, ck, psi, Q, part, tpart, V, AB, drift};
        for (void* q : p)
            if (q) cudaFree(q);
    }
};
}  // namespace

// positions of S into the context (storage = load order) -> mass, field
static int adj_solve(GxCtx* c, const float* S, int64_t n) {
    GX_CUDA(c, cudaMemcpyAsync(c->pbuf[c->cur], S, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
    GX_CUDA(c, cudaMemcpyAsync(c->pbuf[c->cur] + c->cap, S + n, sizeof(float) * n, cudaMemcpyDeviceToDevice,
                               c->stream));
    c->zr_valid = false;  // the mass array is no longer a fused pass's
    int rc = gx_mixed_masset(c);
    if (rc) return rc;
    return gx_mixed_findf(c, 0, true);
}

extern "C" int gx_adjoint(GxCtx* c, int nsteps, int ckpt_every, double* J_out, float* grad,
                          double* dtheta, float* drift_out) {
    if (!c || nsteps < 0 || ckpt_every < 1 || !J_out || !grad || !dtheta) return GX_ERR_ARG;
    if (c->fp64 || c->g.ndim != 2 || c->g.nsect != 1)
        return c->err = "the adjoint runs 2D one-sector grids on the mixed path", GX_ERR_ARG;
    if (c->nzones > 1) return c->err = "the adjoint runs a single time-step zone", GX_ERR_ARG;
    if (c->g.halo > 1) return c->err = "the adjoint differentiates the ISOT halo only", GX_ERR_ARG;
    if (!c->have_green) return c->err = "no Green table (call gx_greenm)", GX_ERR_STATE;
    if (c->spec.nact > 64) return c->err = "more than 64 active harmonics", GX_ERR_RANGE;
    const int64_t n = c->n;
    if (n < 1) return c->err = "no particles loaded", GX_ERR_STATE;
    cudaSetDevice(c->dev);
    {
        const int rc = gx_dense(c);
        if (rc) return rc;
    }
    const DevGeo& g = c->g;
    const int nact = c->spec.nact;
    AdjAct act;
    for (int a = 0; a < 64; a++) act.m[a] = (a < nact) ? c->spec.m[a] : 0;
    const unsigned nb = (unsigned)((n + ADJ_BS - 1) / ADJ_BS);
    const int nck = nsteps / ckpt_every + 1;
    AdjBuf b;
    GX_CUDA(c, cudaMalloc((void**)&b.S, sizeof(float) * 4 * n));
    GX_CUDA(c, cudaMalloc((void**)&b.L, sizeof(float) * 4 * n));
    GX_CUDA(c, cudaMalloc((void**)&b.ck, sizeof(float) * 4 * n * (size_t)nck));
    GX_CUDA(c, cudaMalloc((void**)&b.psi, sizeof(float) * g.mesh));
    GX_CUDA(c, cudaMalloc((void**)&b.Q, sizeof(double) * 2 * g.mesh));
    GX_CUDA(c, cudaMalloc((void**)&b.part, sizeof(double) * 2 * nb));
    GX_CUDA(c, cudaMalloc((void**)&b.tpart, sizeof(double) * 2 * nb));
    GX_CUDA(c, cudaMalloc((void**)&b.V, sizeof(float2) * 2 * nact * g.nr));
    GX_CUDA(c, cudaMalloc((void**)&b.AB, sizeof(float2) * nact * g.nr));
    GX_CUDA(c, cudaMalloc((void**)&b.drift, sizeof(unsigned int)));
    cudaStream_t st = c->stream;
    c->launches = 0;
    GX_CUDA(c, cudaEventRecord(c->ev0, st));
    // initial state in load order
    k_adj_gather<<<nb, ADJ_BS, 0, st>>>(c->pbuf[c->cur], c->cap, n, c->origin, b.S);
    GX_LAUNCHED(c);
    const size_t sbytes = sizeof(float) * 4 * n;
    GX_CUDA(c, cudaMemcpyAsync(b.ck, b.S, sbytes, cudaMemcpyDeviceToDevice, st));
    // forward sweep with checkpoints
    for (int s = 0; s < nsteps; s++) {
        int rc = adj_solve(c, b.S, n);
        if (rc) return rc;
        k_adj_fwd<<<nb, ADJ_BS, 0, st>>>(g, b.S, n, c->field);
        GX_LAUNCHED(c);
        if ((s + 1) % ckpt_every == 0)
            GX_CUDA(c, cudaMemcpyAsync(b.ck + (size_t)((s + 1) / ckpt_every) * 4 * n, b.S, sbytes,
                                       cudaMemcpyDeviceToDevice, st));
    }
    // objective
    k_adj_a2<<<nb, ADJ_BS, 0, st>>>(b.S, n, b.part);
    GX_LAUNCHED(c);
    std::vector<double> hp(2 * (size_t)nb);
    GX_CUDA(c, cudaMemcpyAsync(hp.data(), b.part, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, st));
    GX_CUDA(c, cudaStreamSynchronize(st));
    double sre = 0.0, sim = 0.0;
    for (unsigned i = 0; i < nb; i++) {
        sre += hp[2 * i];
        sim += hp[2 * i + 1];
    }
    const double a2r = sre / (double)n, a2i = sim / (double)n;
    const double J = sqrt(a2r * a2r + a2i * a2i);
    k_adj_init<<<nb, ADJ_BS, 0, st>>>(b.S, n, a2r, a2i, J, b.L);
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaMemsetAsync(b.tpart, 0, sizeof(double) * 2 * nb, st));
    GX_CUDA(c, cudaMemsetAsync(b.drift, 0, sizeof(unsigned int), st));
    // reverse sweep
    for (int s = nsteps - 1; s >= 0; s--) {
        const bool ck = (s % ckpt_every) == 0;
        k_adj_rdrift<<<nb, ADJ_BS, 0, st>>>(b.S, n);
        GX_LAUNCHED(c);
        if (ck) {
            // the reversed positions against the checkpoint, then the checkpoint
            const float* C0 = b.ck + (size_t)(s / ckpt_every) * 4 * n;
            k_adj_drift<<<(unsigned)((2 * n + ADJ_BS - 1) / ADJ_BS), ADJ_BS, 0, st>>>(b.S, C0, 2 * n, b.drift);
            GX_LAUNCHED(c);
            GX_CUDA(c, cudaMemcpyAsync(b.S, C0, sbytes, cudaMemcpyDeviceToDevice, st));
        }
        int rc = adj_solve(c, b.S, n);
        if (rc) return rc;
        GX_CUDA(c, cudaMemsetAsync(b.Q, 0, sizeof(double) * 2 * g.mesh, st));
        k_adj_a<<<nb, ADJ_BS, 0, st>>>(g, b.S, b.L, n, c->field, ck ? 0 : 1, b.Q, b.tpart);
        GX_LAUNCHED(c);
        const int n_syn = 2 * nact * g.nr;
        k_adjt_syn<<<(n_syn + 127) / 128, 128, 0, st>>>(g, act, nact, b.Q, b.V);
        GX_LAUNCHED(c);
        const int n_conv = nact * g.nr * 32;
        k_adjt_conv<<<(n_conv + 255) / 256, 256, 0, st>>>(g, act, nact, c->green32, b.V, b.AB);
        GX_LAUNCHED(c);
        k_adjt_fwd<<<(unsigned)((g.mesh + 255) / 256), 256, 0, st>>>(g, act, nact, b.AB, b.psi);
        GX_LAUNCHED(c);
        k_adj_b<<<nb, ADJ_BS, 0, st>>>(g, b.S, b.L, n, b.psi, g.pmass);
        GX_LAUNCHED(c);
    }
    GX_CUDA(c, cudaEventRecord(c->ev1, st));
    // gradient in load order (x, y, vx, vy)
    std::vector<float> hl(4 * (size_t)n);
    GX_CUDA(c, cudaMemcpyAsync(hl.data(), b.L, sbytes, cudaMemcpyDeviceToHost, st));
    GX_CUDA(c, cudaMemcpyAsync(hp.data(), b.tpart, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, st));
    unsigned int hd = 0;
    GX_CUDA(c, cudaMemcpyAsync(&hd, b.drift, sizeof hd, cudaMemcpyDeviceToHost, st));
    GX_CUDA(c, cudaStreamSynchronize(st));
    GX_CUDA(c, cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1));
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 4; k++) grad[4 * i + k] = hl[(size_t)k * n + i];
    double drc = 0.0, dv2 = 0.0;
    for (unsigned i = 0; i < nb; i++) {
        drc += hp[2 * i];
        dv2 += hp[2 * i + 1];
    }
    dtheta[0] = drc;
    dtheta[1] = dv2;
    *J_out = J;
    if (drift_out) {
        float d;
        memcpy(&d, &hd, sizeof d);
        *drift_out = d;
    }
    // the context again holds the initial particles (load order) and their mass
    k_adj_scatter<<<nb, ADJ_BS, 0, st>>>(b.ck, n, c->pbuf[c->cur], c->cap, c->origin, c->perm);
    GX_LAUNCHED(c);
    if (g.comp)  // the low parts of compensated positions start at zero, as after gx_loadup
        GX_CUDA(c, cudaMemsetAsync(c->pbuf[c->cur] + (size_t)4 * c->cap, 0, sizeof(float) * 2 * c->cap, st));
    c->have_keys = false;
    c->zr_valid = false;
    int rc = gx_mixed_masset(c);
    if (rc) return rc;
    GX_CUDA(c, cudaStreamSynchronize(st));
    c->have_mass = true;
    c->have_field = false;
    int32_t ew = 0;
    GX_CUDA(c, cudaMemcpy(&ew, c->errword, sizeof ew, cudaMemcpyDeviceToHost));
    if (ew) return c->err = "device check raised the error word", GX_ERR_DEVICE;
    return GX_OK;
}
