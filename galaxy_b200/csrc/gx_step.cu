// gx_step.cu -- particle side of the mixed-precision path.
//
//   k_push         one pass per step over the particles in row-sorted order
//                  (getacc + stpgrp + the new cell of massgn's weight
//                  call): weights of the stored cell (weight.f:61-101, 196-250),
//                  gather of the float4 field at the 4/8 corners
//                  (grdacc.f:40-84, 189-218), rigid halo (getacc.f:103-122,
//                  frhalo.f:55-56), v += a, x += v (stpgrp.f:26-32), off-grid
//                  test (offgrd.f:51-77), the key and fractions of the new
//                  cell for the deposit of the same step (whose rows the
//                  pass also counts, gx_deposit.cu).  The interpolation
//                  cell of the current position is recomputed from it
//                  rather than stored from the previous step: the pass is
//                  bound by memory traffic, not by that arithmetic.
#include <algorithm>

#include "gx_common.cuh"

// ---------------------------------------------------------------------------
// row key of a cell (nrow for particles off the grid)
__device__ __forceinline__ uint32_t row_of(const DevGeo& g, const CellW& c) {
    return (c.key >= 0) ? (uint32_t)c.row : (uint32_t)g.nrow;
}

__device__ __forceinline__ void gx_accel(const DevGeo& g, const float4* __restrict__ F, float x,
                                         float y, float z, float& ax, float& ay, float& az,
                                         float& ph) {
    const CellW cw = gx_cell(g, x, y, z, true);
    gx_accel_cell(g, F, cw, x, y, z, ax, ay, az, ph);
}

// the fused particle pass of one step: the interpolation cell of the
// current position, the move, the key and fractions of the new cell,
// counted by row for the deposit's counting sort.
// Eight CTAs per SM (32 registers; four for the 27-point pass, which would
// spill): the pass waits on its gathers, and the extra resident warps hide
// more of that latency than the capped registers cost.
template <bool Q, int ND>
__global__ void __launch_bounds__(256, Q ? 4 : 8) k_push(DevGeo g, const float* __restrict__ Pin,
                                              float* __restrict__ Pout, int64_t cap, int64_t n,
                                              const int32_t* __restrict__ perm,
                                              const int32_t* __restrict__ orig_in,
                                              int32_t* __restrict__ orig_out,
                                              const float4* __restrict__ F,
                                              int32_t* __restrict__ key_out,
                                              float* __restrict__ fr_out,
                                              uint32_t* __restrict__ rowcnt,
                                              float* __restrict__ pot) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool act = s < n;
    uint32_t row = 0;
    if (act) {
        const int p = perm[s];
        constexpr bool d3 = ND == 3;
        float x = Pin[p], y = Pin[cap + p], z = 0.f, vx, vy, vz = 0.f;
        if (d3) {
            z = Pin[2 * cap + p];
            vx = Pin[3 * cap + p];
            vy = Pin[4 * cap + p];
            vz = Pin[5 * cap + p];
        } else {
            vx = Pin[2 * cap + p];
            vy = Pin[3 * cap + p];
        }
        const int32_t o = orig_in[p];
        const CellW cw = gx_cell_t<false, ND>(g, x, y, z, true);
        float ax, ay, az, ph;
        gx_accel_cell_t<Q, ND>(g, F, cw, x, y, z, ax, ay, az, ph);
        vx += ax;
        vy += ay;
        if (d3) vz += az;
        if (g.comp) {
            // compensated drift: the low parts travel with the particle
            const int nw = 2 * g.ndim;
            float xl = Pin[nw * cap + p], yl = Pin[(nw + 1) * cap + p];
            gx_comp_add(x, xl, vx);
            gx_comp_add(y, yl, vy);
            Pout[nw * cap + s] = xl;
            Pout[(nw + 1) * cap + s] = yl;
            if (d3) {
                float zl = Pin[(nw + 2) * cap + p];
                gx_comp_add(z, zl, vz);
                Pout[(nw + 2) * cap + s] = zl;
            }
        } else {
            x += vx;
            y += vy;
            if (d3) z += vz;
        }
        Pout[s] = x;
        Pout[cap + s] = y;
        if (d3) {
            Pout[2 * cap + s] = z;
            Pout[3 * cap + s] = vx;
            Pout[4 * cap + s] = vy;
            Pout[5 * cap + s] = vz;
        } else {
            Pout[2 * cap + s] = vx;
            Pout[3 * cap + s] = vy;
        }
        orig_out[s] = o;
        if (pot) pot[s] = ph;
        const CellW cn = gx_cell_t<true, ND>(g, x, y, z, false);
        key_out[s] = cn.key;
        fr_out[s] = cn.du;
        fr_out[cap + s] = cn.dt;
        if (d3) fr_out[2 * cap + s] = cn.dz;
        row = row_of(g, cn);
    }
    gx_row_count(row, act, rowcnt + (size_t)(blockIdx.x & (NCOPY - 1)) * (g.nrow + 1));
}

// getacc for every particle at its stored position, written in load order
__global__ void k_getacc(DevGeo g, const float* __restrict__ P, int64_t cap, int64_t n,
                         const int32_t* __restrict__ origin, const float4* __restrict__ F,
                         float* __restrict__ acc, float* __restrict__ pot) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nd = g.ndim;
    float z = (nd == 3) ? P[2 * cap + i] : 0.f;
    float ax, ay, az, ph;
    gx_accel(g, F, P[i], P[cap + i], z, ax, ay, az, ph);
    const int64_t o = origin[i];
    acc[o * nd] = ax;
    acc[o * nd + 1] = ay;
    if (nd == 3) acc[o * nd + 2] = az;
    if (pot) pot[o] = ph;
}

// ---------------------------------------------------------------------------
int gx_mixed_step(GxCtx* c, int nsteps, int phys) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    for (int s = 0; s < nsteps; s++) {
        const bool last = (s == nsteps - 1);
        int rc = gx_mixed_findf(c, phys && last, true);
        if (rc) return rc;
        const int nxt = c->cur ^ 1;
        rc = gx_phase_mark(c, PH_PUSH);
        if (rc) return rc;
        if (n > 0) {
            auto kp = g.quad ? k_push<true, 3> : (g.ndim == 3) ? k_push<false, 3> : k_push<false, 2>;
            kp<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
                g, c->pbuf[c->cur], c->pbuf[nxt], c->cap, n, c->perm, c->origin, c->origin_tmp,
                c->field, c->pkey[nxt], c->pfr, c->rowcnt,
                (phys && last) ? c->ppot : nullptr);
            GX_LAUNCHED(c);
        }
        std::swap(c->origin, c->origin_tmp);
        c->cur = nxt;
        // the pass wrote particles in processing order; the new permutation
        // orders them by their new rows
        rc = gx_deposit_rows(c, c->pkey[c->cur], c->pfr, c->perm_next);
        if (rc) return rc;
        std::swap(c->perm, c->perm_next);
    }
    int rc = gx_phase_end(c);
    if (rc) return rc;
    c->have_field = false;
    return GX_OK;
}

int gx_mixed_getacc(GxCtx* c, float* acc, float* pot) {
    const DevGeo& g = c->g;
    const int64_t n = c->n;
    if (n == 0) return GX_OK;
    int bs = 256;
    k_getacc<<<(unsigned)((n + bs - 1) / bs), bs, 0, c->stream>>>(
        g, c->pbuf[c->cur], c->cap, n, c->origin, c->field, c->pacc, c->ppot);
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaMemcpyAsync(acc, c->pacc, sizeof(float) * g.ndim * n, cudaMemcpyDeviceToHost,
                               c->stream));
    if (pot)
        GX_CUDA(c, cudaMemcpyAsync(pot, c->ppot, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    return GX_OK;
}

// ---------------------------------------------------------------------------
// weight entry point (cell numbers and weights of host particle records)
__global__ void k_weight_aos(DevGeo g, const float* __restrict__ aos, int64_t n, int old,
                             int32_t* __restrict__ ncl, float* __restrict__ wt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nw = 2 * g.ndim, nwt = g.quad ? 27 : 8;
    const float* q = aos + i * nw;
    CellW c = gx_cell(g, q[0], q[1], (g.ndim == 3) ? q[2] : 0.f, old != 0);
    float w[27];
    for (int k = 0; k < 27; k++) w[k] = 0.f;
    if (c.key >= 0) {
        if (g.quad) gx_weights27(c, w);
        else gx_weights(g, c, w);
    }
    ncl[i] = c.key;
    for (int k = 0; k < nwt; k++) wt[i * nwt + k] = w[k];
}

extern "C" int gx_weight(GxCtx* c, const float* coords, int64_t n, int old, int32_t* ncl, float* wt) {
    if (!c || n < 0 || (n > 0 && (!coords || !ncl || !wt))) return GX_ERR_ARG;
    if (c->fp64) return c->err = "gx_weight reports the mixed path's FP32 cells", GX_ERR_ARG;
    if (n == 0) return GX_OK;
    cudaSetDevice(c->dev);
    const int nw = 2 * c->g.ndim;
    float *daos = nullptr, *dwt = nullptr;
    int32_t* dncl = nullptr;
    GX_CUDA(c, cudaMallocAsync((void**)&daos, sizeof(float) * nw * n, c->stream));
    const int nwt = c->g.quad ? 27 : 8;
    GX_CUDA(c, cudaMallocAsync((void**)&dwt, sizeof(float) * nwt * n, c->stream));
    GX_CUDA(c, cudaMallocAsync((void**)&dncl, sizeof(int32_t) * n, c->stream));
    GX_CUDA(c, cudaMemcpyAsync(daos, coords, sizeof(float) * nw * n, cudaMemcpyHostToDevice, c->stream));
    k_weight_aos<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, daos, n, old, dncl, dwt);
    GX_LAUNCHED(c);
    GX_CUDA(c, cudaMemcpyAsync(ncl, dncl, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaMemcpyAsync(wt, dwt, sizeof(float) * nwt * n, cudaMemcpyDeviceToHost, c->stream));
    GX_CUDA(c, cudaFreeAsync(daos, c->stream));
    GX_CUDA(c, cudaFreeAsync(dwt, c->stream));
    GX_CUDA(c, cudaFreeAsync(dncl, c->stream));
    GX_CUDA(c, cudaStreamSynchronize(c->stream));
    return GX_OK;
}
