// raster_fwd.cuh -- the forward rasteriser kernel, shared by the plain FP32
// unit (plain.cu, exact blend decision, no FMA contraction) and the
// reduced-storage unit (chosen.cu, fast exp, FMA contraction).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"
#include "raster_common.cuh"

namespace gs3d {
namespace {

// Rasterizer forward (rasterizer_cpu.cpp:38-53, 137-198).  Blend::decide is
// the alpha / transmittance decision (0 skip, 1 blend, 2 stop): exact in the
// plain form on the reference's power (power_rn), fast base-2 exponent in the
// reduced-storage form (Blend::kBase2: q_coeffs / q_at, ex2).  One CTA of 128
// threads per 16x16 tile, two pixels per thread: warp w owns the 16x4 strip
// of rows 4w..4w+3, a thread the pixels (x, 4w + lane/16) and
// (x, 4w + 2 + lane/16).  Batches of 128 records are gathered into shared
// memory with, per record, the warps whose strip the Gaussian can reach
// (band_rows: the rows of the tile's columns inside its alpha >= 1/255
// ellipse); each warp walks its own compacted list of the batch; the CTA
// stops once every pixel saturated.  LOSS: kCountContrib (renders: contributor
// counts kept), kFusedL1 (a train step: sign byte per pixel and the
// double-precision loss sum; the backward starts from each pixel's last
// contributor, no counts) or kLossLater (a train step whose target is still
// being copied in: neither, k_l1_loss follows once it has landed).
//
// PPT (pixels per thread: 1, 2 or 4) sets the threads per tile (256 / PPT)
// and each warp's strip (16 x 2*PPT rows); BATCH (64, 128 or 256) the records
// staged per round.  The results depend on neither.
constexpr int kFwdBatch = 128;
constexpr int kCountContrib = 0, kFusedL1 = 1, kLossLater = 2;

//
// MULTI: one persistent launch over the tiles of several views.  spp is then
// the array of the views' parameters; a CTA takes the next entry of `order`
// (all views' tiles, heavy first) from a work counter, finds the tile's view
// by its global id and renders it with that view's camera into the view's
// slice of the concatenated pixel buffers.  The fused loss adds each view's
// sum weighted by its inv_n.
template <int LOSS, class Blend, bool MULTI = false, int PPT = 2, int BATCH = kFwdBatch>
__global__ void __launch_bounds__(256 / PPT) k_raster_fwd(const StepParams* __restrict__ spp,
                                                            const unsigned* __restrict__ ranges,
                                                            const unsigned* __restrict__ order,
                                                            const unsigned* __restrict__ vals, ScreenPtrs s,
                                                            PixelPtrs px, Control* ctrl, int n_views = 1,
                                                            unsigned n_tiles = 0) {
    __shared__ float4 s_r0[BATCH];
    __shared__ float4 s_r1[BATCH];
    __shared__ float2 s_bt[BATCH];   // (blue, threshold): one 8-byte load per Gaussian
    constexpr int kFwdThreads = 256 / PPT;
    constexpr int kNW = kFwdThreads / 32;
    __shared__ unsigned char s_mask[BATCH];       // warps whose strip the Gaussian can reach
    __shared__ unsigned char s_list[kNW][BATCH];  // per warp: its batch entries, ascending
    __shared__ double s_loss[kFwdThreads / 32];
    __shared__ unsigned s_next;
    for (int iter = 0;; iter++) {
    int tile;
    if (MULTI) {
        if (threadIdx.x == 0) s_next = atomicAdd(&ctrl->work[0], 1u);
        __syncthreads();
        const unsigned t = s_next;
        __syncthreads();
        if (t >= n_tiles) break;
        tile = (int)order[t];
    } else {
        if (iter > 0) break;
        tile = order ? (int)order[blockIdx.x] : (int)blockIdx.x;
    }
    int view = 0;
    if (MULTI) {
        int lo = 0, hi = n_views;   // last view whose tile_base <= tile
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (spp[mid].tile_base <= (unsigned)tile) lo = mid;
            else hi = mid;
        }
        view = lo;
    }
    const StepParams& sp = spp[view];
    const int W = sp.cam.width, H = sp.cam.height;
    const int ltile = tile - (int)sp.tile_base;
    const int tx = ltile % sp.grid_x, ty = ltile / sp.grid_x;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = tx * kTile + (int)(lane & 15);
    const int ybase = ty * kTile + 2 * PPT * (int)warp + (int)(lane >> 4);
    const unsigned rs = ranges[2 * tile], re = ranges[2 * tile + 1];
    const float fx = (float)x;
    const float wx0 = (float)(tx * kTile), wx1 = wx0 + (float)(kTile - 1), ty0 = (float)(ty * kTile);
    float fy[PPT], T[PPT], C[PPT][3];
    int cnt[PPT];
    unsigned last[PPT];
    bool done[PPT];
#pragma unroll
    for (int p = 0; p < PPT; p++) {
        const int y = ybase + 2 * p;
        fy[p] = (float)y;
        T[p] = 1.0f;
        C[p][0] = C[p][1] = C[p][2] = 0.0f;
        cnt[p] = 0;
        last[p] = 0;
        done[p] = !(x < W && y < H);
    }
    for (unsigned b = rs; b < re; b += BATCH) {
        bool all_done = true;
#pragma unroll
        for (int p = 0; p < PPT; p++) all_done = all_done && done[p];
        if (__syncthreads_count(all_done) == kFwdThreads) break;
#pragma unroll
        for (int e = threadIdx.x; e < BATCH; e += kFwdThreads) {
            const unsigned j = b + (unsigned)e;
            if (j < re) {
                const unsigned g = vals[j];
                float4 r0 = s.rec0[g];
                float4 r1 = s.rec1[g];
                const float2 cb = s.cbt[g];
                const float thr = skip_threshold(cb.y);
                // the threshold in the units of Blend's exponent: the stored base-2 one, or the skip bound
                s_bt[e] = make_float2(cb.x, Blend::kBase2 ? cb.y : thr);
                s_mask[e] = (unsigned char)strip_mask<kNW, 2 * PPT>(band_rows(r0, r1, thr, wx0, wx1), ty0);
                if (Blend::kBase2) q_scale(r0, r1);
                s_r0[e] = r0;
                s_r1[e] = r1;
            }
        }
        __syncthreads();
        const int nb = (int)min((unsigned)BATCH, re - b);
        const int nl = warp_list(s_mask, nb, warp, s_list[warp]);
        for (int i = 0; i < nl; i++) {
            bool thread_done = true;
#pragma unroll
            for (int p = 0; p < PPT; p++) thread_done = thread_done && done[p];
            if (thread_done) break;
            const int k = s_list[warp][i];
            const float4 a = s_r0[k];
            const float4 c = s_r1[k];
            const float2 bt = s_bt[k];
            const float thr = bt.y;
            const float dx = a.x - fx;
            const float3 kq = Blend::kBase2 ? q_coeffs(a, c, dx) : make_float3(0.f, 0.f, 0.f);
#pragma unroll
            for (int p = 0; p < PPT; p++) {
                if (done[p]) continue;
                const float dy = a.y - fy[p];
                const float power = Blend::kBase2 ? q_at(kq, dy) : power_rn(a, c, dx, dy);
                // the reference also skips power > 0 (rasterizer_cpu.cpp:146-148); with a positive-definite
                // conic that is rounding at the mean, where the reduced form blends alpha = o instead
                if (Blend::kBase2 ? !(power >= thr) : (power < thr || power > 0.0f)) continue;
                float alpha, e, test_T;
                const int dec = Blend::decide(power, c.y, T[p], alpha, e, test_T);
                if (dec == 0) continue;
                if (dec == 2) {
                    done[p] = true;
                    continue;
                }
                if (Blend::kBase2) {   // single roundings: the image does not depend on PPT
                    const float aT = __fmul_rn(alpha, T[p]);
                    C[p][0] = __fmaf_rn(c.z, aT, C[p][0]);
                    C[p][1] = __fmaf_rn(c.w, aT, C[p][1]);
                    C[p][2] = __fmaf_rn(bt.x, aT, C[p][2]);
                } else {   // the reference's (c * alpha) * T
                    C[p][0] += c.z * alpha * T[p];
                    C[p][1] += c.w * alpha * T[p];
                    C[p][2] += bt.x * alpha * T[p];
                }
                T[p] = test_T;
                if (LOSS == kCountContrib) cnt[p]++;   // a train step's backward needs only the last index
                last[p] = b + (unsigned)k + 1u;
            }
        }
    }
    double lsum = 0.0;
#pragma unroll
    for (int p = 0; p < PPT; p++) {
        const int y = ybase + 2 * p;
        if (x < W && y < H) {
            // 64-bit: a multi-view step holds up to 2^31 pixels, 3 floats each
            const size_t pix = (size_t)sp.pix_base + (size_t)y * W + x;
            const float o0 = C[p][0] + T[p] * sp.cfg.bg_color[0];
            const float o1 = C[p][1] + T[p] * sp.cfg.bg_color[1];
            const float o2 = C[p][2] + T[p] * sp.cfg.bg_color[2];
            px.image[3 * pix] = o0;
            px.image[3 * pix + 1] = o1;
            px.image[3 * pix + 2] = o2;
            if (px.T_final) px.T_final[pix] = T[p];
            if (LOSS == kCountContrib && px.n_contrib) px.n_contrib[pix] = cnt[p];
            if (px.last_j) px.last_j[pix] = last[p];
            if (LOSS == kFusedL1) {
                // loss.cpp:8-14: diff = rendered - gt, sign gradient +-1/n
                const float d0 = o0 - sp.gt[3 * pix], d1 = o1 - sp.gt[3 * pix + 1], d2 = o2 - sp.gt[3 * pix + 2];
                const unsigned sg = (d0 > 0.f ? 1u : (d0 < 0.f ? 2u : 0u)) | (d1 > 0.f ? 4u : (d1 < 0.f ? 8u : 0u)) |
                                    (d2 > 0.f ? 16u : (d2 < 0.f ? 32u : 0u));
                px.dsign[pix] = (unsigned char)sg;
                lsum += (double)fabsf(d0) + (double)fabsf(d1) + (double)fabsf(d2);
            }
        }
    }
    if (LOSS == kFusedL1) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0) s_loss[warp] = lsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < kFwdThreads / 32; w++) t += s_loss[w];
            atomicAdd(&ctrl->loss_sum, MULTI ? t * (double)sp.inv_n : t);
        }
        __syncthreads();
    }
    }
}

// The train step's L1 (loss.cpp:8-14) over a forward image rendered with
// kLossLater: per pixel the sign byte of image - target and the
// double-precision sum |image - target|, as the fused form computes them
// (the sum in a different order: equal to double rounding).  Grid-stride.
__global__ void __launch_bounds__(256) k_l1_loss(const StepParams* __restrict__ spp, PixelPtrs px, size_t n_pix,
                                                 Control* ctrl) {
    __shared__ double s_loss[8];
    const StepParams& sp = *spp;
    double lsum = 0.0;
    for (size_t pix = (size_t)blockIdx.x * blockDim.x + threadIdx.x; pix < n_pix;
         pix += (size_t)gridDim.x * blockDim.x) {
        const float d0 = px.image[3 * pix] - sp.gt[3 * pix], d1 = px.image[3 * pix + 1] - sp.gt[3 * pix + 1],
                    d2 = px.image[3 * pix + 2] - sp.gt[3 * pix + 2];
        const unsigned sg = (d0 > 0.f ? 1u : (d0 < 0.f ? 2u : 0u)) | (d1 > 0.f ? 4u : (d1 < 0.f ? 8u : 0u)) |
                            (d2 > 0.f ? 16u : (d2 < 0.f ? 32u : 0u));
        px.dsign[pix] = (unsigned char)sg;
        lsum += (double)fabsf(d0) + (double)fabsf(d1) + (double)fabsf(d2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((threadIdx.x & 31) == 0) s_loss[threadIdx.x >> 5] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += s_loss[w];
        atomicAdd(&ctrl->loss_sum, t);
    }
}

}  // namespace
}  // namespace gs3d
