// raster_bwd.cu -- Rasterizer backward (rasterizer_backward_cpu.cpp:20-133)
// for sm_100a, plain FP32 form.
//
// Unlike plain.cu this file is compiled with FMA contraction: its outputs are
// gradients, held to a relative tolerance, not bit-exact screen data.  What
// must match the forward exactly -- which (pixel, Gaussian) pairs blended --
// is decided on power_rn (explicit rounding, identical to the forward's value)
// and on alpha_accept_fast below, which agrees with the forward's exact test.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"
#include "raster_common.cuh"

namespace gs3d {
namespace {

// alpha = min(0.99, o exp(power)) and whether it reaches 1/255.  For power in
// [skip_threshold, 0] (|power| < 6) __expf is within 6e-7 relative of exp, so
// o*__expf(power) decides the 1/255 threshold and the 0.99 clamp exactly
// unless it lies within a relative 2e-6 of either bound; there the exact exp
// (exp_ref, the forward's) is recomputed.  Above alpha 0.5 the transmittance
// recovered by dividing by 1 - alpha magnifies alpha's error, so those pairs
// take the accurate expf (a few ulp).  Either way alpha is within the
// gradients' tolerance of the forward's.
__device__ __forceinline__ bool alpha_accept_fast(float power, float o, float& alpha, float& e) {
    e = __expf(power);
    float a = o * e;
    if (fabsf(a - kAlphaMin) <= 2e-6f * kAlphaMin || fabsf(a - 0.99f) <= 2e-6f) {
        e = exp_ref(power);
        a = o * e;
    } else if (a > 0.5f) {
        e = expf(power);
        a = o * e;
    }
    alpha = fmin_ref(0.99f, a);
    return !(alpha < kAlphaMin);
}

// Acceptance policies: the one of the plain form agrees with its exact
// forward; the reduced-storage form's forward decides on o * __expf(power)
// alone, and so does its backward (same power_rn, same __expf, same product).
struct PlainAccept {
    static constexpr bool kBase2 = false;   // the reference's power (power_rn)
    __device__ __forceinline__ static bool accept(float power, float o, float& alpha, float& e) {
        return alpha_accept_fast(power, o, alpha, e);
    }
};
struct FastAccept {
    static constexpr bool kBase2 = true;    // q = power * log2(e) from q_coeffs / q_at, as the forward
    __device__ __forceinline__ static bool accept(float q, float o, float& alpha, float& e) {
        e = ex2_approx(q);
        alpha = fmin_ref(0.99f, o * e);
        return true;   // q passed accept_threshold2, as in the forward
    }
};

// Rasterizer backward (rasterizer_backward_cpu.cpp:20-133): back-to-front
// over each pixel's contributors, transmittance recovered by division from
// T_final instead of a replayed per-pixel list.  One CTA of 256 / PPT threads
// per 16x16 tile, PPT pixels per thread: warp w owns the strip of rows
// 2*PPT*w .. 2*PPT*w + 2*PPT - 1, a thread the pixels (x, 2*PPT*w + lane/16 + 2p).
// A warp walks its compacted list of the batch entries whose alpha >= 1/255
// ellipse reaches its strip (band_rows), from the back.
// Per Gaussian of a batch a thread adds its pixels' contributions, the warp
// sums its 32 * PPT pixels with warp_sum8 + warp_sum, the warps meet in
// shared-memory accumulators and each Gaussian gets one set of global atomics
// per tile.  PPT = 2 by default; the autotuner may pick 1 or 4.
//
// Algebra that keeps the per-pixel work small (same sums, regrouped):
//  - accum_rec (rasterizer_backward_cpu.cpp:101-108) enters d_alpha only as
//    sum_ch accum_rec[ch] * dC[ch], so each pixel carries that one scalar D:
//    d_alpha = T_i (cd - D) with cd = sum_ch c[ch] dC[ch], then D += alpha (cd - D);
//  - d_power = o * d_alpha * exp(power) = u with u = d_alpha * alpha (alpha < 0.99,
//    so alpha = o exp(power)), and the geometric factors
//    of d_means2D / d_conics (:126-132) are polynomials in (dx, dy) with the
//    Gaussian's conic as coefficients, where dx is fixed per thread.  A thread
//    sums u, u dy, u dy^2 over its pixels; the warp reduces u, u dx, u dy,
//    u dx^2, u dx dy, u dy^2 (plus d_rgb) and the conic / opacity factors are
//    applied once per Gaussian when the tile's sums are flushed:
//      d_mean.x = -(a S_x + b S_y)     d_mean.y = -(c S_y + b S_x)
//      d_conic  = -(S_xx / 2, S_xy, S_yy / 2)     d_opacity = S_1 / o.
constexpr int kBwdBatch = 128;

//
// MULTI: one persistent launch over the tiles of several views (spp = the views'
// parameters); a CTA takes the next entry of `order` from a work counter and
// renders the tile with its view's camera and pixel slice.  The screen
// gradients then belong to (view, Gaussian) entries: vals holds view * N + i.
template <bool FROM_SIGN, class Accept, bool MULTI = false, int PPT = 2, int BATCH = kBwdBatch>
__global__ void __launch_bounds__(256 / PPT) k_raster_bwd(const StepParams* __restrict__ spp,
                                                            const unsigned* __restrict__ ranges,
                                                            const unsigned* __restrict__ order,
                                                            const unsigned* __restrict__ vals, ScreenPtrs s,
                                                            PixelPtrs px, RGradPtrs g, Control* ctrl,
                                                            int n_views = 1, unsigned n_tiles = 0) {
    __shared__ float4 s_r0[BATCH];
    __shared__ float4 s_r1[BATCH];
    __shared__ float2 s_bt[BATCH];   // (blue, the forward's threshold): one 8-byte load per Gaussian
    __shared__ unsigned s_idx[BATCH];
    // r, g, b, S_1, S_x, S_y, S_xx, S_xy, S_yy; rows padded by one word so that the
    // eight lanes adding values 0..7 of one Gaussian hit eight different banks
    __shared__ float s_acc[9][BATCH + 1];
    __shared__ unsigned s_maxlast;
    __shared__ unsigned s_next;
    constexpr int kBwdThreads = 256 / PPT;
    constexpr int kNW = kBwdThreads / 32;
    __shared__ unsigned char s_mask[BATCH];       // warps whose strip the Gaussian can reach
    __shared__ unsigned char s_list[kNW][BATCH];  // per warp: its batch entries, ascending
    if (FROM_SIGN && ((ctrl->status & kStatusOverflow) || spp->persist->sticky_overflow)) return;
    for (int iter = 0;; iter++) {
    int tile;
    if (MULTI) {
        if (threadIdx.x == 0) s_next = atomicAdd(&ctrl->work[1], 1u);
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
    const unsigned rs = ranges[2 * tile];
    const float fx = (float)x;
    float fy[PPT], T[PPT], dC[PPT][3], D[PPT];
    unsigned last[PPT];
#pragma unroll
    for (int p = 0; p < PPT; p++) {
        const int y = ybase + 2 * p;
        fy[p] = (float)y;
        T[p] = 0.0f;
        last[p] = 0;
        dC[p][0] = dC[p][1] = dC[p][2] = 0.0f;
        if (x < W && y < H) {
            const size_t pix = (size_t)sp.pix_base + (size_t)y * W + x;   // up to 2^31 pixels, 3 floats each
            T[p] = px.T_final[pix];
            last[p] = px.last_j[pix];
            if (FROM_SIGN) {
                const unsigned sg = px.dsign[pix];
                const float inv_n = sp.inv_n;
                dC[p][0] = (sg & 1u) ? inv_n : ((sg & 2u) ? -inv_n : 0.0f);
                dC[p][1] = (sg & 4u) ? inv_n : ((sg & 8u) ? -inv_n : 0.0f);
                dC[p][2] = (sg & 16u) ? inv_n : ((sg & 32u) ? -inv_n : 0.0f);
            } else {
                dC[p][0] = px.d_image[3 * pix];
                dC[p][1] = px.d_image[3 * pix + 1];
                dC[p][2] = px.d_image[3 * pix + 2];
            }
        }
        D[p] = sp.cfg.bg_color[0] * dC[p][0] + sp.cfg.bg_color[1] * dC[p][1] + sp.cfg.bg_color[2] * dC[p][2];
    }
    if (threadIdx.x == 0) s_maxlast = 0;
    __syncthreads();
    unsigned mylast = 0;
#pragma unroll
    for (int p = 0; p < PPT; p++) mylast = max(mylast, last[p]);
    if (mylast) atomicMax(&s_maxlast, mylast);
    __syncthreads();
    const unsigned maxlast = s_maxlast;
    if (maxlast <= rs) continue;   // uniform: nothing of this tile contributed
    const unsigned wlast = __reduce_max_sync(0xffffffffu, mylast);
    const float wx0 = (float)(tx * kTile), wx1 = wx0 + (float)(kTile - 1), ty0 = (float)(ty * kTile);
    // batches [bs, be) walked from the back; the first one ends at maxlast
    for (unsigned be = maxlast; be > rs;) {
        const unsigned bs = (be - rs > (unsigned)BATCH) ? be - BATCH : rs;
#pragma unroll
        for (int e = threadIdx.x; e < BATCH; e += kBwdThreads) {
            const unsigned j = bs + (unsigned)e;
            if (j < be) {
                const unsigned gi = vals[j];
                float4 r0 = s.rec0[gi];
                float4 r1 = s.rec1[gi];
                const float2 cb = s.cbt[gi];
                const float thr = skip_threshold(cb.y);
                s_idx[e] = gi;
                s_bt[e] = make_float2(cb.x, Accept::kBase2 ? cb.y : thr);   // the forward's
                s_mask[e] = (unsigned char)strip_mask<kNW, 2 * PPT>(band_rows(r0, r1, thr, wx0, wx1), ty0);
                if (Accept::kBase2) q_scale(r0, r1);   // as the forward stages it
                s_r0[e] = r0;
                s_r1[e] = r1;
            }
#pragma unroll
            for (int v = 0; v < 9; v++) s_acc[v][e] = 0.0f;
        }
        __syncthreads();
        // this warp only needs the entries below its own last contributor
        const int kstart = (int)(min(be, wlast) - min(bs, wlast)) - 1;
        const int nl = warp_list(s_mask, kstart + 1, warp, s_list[warp]);
        // this thread's contributions to batch entry k (walked back to front): gv = d_rgb and the
        // moments S_1, S_x, S_y, S_xx, S_xy of its pixels, t2 = S_yy; returns whether any pixel blended
        auto item = [&](int k, float gv[8], float& s_yy) -> bool {
            const unsigned jj = bs + (unsigned)k;
            const float4 a = s_r0[k];
            const float4 c = s_r1[k];
            const float2 bt = s_bt[k];
            const float cb = bt.x, thr = bt.y;
            const float dx = a.x - fx;
            const float3 kq = Accept::kBase2 ? q_coeffs(a, c, dx) : make_float3(0.f, 0.f, 0.f);
            bool contrib = false;
            float gr = 0.f, gg = 0.f, gb = 0.f;     // d_rgb
            float t0 = 0.f, t1 = 0.f, t2 = 0.f;     // sum of t, t dy, t dy^2 over this thread's pixels
#pragma unroll
            for (int p = 0; p < PPT; p++) {
                if (jj < last[p]) {
                    const float dy = a.y - fy[p];
                    const float power = Accept::kBase2 ? q_at(kq, dy) : power_rn(a, c, dx, dy);
                    float alpha, ep;
                    const bool in_range = Accept::kBase2 ? power >= thr : !(power < thr) && !(power > 0.0f);
                    if (in_range && Accept::accept(power, c.y, alpha, ep)) {
                        contrib = true;
                        // alpha <= 0.99, so 1 - alpha >= 0.01 passes the reference's 1e-6 guard (:84-85)
                        const float Ti = __fdividef(T[p], 1.0f - alpha);
                        const float aT = alpha * Ti;
                        gr += aT * dC[p][0];
                        gg += aT * dC[p][1];
                        gb += aT * dC[p][2];
                        const float cd = c.z * dC[p][0] + c.w * dC[p][1] + cb * dC[p][2];
                        const float diff = cd - D[p];
                        D[p] += alpha * diff;
                        T[p] = Ti;
                        if (alpha < 0.99f) {
                            // d_alpha * alpha = o * (d_alpha * exp(power)): o is divided out at the flush
                            const float t = diff * aT;
                            t0 += t;
                            const float tdy = t * dy;
                            t1 += tdy;
                            t2 += tdy * dy;
                        }
                    }
                }
            }
            const float tx0 = t0 * dx;
            gv[0] = gr;
            gv[1] = gg;
            gv[2] = gb;
            gv[3] = t0;
            gv[4] = tx0;
            gv[5] = t1;
            gv[6] = tx0 * dx;
            gv[7] = t1 * dx;
            s_yy = t2;
            return contrib;
        };
        for (int i = nl - 1; i >= 0; i--) {
            const int k = s_list[warp][i];
            float gv[8], t2;
            if (__any_sync(0xffffffffu, item(k, gv, t2))) {
                int idx;
                const float s8 = warp_sum8(gv, &idx);
                const float s9 = warp_sum(t2);
                if ((lane & 3) == 0 && s8 != 0.0f) atomicAdd(&s_acc[idx][k], s8);
                if (lane == 1 && s9 != 0.0f) atomicAdd(&s_acc[8][k], s9);
            }
        }
        __syncthreads();
#pragma unroll
        for (int e = threadIdx.x; e < BATCH; e += kBwdThreads) {
            if (bs + (unsigned)e < be) {
                const size_t gi = s_idx[e];   // (view, Gaussian) entry: 3 * gi can pass 2^32
                float* const dst[9] = {&g.drgb[3 * gi], &g.drgb[3 * gi + 1], &g.drgb[3 * gi + 2], &g.dop[gi],
                                       &g.dm2[2 * gi], &g.dm2[2 * gi + 1], &g.dcon[3 * gi], &g.dcon[3 * gi + 1],
                                       &g.dcon[3 * gi + 2]};
                const float4 r0 = s_r0[e];
                const float o = s_r1[e].y, cc = s_r1[e].x;
                const float Sx = s_acc[4][e], Sy = s_acc[5][e];
                // d_mean = -(a S_x + b S_y, c S_y + b S_x); from the pre-scaled conic
                // (-a L / 2, -b L, -c L / 2), L = log2(e): (1 / L) (2 A S_x + B S_y, 2 H S_y + B S_x)
                const float dmx = Accept::kBase2 ? (1.0f / kLog2e) * (2.0f * r0.z * Sx + r0.w * Sy)
                                                 : -(r0.z * Sx + r0.w * Sy);
                const float dmy = Accept::kBase2 ? (1.0f / kLog2e) * (2.0f * cc * Sy + r0.w * Sx)
                                                 : -(cc * Sy + r0.w * Sx);
                const float val[9] = {s_acc[0][e], s_acc[1][e], s_acc[2][e], __fdividef(s_acc[3][e], o), dmx, dmy,
                                      -0.5f * s_acc[6][e], -s_acc[7][e], -0.5f * s_acc[8][e]};
#pragma unroll
                for (int v = 0; v < 9; v++)
                    if (val[v] != 0.0f) atomicAdd(dst[v], val[v]);
            }
        }
        __syncthreads();
        be = bs;
    }
    }
}

// ---- stored-list variant (memory comparison only) ----
// The reference holds each pixel's contributors as a list: its CPU backward
// replays the forward into a per-pixel vector of (Gaussian, alpha)
// (rasterizer_backward_cpu.cpp:40-67) and its OpenCL kernel into private arrays
// of up to 128 entries (rasterize_backward.cl:79-121), then walks the list back
// to front.  k_list_fill / k_list_bwd do the same with the lists in one device
// buffer (entry offsets = exclusive scan of n_contrib), so that their memory
// can be measured against the recompute backward above, which keeps no list.
// One thread per pixel, no staging: these kernels are not on the train step.
__global__ void __launch_bounds__(256) k_list_fill(const StepParams* __restrict__ spp,
                                                   const unsigned* __restrict__ ranges,
                                                   const unsigned* __restrict__ vals, ScreenPtrs s,
                                                   const int* __restrict__ n_contrib, const int* __restrict__ offset,
                                                   uint2* __restrict__ list) {
    const StepParams& sp = *spp;
    const int tile = blockIdx.x;
    const int tx = tile % sp.grid_x, ty = tile / sp.grid_x;
    const int x = tx * kTile + (int)(threadIdx.x & 15), y = ty * kTile + (int)(threadIdx.x >> 4);
    if (x >= sp.cam.width || y >= sp.cam.height) return;
    const size_t pix = (size_t)y * sp.cam.width + x;
    const int n = n_contrib[pix];
    uint2* out = list + offset[pix];
    const float fx = (float)x, fy = (float)y;
    float T = 1.0f;
    int c = 0;
    for (unsigned j = ranges[2 * tile]; j < ranges[2 * tile + 1] && c < n; j++) {
        const unsigned g = vals[j];
        const float4 r0 = s.rec0[g], r1 = s.rec1[g];
        const float power = power_rn(r0, r1, __fsub_rn(r0.x, fx), __fsub_rn(r0.y, fy));
        if (power > 0.0f) continue;
        const float alpha = fmin_ref(0.99f, __fmul_rn(r1.y, exp_ref(power)));   // the forward's exact alpha
        if (alpha < kAlphaMin) continue;
        const float test_T = __fmul_rn(T, __fsub_rn(1.0f, alpha));
        if (test_T < kTMin) break;
        out[c++] = make_uint2(g, __float_as_uint(alpha));
        T = test_T;
    }
}

// RasterizerBackwardCPU::backward's back-to-front walk
// (rasterizer_backward_cpu.cpp:69-133) over a pixel's stored list, with the
// explicit image gradient d_image; nine atomics per (pixel, contributor).
__global__ void __launch_bounds__(256) k_list_bwd(const StepParams* __restrict__ spp, ScreenPtrs s, PixelPtrs px,
                                                  const int* __restrict__ offset, const uint2* __restrict__ list,
                                                  RGradPtrs g) {
    const StepParams& sp = *spp;
    const int tile = blockIdx.x;
    const int tx = tile % sp.grid_x, ty = tile / sp.grid_x;
    const int x = tx * kTile + (int)(threadIdx.x & 15), y = ty * kTile + (int)(threadIdx.x >> 4);
    if (x >= sp.cam.width || y >= sp.cam.height) return;
    const size_t pix = (size_t)y * sp.cam.width + x;
    const int n = px.n_contrib[pix];
    if (n == 0) return;
    const uint2* in = list + offset[pix];
    const float dC[3] = {px.d_image[3 * pix], px.d_image[3 * pix + 1], px.d_image[3 * pix + 2]};
    float T = px.T_final[pix];
    float acc[3] = {sp.cfg.bg_color[0], sp.cfg.bg_color[1], sp.cfg.bg_color[2]};
    for (int i = n - 1; i >= 0; i--) {
        const unsigned gi = in[i].x;
        const float alpha = __uint_as_float(in[i].y);
        const float oma = 1.0f - alpha;
        const float Ti = oma > 1e-6f ? T / oma : 0.0f;
        const float4 r0 = s.rec0[gi], r1 = s.rec1[gi];
        const float col[3] = {r1.z, r1.w, s.cbt[gi].x};
        const float dx = r0.x - (float)x, dy = r0.y - (float)y;
        float d_alpha = 0.0f;
#pragma unroll
        for (int ch = 0; ch < 3; ch++) {
            atomicAdd(&g.drgb[3 * (size_t)gi + ch], alpha * Ti * dC[ch]);
            d_alpha += Ti * (col[ch] - acc[ch]) * dC[ch];
            acc[ch] = alpha * col[ch] + oma * acc[ch];
        }
        T = Ti;
        if (alpha < 0.99f) {
            const float e = expf(-0.5f * (r0.z * dx * dx + r1.x * dy * dy) - r0.w * dx * dy);
            const float d_power = d_alpha * r1.y * e;
            atomicAdd(&g.dop[gi], d_alpha * e);
            atomicAdd(&g.dm2[2 * (size_t)gi], d_power * (-r0.z * dx - r0.w * dy));
            atomicAdd(&g.dm2[2 * (size_t)gi + 1], d_power * (-r1.x * dy - r0.w * dx));
            atomicAdd(&g.dcon[3 * (size_t)gi], d_power * (-0.5f * dx * dx));
            atomicAdd(&g.dcon[3 * (size_t)gi + 1], d_power * (-dx * dy));
            atomicAdd(&g.dcon[3 * (size_t)gi + 2], d_power * (-0.5f * dy * dy));
        }
    }
}

}  // namespace

cudaError_t launch_list_fill(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                             const unsigned* vals, ScreenPtrs s, const int* n_contrib, const int* offset,
                             uint2* list) {
    if (num_tiles <= 0) return cudaSuccess;
    k_list_fill<<<num_tiles, 256, 0, st>>>(sp, ranges, vals, s, n_contrib, offset, list);
    return cudaGetLastError();
}

cudaError_t launch_list_bwd(cudaStream_t st, const StepParams* sp, int num_tiles, ScreenPtrs s, PixelPtrs px,
                            const int* offset, const uint2* list, RGradPtrs g) {
    if (num_tiles <= 0) return cudaSuccess;
    k_list_bwd<<<num_tiles, 256, 0, st>>>(sp, s, px, offset, list, g);
    return cudaGetLastError();
}

namespace {

// Resident CTAs per SM of a kernel at its block size (persistent launches).
template <class F>
int resident_ctas(F kernel, int threads) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

}  // namespace

cudaError_t launch_raster_bwd_plain(cudaStream_t st, const StepParams* sp, int num_tiles, bool from_sign,
                                    const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                    ScreenPtrs s, PixelPtrs px, RGradPtrs g, Control* ctrl, int ppt, int batch) {
    if (num_tiles <= 0) return cudaSuccess;
    if (!from_sign) batch = 128;   // the stage API (explicit d_image)
    return with_ppt_batch(ppt, batch, [&](auto P, auto Bt) {
        constexpr int kP = decltype(P)::value, kB = decltype(Bt)::value;
        if (from_sign)
            k_raster_bwd<true, PlainAccept, false, kP, kB><<<num_tiles, 256 / kP, 0, st>>>(sp, ranges, order, vals, s,
                                                                                          px, g, ctrl);
        else
            k_raster_bwd<false, PlainAccept, false, kP, kBwdBatch><<<num_tiles, 256 / kP, 0, st>>>(
                sp, ranges, order, vals, s, px, g, ctrl);
        return cudaGetLastError();
    });
}

cudaError_t launch_raster_bwd_fast(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                                   const unsigned* order, const unsigned* vals, ScreenPtrs s, PixelPtrs px,
                                   RGradPtrs g, Control* ctrl, int ppt, int batch) {
    if (num_tiles <= 0) return cudaSuccess;
    return with_ppt_batch(ppt, batch, [&](auto P, auto Bt) {
        constexpr int kP = decltype(P)::value, kB = decltype(Bt)::value;
        k_raster_bwd<true, FastAccept, false, kP, kB><<<num_tiles, 256 / kP, 0, st>>>(sp, ranges, order, vals, s, px,
                                                                                      g, ctrl);
        return cudaGetLastError();
    });
}

cudaError_t launch_raster_bwd_fast_multi(cudaStream_t st, const StepParams* views, int n_views, unsigned n_tiles,
                                         const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                         ScreenPtrs s, PixelPtrs px, RGradPtrs g, Control* ctrl, int ppt, int batch) {
    if (n_tiles == 0) return cudaSuccess;
    // persistent: as many CTAs as fit resident
    return with_ppt_batch(ppt, batch, [&](auto P, auto Bt) {
        constexpr int kP = decltype(P)::value, kB = decltype(Bt)::value;
        static int per_sm = 0;
        if (!per_sm) per_sm = resident_ctas(k_raster_bwd<true, FastAccept, true, kP, kB>, 256 / kP);
        k_raster_bwd<true, FastAccept, true, kP, kB><<<per_sm * sm_count(), 256 / kP, 0, st>>>(
            views, ranges, order, vals, s, px, g, ctrl, n_views, n_tiles);
        return cudaGetLastError();
    });
}

}  // namespace gs3d
