// plain.cu -- plain-FP32 form of the 3DGS hot path for sm_100a.
//
// Compiled with -fmad=false and IEEE division / square root so that every
// float operation rounds like the reference's x86 build with
// -ffp-contract=off (harmonyos_3dgs CMakeLists.txt:19); the operation order
// below follows the reference's CPU stages line by line, which is what makes
// depths, radii, tile counts, keys, sorted order and tile ranges bit-exact.
//
// Kernels:
//   k_preprocess    one thread per Gaussian: (activation) -> projection ->
//                   EWA covariance -> conic / radius / tile rect -> SH colour,
//                   then a block scan + decoupled look-back over tiles_touched
//                   and a block-cooperative emission of (tile|depth, index)
//                   pairs.  Replaces preprocess + prefix sum + binning.
//   k_bin_arrays    the same scan + emission from host-provided screen arrays.
//   k_raster_fwd    one CTA per 16x16 tile, one thread per pixel; pairs are
//                   gathered in batches of 128 into shared memory; CTA-wide
//                   early exit once every pixel saturated.  Optional fused L1.
//   (k_raster_bwd lives in raster_bwd.cu, compiled with FMA contraction.)
//   k_preprocess_bwd  the full per-Gaussian adjoint chain, fused with Adam.
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "common.cuh"
#include "kernels.cuh"
#include "raster_common.cuh"
#include "ref_math.cuh"

namespace gs3d {
namespace {

// Alpha / transmittance decisions of the front-to-back blend
// (rasterizer_cpu.cpp:149-166).  A Gaussian that is clearly below the alpha
// threshold is skipped on the fast exp alone; every other evaluation --
// near the threshold, or accepted -- recomputes exp correctly
// rounded, so alpha, the transmittance chain T and the stop decision follow
// the reference's glibc-based values (they differ only where glibc's expf is
// itself 1 ulp off, ~0.006% of inputs).
// Returns 0 = skip, 1 = blend, 2 = stop (transmittance would saturate).
__device__ __forceinline__ int blend_decision(float power, float o, float T, float& alpha, float& e,
                                              float& test_T) {
    // screening on the fast exp: for power in [skip_threshold, 0] (|power| < 6)
    // __expf is within 6e-7 relative of exp, far inside the 4e-6 band kept here
    if (o * __expf(power) < kAlphaMin * (1.0f - 4e-6f)) return 0;
    e = exp_ref(power);
    alpha = fmin_ref(0.99f, o * e);
    if (alpha < kAlphaMin) return 0;
    test_T = T * (1.0f - alpha);
    if (test_T < kTMin) return 2;
    return 1;
}

// The plain form's blend decision for the shared forward kernel.
struct ExactBlend {
    static constexpr bool kBase2 = false;   // decides on the reference's power (power_rn)
    __device__ __forceinline__ static int decide(float power, float o, float T, float& alpha, float& e,
                                                 float& test_T) {
        return blend_decision(power, o, T, alpha, e, test_T);
    }
};

}  // namespace
}  // namespace gs3d

#include "raster_fwd.cuh"

namespace gs3d {
namespace {

// ---------------- block scan + look-back + pair emission ----------------

constexpr int kEmitRun = 4;                      // consecutive pair slots walked by one thread
constexpr int kEmitBlock = 512;                  // CTA of the train step's pair emission (k_emit_ranked)
constexpr unsigned kNoPair = 0xffffffffu;        // staged tile of a slot left unwritten (beyond `limit`)

// Shared memory of a CTA of B threads (one Gaussian each) emitting its pairs.
template <int B = kBlock>
struct EmitShared {
    static constexpr int kChunk = B * kEmitRun;   // pair slots staged per round
    int warp[B / 32];
    int excl[B];
    int rect[B];      // xmin | ymin << 16
    int width[B];
    float winv[B];    // 1 / width (round to nearest): the row of a pair without an integer division
    int limit[B];     // pairs actually emitted (rect area, <= count)
    unsigned depth[B];
    unsigned gid[B];  // Gaussian index written as the pair's value
    unsigned tbase[B];  // first global tile id of the Gaussian's view (0 for one view)
    int gx[B];          // tile-grid width of the Gaussian's view
    alignas(16) unsigned ctile[kChunk];   // one round's pairs: tile id (or kNoPair)
    alignas(16) unsigned cown[kChunk];    // and the owning thread of the CTA
    unsigned long long base;
};

// Scans cnt over the CTA, finds the CTA's global offset by decoupled
// look-back and writes the CTA's pairs with consecutive threads writing
// consecutive pairs (fully coalesced, balanced however uneven the rects).
// Pair order: Gaussian-major, then row-major inside the rect
// (tile_binner_cpu.cpp:90-97).
// The pairs go out in rounds of EmitShared<B>::kChunk slots (B = the CTA's
// threads): each thread finds the owner
// of its first kEmitRun consecutive slots by one binary search over the
// CTA's exclusive scan and walks them (column, row and owner advance by
// increments), staging tile and owner in shared memory; then the CTA writes
// the round with consecutive threads on consecutive slots.  The CTA's
// aggregate is published before the first round is staged, so the look-back
// (warp 0, after its staging) usually finds its predecessors' prefixes ready.
// With pr.tiles32 set, writes tile-only keys and counts the first nd 8-bit
// digits of every tile into thist[nd][256] (shared memory).
//
// DepthFn(dbits, gid, tile) gives the low 32 key bits of each pair: the
// Gaussian's depth bits here, a depth per tile in the 3D-evaluation mode.
struct KeepDepth {
    __device__ __forceinline__ unsigned operator()(unsigned dbits, unsigned, unsigned) const { return dbits; }
};

template <int B = kBlock, class DepthFn = KeepDepth>
__device__ __forceinline__ void scan_and_emit(EmitShared<B>& sm, int blk, unsigned gid, int cnt, int emit, int rx, int ry,
                                              int rw, unsigned dbits, int grid_x, PairPtrs pr,
                                              Control* ctrl, unsigned spin_limit, Persist* persist,
                                              unsigned* thist = nullptr, int nd = 0, unsigned tile_base_t = 0u,
                                              int grid_x_t = -1, DepthFn depth_fn = DepthFn()) {
    const int tid = threadIdx.x;
    int total;
    const int incl = block_inclusive_scan<B / 32>(cnt, sm.warp, &total);
    sm.excl[tid] = incl - cnt;
    sm.rect[tid] = rx | (ry << 16);
    sm.width[tid] = rw;
    sm.winv[tid] = 1.0f / (float)rw;
    sm.limit[tid] = emit;
    sm.depth[tid] = dbits;
    sm.gid[tid] = gid;
    sm.tbase[tid] = tile_base_t;
    sm.gx[tid] = grid_x_t < 0 ? grid_x : grid_x_t;
    if (tid == 0) lookback_publish(pr.scan_desc, blk, (unsigned long long)total);
    __syncthreads();
    for (int c0 = 0;; c0 += EmitShared<B>::kChunk) {
        // stage this round: slots c0 + kEmitRun * tid ..
        const int k0 = c0 + kEmitRun * tid;
        if (k0 < total) {
            int lo = 0, hi = B;   // the owner: last thread whose exclusive offset is <= k0
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (sm.excl[mid] <= k0) lo = mid;
                else hi = mid;
            }
            int local = k0 - sm.excl[lo];
            int end = lo + 1 < B ? sm.excl[lo + 1] : total;
            int w = sm.width[lo], lim = sm.limit[lo], gx = sm.gx[lo];
            // local / w from the rounded reciprocal: for local < 2^23 the product is within one of the
            // quotient, and one correction step each way makes it exact
            int row = __float2int_rz((float)local * sm.winv[lo]);
            if ((row + 1) * w <= local) row++;
            else if (row * w > local) row--;
            int col = local - row * w;
            int r = sm.rect[lo];
            unsigned tile = sm.tbase[lo] + (unsigned)(((r >> 16) + row) * gx + (r & 0xffff) + col);
            unsigned st[kEmitRun], so[kEmitRun];
#pragma unroll
            for (int i = 0; i < kEmitRun; i++) {
                const int k = k0 + i;
                if (k < total && k == end) {   // next thread with pairs
                    do {
                        lo++;
                        end = lo + 1 < B ? sm.excl[lo + 1] : total;
                    } while (end == k);
                    local = 0;
                    col = 0;
                    w = sm.width[lo];
                    lim = sm.limit[lo];
                    gx = sm.gx[lo];
                    r = sm.rect[lo];
                    tile = sm.tbase[lo] + (unsigned)((r >> 16) * gx + (r & 0xffff));
                }
                st[i] = local < lim ? tile : kNoPair;
                so[i] = (unsigned)lo;
                local++;
                tile++;
                if (++col == w) {
                    col = 0;
                    tile += (unsigned)(gx - w);
                }
            }
            *reinterpret_cast<uint4*>(&sm.ctile[kEmitRun * tid]) = make_uint4(st[0], st[1], st[2], st[3]);
            *reinterpret_cast<uint4*>(&sm.cown[kEmitRun * tid]) = make_uint4(so[0], so[1], so[2], so[3]);
        }
        if (c0 == 0 && tid < 32) {
            const unsigned long long ex =
                warp_lookback_walk(pr.scan_desc, blk, (unsigned long long)total, &ctrl->status, spin_limit);
            if (tid == 0) {
                sm.base = ex;
                if (blk == (int)gridDim.x - 1) ctrl->total_pairs = ex + (unsigned long long)total;
                if (ex + (unsigned long long)total > pr.capacity) {
                    atomicOr(&ctrl->status, kStatusOverflow);
                    if (persist) atomicOr(&persist->sticky_overflow, 1u);
                }
            }
        }
        __syncthreads();
        const unsigned long long base = sm.base;
        const int n = min(EmitShared<B>::kChunk, total - c0);
        for (int j = tid; j < n; j += B) {
            const unsigned tile = sm.ctile[j];
            const unsigned long long dst = base + (unsigned long long)(c0 + j);
            if (tile == kNoPair || dst >= pr.capacity) continue;
            const unsigned own = sm.cown[j];
            if (pr.tiles32) {
                pr.tiles32[dst] = tile;
                for (int d = 0; d < nd; d++) atomicAdd(&thist[d * 256 + ((tile >> (8 * d)) & 255u)], 1u);
            } else {
                pr.keys[dst] = ((unsigned long long)tile << 32) | depth_fn(sm.depth[own], sm.gid[own], tile);
            }
            pr.vals[dst] = sm.gid[own];
        }
        if (c0 + EmitShared<B>::kChunk >= total) break;
        __syncthreads();   // the next round restages the buffers
    }
}

// ---------------- kernels ----------------

template <bool TRAIN, bool CACHE, bool EMIT>
__global__ void __launch_bounds__(kBlock) k_preprocess(const StepParams* __restrict__ spp, int N, ModelPtrs m,
                                                       ScreenPtrs s, PairPtrs pr, DepthKeys dk, Control* ctrl) {
    __shared__ EmitShared<> sm;
    __shared__ int s_blk;
    const StepParams& sp = *spp;
    if (EMIT) {
        if (threadIdx.x == 0) s_blk = (int)atomicAdd(&ctrl->tickets[0], 1u);
        __syncthreads();
    }
    const int blk = EMIT ? s_blk : (int)blockIdx.x;
    const int i = blk * kBlock + threadIdx.x;
    int cnt = 0, rx = 0, ry = 0, rw = 1;
    unsigned dbits = 0;
    if (i < N) {
        const int mc3 = sp.max_coeffs * 3;
        const float p[3] = {m.pos[3 * i], m.pos[3 * i + 1], m.pos[3 * i + 2]};
        float sc[3], q[4], op;
        if (TRAIN) {
            const float rsc[3] = {m.sc[3 * i], m.sc[3 * i + 1], m.sc[3 * i + 2]};
            const float rq[4] = {m.rot[4 * i], m.rot[4 * i + 1], m.rot[4 * i + 2], m.rot[4 * i + 3]};
            activate_one(rsc, rq, m.op[i], sc, q, &op);
        } else {
#pragma unroll
            for (int k = 0; k < 3; k++) sc[k] = m.sc[3 * i + k];
#pragma unroll
            for (int k = 0; k < 4; k++) q[k] = m.rot[4 * i + k];
            op = m.op[i];
        }
        Proj r;
        const float* shrow = m.sh + (size_t)mc3 * i;
        bool vis;
        if (mc3 == 48) {
            // degree-3 storage: the 192-byte row (16-byte aligned) as twelve 16-byte loads
            float4 shv[12];
#pragma unroll
            for (int k = 0; k < 12; k++) shv[k] = reinterpret_cast<const float4*>(shrow)[k];
            vis = project_one(sp, p, sc, q, op, reinterpret_cast<const float*>(shv), r);
        } else {
            vis = project_one(sp, p, sc, q, op, shrow, r);
        }
        if (vis) {
            cnt = (r.rmx[1] - r.rmn[1]) * (r.rmx[0] - r.rmn[0]);
            rx = r.rmn[0];
            ry = r.rmn[1];
            rw = r.rmx[0] - r.rmn[0];
            dbits = __float_as_uint(r.depth);
            s.rec0[i] = make_float4(r.px, r.py, r.con[0], r.con[1]);
            s.rec1[i] = make_float4(r.con[2], r.opac, r.rgb[0], r.rgb[1]);
            s.cbt[i] = blue_thr(r.rgb[2], r.opac);
            s.depth[i] = r.depth;
            s.radius[i] = r.radius;
        } else {
            s.rec0[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            s.rec1[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            s.cbt[i] = blue_thr(0.f, 0.f);
            s.depth[i] = 0.f;
            s.radius[i] = 0;
        }
        s.tiles[i] = cnt;
        if (CACHE) {
#pragma unroll
            for (int k = 0; k < 6; k++) s.cov3D[6 * i + k] = vis ? r.cov3[k] : 0.f;
#pragma unroll
            for (int k = 0; k < 3; k++) s.p_view[3 * i + k] = vis ? r.pv[k] : 0.f;
            s.p_hom_w[i] = vis ? r.phw : 0.f;
#pragma unroll
            for (int k = 0; k < 3; k++) s.cov2D[3 * i + k] = vis ? r.cov2[k] : 0.f;
            s.det[i] = vis ? r.det : 0.f;
        }
    }
    if (EMIT) {
        scan_and_emit(sm, blk, (unsigned)i, cnt, cnt, rx, ry, rw, dbits, sp.grid_x, pr, ctrl, sp.spin_limit,
                      sp.persist);
    } else if (i < N) {
        // depth-sort input: Gaussians without pairs sort last (no finite depth has these bits)
        dk.keys[i] = cnt > 0 ? dbits : 0xFFFFFFFFu;
        dk.vals[i] = (unsigned)i;
        if (dk.rects)   // the emission reads the rectangle (and its area, the pair count) in one load
            dk.rects[i] = cnt > 0 ? make_uint2((unsigned)rx | ((unsigned)ry << 16),
                                               (unsigned)(rx + rw) | ((unsigned)(ry + cnt / rw) << 16))
                                  : make_uint2(0u, 0u);
        if (i == 0) ctrl->gauss_keys = (unsigned long long)N;
    }
}

// Pair emission in depth order: thread r takes the Gaussian of depth rank r,
// recomputes its tile rectangle from the stored mean and radius (the same
// tile_rect the preprocess used) and emits its pairs row-major.  With the
// Gaussians stably sorted by depth bits, a stable sort of these pairs by tile
// alone gives the (tile, depth bits, Gaussian index) order of the full-key sort.
template <int B>
__global__ void __launch_bounds__(B) k_emit_ranked(const StepParams* __restrict__ spp, int N,
                                                   const unsigned* __restrict__ rank_gid, ScreenPtrs s,
                                                   PairPtrs pr, const uint2* __restrict__ rects,
                                                   Control* ctrl, int n_per_view, int hist_slot,
                                                   unsigned* __restrict__ hist_parts) {
    __shared__ EmitShared<B> sm;
    __shared__ int s_blk;
    __shared__ unsigned s_thist[kMaxPasses - kDepthDigits][256];
    const StepParams& sp = *spp;
    const int nd = sp.sort_passes - kDepthDigits;   // 8-bit digits of the tile ids (control slots hist_slot..)
    for (int e = threadIdx.x; e < nd * 256; e += B) (&s_thist[0][0])[e] = 0;
    if (threadIdx.x == 0) s_blk = (int)atomicAdd(&ctrl->tickets[0], 1u);
    __syncthreads();
    const int blk = s_blk;
    const int r = blk * B + threadIdx.x;
    int cnt = 0, rx = 0, ry = 0, rw = 1, gx = sp.grid_x;
    unsigned g = 0, dbits = 0, tbase = 0;
    if (r < N) {
        g = rank_gid[r];
    }
    if (r < N && g != 0xFFFFFFFFu) {   // several views: 0xFFFFFFFF is the padding of a view's sort segment
        if (n_per_view > 0) {
            // several views: entry g = view * n_per_view + Gaussian, spp is the views' parameter array;
            // the key is the view's local tile id, with the view above the nd sorted digits
            const unsigned view = g / (unsigned)n_per_view;
            gx = spp[view].grid_x;
            tbase = view << (8 * nd);
        }
        if (rects) {
            // tile rectangle stored by the preprocess: (xmin | ymin << 16, xmax | ymax << 16); its
            // area is the Gaussian's pair count (0 without pairs)
            const uint2 rc = rects[g];
            rx = (int)(rc.x & 0xffffu);
            ry = (int)(rc.x >> 16);
            rw = (int)(rc.y & 0xffffu) - rx;
            cnt = rw * ((int)(rc.y >> 16) - ry);
            if (cnt <= 0) {
                cnt = 0;
                rw = 1;
            }
        } else {
            cnt = s.tiles[g];
            if (cnt > 0) {
                const float4 r0 = s.rec0[g];
                int rmn[2], rmx[2];
                tile_rect(r0.x, r0.y, s.radius[g], sp.grid_x, sp.grid_y, sp.cfg.tile_w, sp.cfg.tile_h, rmn, rmx);
                rx = rmn[0];
                ry = rmn[1];
                rw = rmx[0] - rmn[0];
            }
        }
        // the depth goes into 64-bit keys only; tile-only keys do not carry it
        if (cnt > 0 && !pr.tiles32) dbits = __float_as_uint(s.depth[g]);
    }
    scan_and_emit(sm, blk, g, cnt, cnt, rx, ry, rw, dbits, sp.grid_x, pr, ctrl, sp.spin_limit, sp.persist,
                  &s_thist[0][0], nd, tbase, gx);
    __syncthreads();
    // many CTAs (several views): spread the counts over kHistParts copies so that the atomics of
    // different CTAs rarely meet on one address; k_hist_parts_reduce adds the copies up
    unsigned* dst = hist_parts ? hist_parts + (size_t)(blk % kHistParts) * (kMaxPasses - kDepthDigits) * 256
                               : &ctrl->hist[hist_slot][0];
    for (int e = threadIdx.x; e < nd * 256; e += B) {
        const unsigned v = (&s_thist[0][0])[e];
        if (v) atomicAdd(&dst[e], v);
    }
}

// Sums the kHistParts copies of the tile-digit counts into the control
// block's histogram slots hist_slot.. (one CTA; the copies are zeroed with the
// other per-step scratch).
__global__ void __launch_bounds__(256) k_hist_parts_reduce(const unsigned* __restrict__ hist_parts,
                                                           const StepParams* __restrict__ spp, Control* ctrl,
                                                           int hist_slot) {
    const int nd = spp->sort_passes - kDepthDigits;
    for (int e = threadIdx.x; e < nd * 256; e += blockDim.x) {
        unsigned v = 0;
        for (int p = 0; p < kHistParts; p++) v += hist_parts[(size_t)p * (kMaxPasses - kDepthDigits) * 256 + e];
        ctrl->hist[hist_slot + (e >> 8)][e & 255] = v;
    }
}

// TileBinner::bin over host-provided screen arrays (tile_binner_cpu.cpp:33-99):
// offsets from tiles_touched, pairs from the rect recomputed from (mean, radius).
__global__ void __launch_bounds__(kBlock) k_bin_arrays(const StepParams* __restrict__ spp, int N,
                                                       ScreenArrays a, PairPtrs pr, Control* ctrl) {
    __shared__ EmitShared<> sm;
    __shared__ int s_blk;
    const StepParams& sp = *spp;
    if (threadIdx.x == 0) s_blk = (int)atomicAdd(&ctrl->tickets[0], 1u);
    __syncthreads();
    const int blk = s_blk;
    const int i = blk * kBlock + threadIdx.x;
    int cnt = 0, emit = 0, rx = 0, ry = 0, rw = 1;
    unsigned dbits = 0;
    if (i < N) {
        cnt = a.tiles[i];
        if (a.radii[i] > 0) {
            int rmn[2], rmx[2];
            tile_rect(a.means2D[2 * i], a.means2D[2 * i + 1], a.radii[i], sp.grid_x, sp.grid_y,
                      sp.cfg.tile_w, sp.cfg.tile_h, rmn, rmx);
            rx = rmn[0];
            ry = rmn[1];
            rw = max(1, rmx[0] - rmn[0]);
            emit = min(cnt, (rmx[0] - rmn[0]) * (rmx[1] - rmn[1]));
            dbits = __float_as_uint(a.depths[i]);
        }
    }
    scan_and_emit(sm, blk, (unsigned)i, cnt, emit, rx, ry, rw, dbits, sp.grid_x, pr, ctrl, sp.spin_limit, nullptr);
}

// Unpacks the screen records into PreprocessOutput's layout.
__global__ void k_export_screen(int N, ScreenPtrs s, ScreenArrays a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 r0 = s.rec0[i], r1 = s.rec1[i];
    a.means2D[2 * i] = r0.x;
    a.means2D[2 * i + 1] = r0.y;
    a.conics[3 * i] = r0.z;
    a.conics[3 * i + 1] = r0.w;
    a.conics[3 * i + 2] = r1.x;
    a.opac2d[i] = r1.y;
    a.rgb[3 * i] = r1.z;
    a.rgb[3 * i + 1] = r1.w;
    a.rgb[3 * i + 2] = s.cbt[i].x;
    a.depths[i] = s.depth[i];
    a.radii[i] = s.radius[i];
    a.tiles[i] = s.tiles[i];
}


// The inverse: PreprocessOutput arrays of a caller (screen means, conics,
// opacities, colours) packed into the screen records the rasterisers read.
__global__ void k_import_screen(int N, ScreenArrays a, ScreenPtrs s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    s.rec0[i] = make_float4(a.means2D[2 * i], a.means2D[2 * i + 1], a.conics[3 * i], a.conics[3 * i + 1]);
    s.rec1[i] = make_float4(a.conics[3 * i + 2], a.opac2d[i], a.rgb[3 * i], a.rgb[3 * i + 1]);
    s.cbt[i] = blue_thr(a.rgb[3 * i + 2], a.opac2d[i]);
}

// ---- fused preprocess backward + optimiser, staged by TMA into shared memory ----
//
// One CTA owns kBwdG consecutive Gaussians.  A single thread issues TMA bulk
// copies (cp.async.bulk) of the CTA's slices of every parameter array, of the
// screen-space gradients and of the radii onto mbarrier A, and of the Adam
// moments onto mbarrier B.  The CTA waits on A, runs the per-Gaussian adjoint
// (one thread per Gaussian) while the moments are still arriving, then waits on
// B and applies the optimiser element by element out of shared memory with
// coalesced vector stores.  The partial slice at the end of the model (sizes
// not multiples of 16 bytes) is staged with ordinary loads instead.
constexpr int kBwdG = 128;        // Gaussians (= threads) per CTA
constexpr int kMaxMc3 = 48;       // SH floats per Gaussian at degree 3
constexpr int kBasisPitch = 17;   // padded row of the per-Gaussian SH basis values

// The Adam moments come last: modes without the fused optimiser launch with
// offsetof(BwdShared, m_sh) bytes of shared memory and fit more CTAs per SM.
struct __align__(16) BwdShared {
    unsigned long long bar_a, bar_b;
    float sh[kBwdG * kMaxMc3];
    float pos[kBwdG * 3], sc[kBwdG * 3], rot[kBwdG * 4], op[kBwdG];
    float dm2[kBwdG * 2], dcon[kBwdG * 3], drgb[kBwdG * 3], dop[kBwdG];
    int radius[kBwdG];
    float basis[kBwdG * kBasisPitch], geff[kBwdG * 3];
    float gpos[kBwdG * 3], gsc[kBwdG * 3], grot[kBwdG * 4], gop[kBwdG];
    float m_sh[kBwdG * kMaxMc3], v_sh[kBwdG * kMaxMc3];
    float m_pos[kBwdG * 3], v_pos[kBwdG * 3], m_sc[kBwdG * 3], v_sc[kBwdG * 3];
    float m_rot[kBwdG * 4], v_rot[kBwdG * 4], m_op[kBwdG], v_op[kBwdG];
};

// Ordinary (tail-slice) staging of n floats.
__device__ __forceinline__ void copy_in(float* dst, const float* src, int n) {
    for (int e = threadIdx.x; e < n; e += kBwdG) dst[e] = src[e];
}

// Zeroes n floats of a gradient accumulator (coalesced, vectorised when aligned).
__device__ __forceinline__ void zero_out(float* dst, int n) {
    const int n4 = (((size_t)dst & 15) == 0) ? (n >> 2) : 0;
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (int q = threadIdx.x; q < n4; q += kBwdG) d4[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int e = 4 * n4 + threadIdx.x; e < n; e += kBwdG) dst[e] = 0.f;
}

// Optimiser over one parameter-group slice of n elements: parameters, moments
// and gradients read from shared memory, results stored to global memory.
template <class GradFn>
__device__ __forceinline__ void update_slice(const StepParams& sp, float* p_g, float* m_g, float* v_g,
                                             const float* p_s, const float* m_s, const float* v_s, int n,
                                             float lr, GradFn grad) {
    const bool vec = (((size_t)p_g | (size_t)m_g | (size_t)v_g) & 15) == 0;
    const int n4 = vec ? (n >> 2) : 0;
    for (int q = threadIdx.x; q < n4; q += kBwdG) {
        float pp[4], mm[4], vv[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = 4 * q + u;
            pp[u] = p_s[e];
            if (sp.use_adam) {
                mm[u] = m_s[e];
                vv[u] = v_s[e];
                pp[u] = adam_elem(pp[u], mm[u], vv[u], grad(e), lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            } else {
                pp[u] = pp[u] - lr * grad(e);
            }
        }
        reinterpret_cast<float4*>(p_g)[q] = make_float4(pp[0], pp[1], pp[2], pp[3]);
        if (sp.use_adam) {
            reinterpret_cast<float4*>(m_g)[q] = make_float4(mm[0], mm[1], mm[2], mm[3]);
            reinterpret_cast<float4*>(v_g)[q] = make_float4(vv[0], vv[1], vv[2], vv[3]);
        }
    }
    for (int e = 4 * n4 + threadIdx.x; e < n; e += kBwdG) {
        float pe = p_s[e];
        if (sp.use_adam) {
            float mm = m_s[e], vv = v_s[e];
            pe = adam_elem(pe, mm, vv, grad(e), lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            m_g[e] = mm;
            v_g[e] = vv;
        } else {
            pe = pe - lr * grad(e);
        }
        p_g[e] = pe;
    }
}

// Modes of k_preprocess_bwd.
constexpr int kBwdGrads = 0;   // stage API: write GradientOutput
constexpr int kBwdFused = 1;   // train step: apply the optimiser in the same kernel
constexpr int kBwdSplit = 2;   // train step: write GradientOutput for k_optimizer, zero the accumulators

// Preprocess backward (preprocessor_backward_cpu.cpp:8-645) for models whose
// SH arrays hold MC3 floats per Gaussian, fused with the optimiser update of all
// parameters or writing GradientOutput (see the modes above).
template <int MODE, int MC3>
__global__ void __launch_bounds__(kBwdG, MODE == 1 ? 2 : 4) k_preprocess_bwd(const StepParams* __restrict__ spp, int N,
                                                             ModelPtrs raw, AdamPtrs adam, ScreenPtrs s,
                                                             RGradPtrs rg, GradPtrs gout, Control* ctrl) {
    constexpr bool FUSED = MODE == kBwdFused;
    constexpr bool TRAIN = MODE != kBwdGrads;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    BwdShared& sm = *reinterpret_cast<BwdShared*>(smem_raw);
    const StepParams& sp = *spp;
    // an overflowed (or timed-out) step, or any step after one the host has not
    // acknowledged yet, updates nothing
    if (TRAIN && ((ctrl->status & (kStatusOverflow | kStatusTimeout)) || sp.persist->sticky_overflow)) return;
    if (FUSED && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&sp.persist->applied_steps, 1ull);
    const int tid = threadIdx.x;
    const size_t g0 = (size_t)blockIdx.x * kBwdG;
    const int ng = min(kBwdG, N - (int)g0);
    constexpr int mc3 = MC3;
    const bool want_mv = FUSED && sp.use_adam;
    const bool bulk = ng == kBwdG;   // every slice of a full CTA is a multiple of 512 bytes

    // ---- phase 0: staging ----
    if (bulk) {
        if (tid == 0) {
            mbar_init(&sm.bar_a, 1);
            mbar_init(&sm.bar_b, 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (tid == 0) {
            const unsigned B = 4u * kBwdG;   // bytes of one float per Gaussian
            mbar_arrive_expect_tx(&sm.bar_a, B * (11u + (unsigned)mc3 + 9u + 1u));
            tma_load_1d(sm.pos, raw.pos + 3 * g0, 3 * B, &sm.bar_a);
            tma_load_1d(sm.sc, raw.sc + 3 * g0, 3 * B, &sm.bar_a);
            tma_load_1d(sm.rot, raw.rot + 4 * g0, 4 * B, &sm.bar_a);
            tma_load_1d(sm.op, raw.op + g0, B, &sm.bar_a);
            tma_load_1d(sm.sh, raw.sh + (size_t)mc3 * g0, (unsigned)mc3 * B, &sm.bar_a);
            tma_load_1d(sm.dm2, rg.dm2 + 2 * g0, 2 * B, &sm.bar_a);
            tma_load_1d(sm.dcon, rg.dcon + 3 * g0, 3 * B, &sm.bar_a);
            tma_load_1d(sm.drgb, rg.drgb + 3 * g0, 3 * B, &sm.bar_a);
            tma_load_1d(sm.dop, rg.dop + g0, B, &sm.bar_a);
            tma_load_1d(sm.radius, s.radius + g0, B, &sm.bar_a);
            if (want_mv) {
                mbar_arrive_expect_tx(&sm.bar_b, 2u * B * (11u + (unsigned)mc3));
                tma_load_1d(sm.m_pos, adam.m_pos + 3 * g0, 3 * B, &sm.bar_b);
                tma_load_1d(sm.v_pos, adam.v_pos + 3 * g0, 3 * B, &sm.bar_b);
                tma_load_1d(sm.m_sc, adam.m_sc + 3 * g0, 3 * B, &sm.bar_b);
                tma_load_1d(sm.v_sc, adam.v_sc + 3 * g0, 3 * B, &sm.bar_b);
                tma_load_1d(sm.m_rot, adam.m_rot + 4 * g0, 4 * B, &sm.bar_b);
                tma_load_1d(sm.v_rot, adam.v_rot + 4 * g0, 4 * B, &sm.bar_b);
                tma_load_1d(sm.m_op, adam.m_op + g0, B, &sm.bar_b);
                tma_load_1d(sm.v_op, adam.v_op + g0, B, &sm.bar_b);
                tma_load_1d(sm.m_sh, adam.m_sh + (size_t)mc3 * g0, (unsigned)mc3 * B, &sm.bar_b);
                tma_load_1d(sm.v_sh, adam.v_sh + (size_t)mc3 * g0, (unsigned)mc3 * B, &sm.bar_b);
            }
        }
        mbar_wait(&sm.bar_a, 0, sp.spin_limit, &ctrl->status);
    } else {
        copy_in(sm.pos, raw.pos + 3 * g0, 3 * ng);
        copy_in(sm.sc, raw.sc + 3 * g0, 3 * ng);
        copy_in(sm.rot, raw.rot + 4 * g0, 4 * ng);
        copy_in(sm.op, raw.op + g0, ng);
        copy_in(sm.sh, raw.sh + (size_t)mc3 * g0, mc3 * ng);
        copy_in(sm.dm2, rg.dm2 + 2 * g0, 2 * ng);
        copy_in(sm.dcon, rg.dcon + 3 * g0, 3 * ng);
        copy_in(sm.drgb, rg.drgb + 3 * g0, 3 * ng);
        copy_in(sm.dop, rg.dop + g0, ng);
        for (int e = tid; e < ng; e += kBwdG) sm.radius[e] = s.radius[g0 + e];
        if (want_mv) {
            copy_in(sm.m_pos, adam.m_pos + 3 * g0, 3 * ng);
            copy_in(sm.v_pos, adam.v_pos + 3 * g0, 3 * ng);
            copy_in(sm.m_sc, adam.m_sc + 3 * g0, 3 * ng);
            copy_in(sm.v_sc, adam.v_sc + 3 * g0, 3 * ng);
            copy_in(sm.m_rot, adam.m_rot + 4 * g0, 4 * ng);
            copy_in(sm.v_rot, adam.v_rot + 4 * g0, 4 * ng);
            copy_in(sm.m_op, adam.m_op + g0, ng);
            copy_in(sm.v_op, adam.v_op + g0, ng);
            copy_in(sm.m_sh, adam.m_sh + (size_t)mc3 * g0, mc3 * ng);
            copy_in(sm.v_sh, adam.v_sh + (size_t)mc3 * g0, mc3 * ng);
        }
        __syncthreads();
    }
    if (TRAIN) {
        // the screen-gradient accumulators start at zero for the next step's raster backward
        zero_out(rg.dm2 + 2 * g0, 2 * ng);
        zero_out(rg.dcon + 3 * g0, 3 * ng);
        zero_out(rg.drgb + 3 * g0, 3 * ng);
        zero_out(rg.dop + g0, ng);
    }

    // ---- phase 1: per-Gaussian adjoint ----
    BwdOut o;
#pragma unroll
    for (int k = 0; k < 3; k++) { o.gp[k] = 0.f; o.gs[k] = 0.f; o.geff[k] = 0.f; }
#pragma unroll
    for (int k = 0; k < 4; k++) o.gq[k] = 0.f;
    o.gop = 0.f;
#pragma unroll
    for (int k = 0; k < 16; k++) o.basis[k] = 0.f;
    if (tid < ng && sm.radius[tid] > 0) {
        float shr[kMaxMc3];
        if (mc3 == kMaxMc3) {
            const float4* s4 = reinterpret_cast<const float4*>(sm.sh + tid * kMaxMc3);
#pragma unroll
            for (int q = 0; q < kMaxMc3 / 4; q++) {
                const float4 v = s4[q];
                shr[4 * q] = v.x; shr[4 * q + 1] = v.y; shr[4 * q + 2] = v.z; shr[4 * q + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kMaxMc3; k++) shr[k] = k < mc3 ? sm.sh[tid * mc3 + k] : 0.0f;
        }
        BwdIn in;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            in.p[k] = sm.pos[3 * tid + k];
            in.rsc[k] = sm.sc[3 * tid + k];
            in.dcn[k] = sm.dcon[3 * tid + k];
            in.drgb[k] = sm.drgb[3 * tid + k];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) in.rq[k] = sm.rot[4 * tid + k];
        in.rop = sm.op[tid];
        in.act = nullptr;
        float act[8];
        if (MODE == kBwdGrads && sp.raw_rot) {
            // activated device model (stage API): its values are the activation, raw_rot the raw quaternion
#pragma unroll
            for (int k = 0; k < 3; k++) act[k] = sm.sc[3 * tid + k];
#pragma unroll
            for (int k = 0; k < 4; k++) act[3 + k] = sm.rot[4 * tid + k];
            act[7] = sm.op[tid];
#pragma unroll
            for (int k = 0; k < 4; k++) in.rq[k] = sp.raw_rot[4 * (g0 + tid) + k];
            in.act = act;
        }
        in.dm[0] = sm.dm2[2 * tid];
        in.dm[1] = sm.dm2[2 * tid + 1];
        in.dop = sm.dop[tid];
        in.sh = shr;
        backward_one(sp, in, o);
    }
    if (tid < ng) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            sm.gpos[3 * tid + k] = o.gp[k];
            sm.gsc[3 * tid + k] = o.gs[k];
            sm.geff[3 * tid + k] = o.geff[k];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) sm.grot[4 * tid + k] = o.gq[k];
        sm.gop[tid] = o.gop;
#pragma unroll
        for (int k = 0; k < 16; k++) sm.basis[tid * kBasisPitch + k] = o.basis[k];
    }
    __syncthreads();

    // ---- phase 2: element-wise optimiser (or GradientOutput) ----
    auto sh_grad = [&](int e) {
        const int gg = e / mc3, j = e - gg * mc3;
        const int k = j / 3, c = j - 3 * k;
        return sm.basis[gg * kBasisPitch + k] * sm.geff[3 * gg + c];
    };
    if (FUSED) {
        if (bulk && want_mv) mbar_wait(&sm.bar_b, 0, sp.spin_limit, &ctrl->status);
        update_slice(sp, raw.pos + 3 * g0, adam.m_pos + 3 * g0, adam.v_pos + 3 * g0, sm.pos, sm.m_pos, sm.v_pos,
                     3 * ng, sp.lr_pos, [&](int e) { return sm.gpos[e]; });
        update_slice(sp, raw.sc + 3 * g0, adam.m_sc + 3 * g0, adam.v_sc + 3 * g0, sm.sc, sm.m_sc, sm.v_sc, 3 * ng,
                     sp.lr_scale, [&](int e) { return sm.gsc[e]; });
        update_slice(sp, raw.rot + 4 * g0, adam.m_rot + 4 * g0, adam.v_rot + 4 * g0, sm.rot, sm.m_rot, sm.v_rot,
                     4 * ng, sp.lr_rot, [&](int e) { return sm.grot[e]; });
        update_slice(sp, raw.op + g0, adam.m_op + g0, adam.v_op + g0, sm.op, sm.m_op, sm.v_op, ng, sp.lr_opac,
                     [&](int e) { return sm.gop[e]; });
        update_slice(sp, raw.sh + (size_t)mc3 * g0, adam.m_sh + (size_t)mc3 * g0, adam.v_sh + (size_t)mc3 * g0,
                     sm.sh, sm.m_sh, sm.v_sh, mc3 * ng, sp.lr_sh, sh_grad);
    } else {
        for (int e = tid; e < 3 * ng; e += kBwdG) {
            gout.g_pos[3 * g0 + e] = sm.gpos[e];
            gout.g_sc[3 * g0 + e] = sm.gsc[e];
        }
        for (int e = tid; e < 4 * ng; e += kBwdG) gout.g_rot[4 * g0 + e] = sm.grot[e];
        for (int e = tid; e < ng; e += kBwdG) gout.g_op[g0 + e] = sm.gop[e];
        for (int e = tid; e < mc3 * ng; e += kBwdG) gout.g_sh[(size_t)mc3 * g0 + e] = sh_grad(e);
    }
}

// Optimiser over one parameter array: element-wise Adam / SGD (optimizer.cpp:9-43)
// with float4 loads and stores.
__device__ __forceinline__ void update_array(const StepParams& sp, float* __restrict__ p, float* __restrict__ m,
                                             float* __restrict__ v, const float* __restrict__ g, long long n,
                                             float lr) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long n4 = n >> 2;
    float4* p4 = reinterpret_cast<float4*>(p);
    float4* m4 = reinterpret_cast<float4*>(m);
    float4* v4 = reinterpret_cast<float4*>(v);
    const float4* g4 = reinterpret_cast<const float4*>(g);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
        float4 pp = p4[q];
        const float4 gg = g4[q];
        if (sp.use_adam) {
            float4 mm = m4[q], vv = v4[q];
            pp.x = adam_elem(pp.x, mm.x, vv.x, gg.x, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            pp.y = adam_elem(pp.y, mm.y, vv.y, gg.y, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            pp.z = adam_elem(pp.z, mm.z, vv.z, gg.z, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            pp.w = adam_elem(pp.w, mm.w, vv.w, gg.w, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            m4[q] = mm;
            v4[q] = vv;
        } else {
            pp.x = pp.x - lr * gg.x;
            pp.y = pp.y - lr * gg.y;
            pp.z = pp.z - lr * gg.z;
            pp.w = pp.w - lr * gg.w;
        }
        p4[q] = pp;
    }
    for (long long i = 4 * n4 + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        apply_update(sp, &p[i], &m[i], &v[i], g[i], lr);
}

// Stand-alone optimiser step over the gradient arrays (optimizer.cpp:9-101).
// With ctrl (the split train step) an overflowed or unacknowledged step updates nothing.
__global__ void __launch_bounds__(256) k_optimizer(const StepParams* __restrict__ spp, long long n, int mc3,
                                                   ModelPtrs raw, AdamPtrs adam, GradPtrs g, const Control* ctrl) {
    const StepParams& sp = *spp;
    if (ctrl && ((ctrl->status & (kStatusOverflow | kStatusTimeout)) || sp.persist->sticky_overflow)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0 && sp.use_adam) atomicAdd(&sp.persist->applied_steps, 1ull);
    update_array(sp, raw.sh, adam.m_sh, adam.v_sh, g.g_sh, n * mc3, sp.lr_sh);
    update_array(sp, raw.pos, adam.m_pos, adam.v_pos, g.g_pos, 3 * n, sp.lr_pos);
    update_array(sp, raw.sc, adam.m_sc, adam.v_sc, g.g_sc, 3 * n, sp.lr_scale);
    update_array(sp, raw.rot, adam.m_rot, adam.v_rot, g.g_rot, 4 * n, sp.lr_rot);
    update_array(sp, raw.op, adam.m_op, adam.v_op, g.g_op, n, sp.lr_opac);
}

inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace
}  // namespace gs3d

#include "eval3d.cuh"

namespace gs3d {

cudaError_t launch_preprocess_plain(cudaStream_t st, const StepParams* sp, int N, bool train, bool cache,
                                    ModelPtrs m, ScreenPtrs s, PairPtrs pr, Control* ctrl, DepthKeys dk) {
    if (N <= 0) return cudaSuccess;
    const int grid = blocks_for(N, kBlock);
    if (dk.keys) {
        if (train) {
            if (cache) k_preprocess<true, true, false><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
            else k_preprocess<true, false, false><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
        } else {
            if (cache) k_preprocess<false, true, false><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
            else k_preprocess<false, false, false><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
        }
    } else if (train) {
        if (cache) k_preprocess<true, true, true><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
        else k_preprocess<true, false, true><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
    } else {
        if (cache) k_preprocess<false, true, true><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
        else k_preprocess<false, false, true><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
    }
    return cudaGetLastError();
}

cudaError_t launch_emit_ranked(cudaStream_t st, const StepParams* sp, int N, const unsigned* rank_gid,
                               ScreenPtrs s, PairPtrs pr, Control* ctrl, const uint2* rects, int n_per_view,
                               int hist_slot, unsigned* hist_parts) {
    if (N <= 0) return cudaSuccess;
    // 512 Gaussians per CTA: half the CTAs of the preprocess's 256, so half the look-backs and
    // histogram flushes
    k_emit_ranked<kEmitBlock><<<blocks_for(N, kEmitBlock), kEmitBlock, 0, st>>>(sp, N, rank_gid, s, pr, rects, ctrl,
                                                                                n_per_view, hist_slot, hist_parts);
    if (hist_parts) k_hist_parts_reduce<<<1, 256, 0, st>>>(hist_parts, sp, ctrl, hist_slot);
    return cudaGetLastError();
}

cudaError_t launch_bin_arrays(cudaStream_t st, const StepParams* sp, int N, ScreenArrays a, PairPtrs pr,
                              Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    k_bin_arrays<<<blocks_for(N, kBlock), kBlock, 0, st>>>(sp, N, a, pr, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_export_screen(cudaStream_t st, int N, ScreenPtrs s, ScreenArrays a) {
    if (N <= 0) return cudaSuccess;
    k_export_screen<<<blocks_for(N, 256), 256, 0, st>>>(N, s, a);
    return cudaGetLastError();
}

cudaError_t launch_import_screen(cudaStream_t st, int N, ScreenArrays a, ScreenPtrs s) {
    if (N <= 0) return cudaSuccess;
    k_import_screen<<<blocks_for(N, 256), 256, 0, st>>>(N, a, s);
    return cudaGetLastError();
}

cudaError_t launch_e3_view(cudaStream_t st, const StepParams* sp, int num_tiles, E3Ptrs e) {
    k_e3_view<<<blocks_for(num_tiles > 0 ? num_tiles : 1, 256), 256, 0, st>>>(sp, e.tdir, e.view);
    return cudaGetLastError();
}

cudaError_t launch_preprocess_e3(cudaStream_t st, const StepParams* sp, int N, bool raw, ModelPtrs m,
                                 const float* filt, ScreenPtrs s, E3Ptrs e, PairPtrs pr, Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    if (raw) k_preprocess_e3<true><<<blocks_for(N, kBlock), kBlock, 0, st>>>(sp, N, m, filt, s, e, pr, ctrl);
    else k_preprocess_e3<false><<<blocks_for(N, kBlock), kBlock, 0, st>>>(sp, N, m, filt, s, e, pr, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_bin_arrays_e3(cudaStream_t st, const StepParams* sp, int N, ScreenArrays a, E3Ptrs e,
                                 PairPtrs pr, Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    k_bin_arrays_e3<<<blocks_for(N, kBlock), kBlock, 0, st>>>(sp, N, a, e.ci, e.mo, e.tdir, pr, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_raster_e3(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                             const unsigned* order, const unsigned* vals, E3Ptrs e, PixelPtrs px, Control* ctrl) {
    if (num_tiles <= 0) return cudaSuccess;
    static std::atomic<unsigned long long> attr_done{0};   // the kernel's dynamic shared memory above 48 KB
    const cudaError_t err = set_smem_once(attr_done, k_raster_e3, (int)kE3RasterSmem);
    if (err != cudaSuccess) return err;
    k_raster_e3<<<num_tiles, kE3Threads, kE3RasterSmem, st>>>(sp, ranges, order, vals, e, px, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_raster_fwd_plain(cudaStream_t st, const StepParams* sp, int num_tiles, bool fused_loss,
                                    const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                    ScreenPtrs s, PixelPtrs px, Control* ctrl, int ppt, int batch, bool loss_later) {
    if (num_tiles <= 0) return cudaSuccess;
    if (!fused_loss) batch = 128;   // renders and the stage API
    return with_ppt_batch(ppt, batch, [&](auto P, auto Bt) {
        constexpr int kP = decltype(P)::value, kB = decltype(Bt)::value;
        if (fused_loss && loss_later)
            k_raster_fwd<kLossLater, ExactBlend, false, kP, kB><<<num_tiles, 256 / kP, 0, st>>>(
                sp, ranges, order, vals, s, px, ctrl);
        else if (fused_loss)
            k_raster_fwd<kFusedL1, ExactBlend, false, kP, kB><<<num_tiles, 256 / kP, 0, st>>>(sp, ranges, order, vals,
                                                                                             s, px, ctrl);
        else
            k_raster_fwd<kCountContrib, ExactBlend, false, kP, kFwdBatch><<<num_tiles, 256 / kP, 0, st>>>(
                sp, ranges, order, vals, s, px, ctrl);
        return cudaGetLastError();
    });
}

cudaError_t launch_l1_loss(cudaStream_t st, const StepParams* sp, PixelPtrs px, size_t n_pix, Control* ctrl) {
    if (n_pix == 0) return cudaSuccess;
    const size_t want = (n_pix + 255) / 256;
    const size_t cap = 8ull * (size_t)sm_count();
    k_l1_loss<<<(unsigned)(want < cap ? want : cap), 256, 0, st>>>(sp, px, n_pix, ctrl);
    return cudaGetLastError();
}

namespace {
template <int MODE, int MC3>
cudaError_t launch_bwd_mc(cudaStream_t st, const StepParams* sp, int N, ModelPtrs raw, AdamPtrs adam, ScreenPtrs s,
                          RGradPtrs rg, GradPtrs gout, Control* ctrl) {
    const int smem = MODE == kBwdFused ? (int)sizeof(BwdShared) : (int)offsetof(BwdShared, m_sh);
    static std::atomic<unsigned long long> attr_done{0};
    const cudaError_t e = set_smem_once(attr_done, k_preprocess_bwd<MODE, MC3>, smem);
    if (e != cudaSuccess) return e;
    k_preprocess_bwd<MODE, MC3><<<blocks_for(N, kBwdG), kBwdG, smem, st>>>(sp, N, raw, adam, s, rg, gout, ctrl);
    return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_bwd_mode(cudaStream_t st, const StepParams* sp, int N, int mc3, ModelPtrs raw, AdamPtrs adam,
                            ScreenPtrs s, RGradPtrs rg, GradPtrs gout, Control* ctrl) {
    switch (mc3) {
        case 3: return launch_bwd_mc<MODE, 3>(st, sp, N, raw, adam, s, rg, gout, ctrl);
        case 12: return launch_bwd_mc<MODE, 12>(st, sp, N, raw, adam, s, rg, gout, ctrl);
        case 27: return launch_bwd_mc<MODE, 27>(st, sp, N, raw, adam, s, rg, gout, ctrl);
        case 48: return launch_bwd_mc<MODE, 48>(st, sp, N, raw, adam, s, rg, gout, ctrl);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace

cudaError_t launch_preprocess_bwd_plain(cudaStream_t st, const StepParams* sp, int N, int mc3, int mode,
                                        ModelPtrs raw, AdamPtrs adam, ScreenPtrs s, RGradPtrs rg, GradPtrs gout,
                                        Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    switch (mode) {
        case kBwdGrads: return launch_bwd_mode<kBwdGrads>(st, sp, N, mc3, raw, adam, s, rg, gout, ctrl);
        case kBwdFused: return launch_bwd_mode<kBwdFused>(st, sp, N, mc3, raw, adam, s, rg, gout, ctrl);
        case kBwdSplit: return launch_bwd_mode<kBwdSplit>(st, sp, N, mc3, raw, adam, s, rg, gout, ctrl);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_optimizer_plain(cudaStream_t st, const StepParams* sp, int N, int mc3, ModelPtrs raw,
                                   AdamPtrs adam, GradPtrs g, const Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    k_optimizer<<<8 * sm_count(), 256, 0, st>>>(sp, (long long)N, mc3, raw, adam, g, ctrl);
    return cudaGetLastError();
}

}  // namespace gs3d
