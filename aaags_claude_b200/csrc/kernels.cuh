// kernels.cuh -- argument structs and host-side launchers of the 3DGS kernels.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "common.cuh"

namespace gs3d {

// Calls f(PPT, BATCH) with the rasterisers' compile-time pixels per thread
// (1, 2, 4; anything else: 2) and staging batch (64, 128, 256; anything else: 128).
template <class F>
cudaError_t with_ppt_batch(int ppt, int batch, F&& f) {
    auto pick_batch = [&](auto P) -> cudaError_t {
        if (batch == 64) return f(P, std::integral_constant<int, 64>{});
        if (batch == 256) return f(P, std::integral_constant<int, 256>{});
        return f(P, std::integral_constant<int, 128>{});
    };
    if (ppt == 1) return pick_batch(std::integral_constant<int, 1>{});
    if (ppt == 4) return pick_batch(std::integral_constant<int, 4>{});
    return pick_batch(std::integral_constant<int, 2>{});
}

// Model parameters in the reference layouts: raw (training) or activated (render).
struct ModelPtrs {
    float* pos;   // [N*3]
    float* sc;    // [N*3]
    float* rot;   // [N*4]
    float* sh;    // [N*K*3]
    float* op;    // [N]
};

struct AdamPtrs {
    float *m_pos, *v_pos, *m_sc, *v_sc, *m_rot, *v_rot, *m_sh, *v_sh, *m_op, *v_op;
};

// Screen-space records written by the preprocess and read by both rasterisers.
//   rec0[i] = (mean.x, mean.y, conic.a, conic.b)
//   rec1[i] = (conic.c, opacity_2d, r, g)
//   cbt[i]  = (b, -log2(255 opacity_2d)): the blue channel and the base-2
//             accept threshold (blue_thr), computed once per Gaussian instead
//             of once per (Gaussian, tile) by the rasterisers' staging
struct ScreenPtrs {
    float4* rec0;
    float4* rec1;
    float2* cbt;
    float* depth;
    int* radius;
    int* tiles;
    // optional ForwardCache fields (NULL unless requested)
    float* cov3D;
    float* p_view;
    float* p_hom_w;
    float* cov2D;
    float* det;
};

struct PairPtrs {
    unsigned long long* keys;   // [capacity]
    unsigned* vals;             // [capacity]
    unsigned long long capacity;
    unsigned long long* scan_desc;  // look-back descriptors, one per emitting CTA (at most one per 256 Gaussians)
    unsigned* tiles32 = nullptr;    // depth-ordered emission: tile-only keys [capacity] instead of keys
};

struct PixelPtrs {
    float* image;          // [H*W*3]
    float* T_final;        // [H*W]
    int* n_contrib;        // [H*W] contributor count (ForwardCache::n_contrib)
    unsigned* last_j;      // [H*W] one past the last contributing pair index
    unsigned char* dsign;  // [H*W] L1 signs: bits 0-1 ch0, 2-3 ch1, 4-5 ch2 (1:+, 2:-)
    const float* d_image;  // [H*W*3] explicit image gradient (stage API)
};

// Screen-space gradients (RasterGradOutput, include/train_types.h:25-32).
struct RGradPtrs {
    float* dm2;   // [N*2]
    float* dcon;  // [N*3]
    float* drgb;  // [N*3]
    float* dop;   // [N]
};

// Raw-parameter gradients (GradientOutput, include/train_types.h:35-43).
struct GradPtrs {
    float *g_pos, *g_sc, *g_rot, *g_sh, *g_op;
};

// Host arrays in PreprocessOutput layout, on the device (export / import).
// Adaptive density control: statistics and the scratch of densify_and_prune.
struct DensityPtrs {
    float* accum;     // [N] sum of |d_means2D|
    float* denom;     // [N] steps counted
    int* max_radii;   // [N] largest screen radius seen
    int* clone;       // [N] flags
    int* split;       // [N]
    int* crank;       // [N] exclusive rank among the clones
    int* srank;       // [N] exclusive rank among the splits
    int* src;         // [M] source Gaussian of each post-split entry; reused as the gather map
    int* keep;        // [M] kept after pruning
    int* out;         // [M] exclusive rank among the kept
    int* sums;        // scan block sums (+ the grand total at the end)
};

cudaError_t launch_dc_accumulate(cudaStream_t st, int N, float* dm2, const int* radii, DensityPtrs d, bool clear);
cudaError_t launch_scan_int(cudaStream_t st, const int* in, int* out, int* sums, int n);
cudaError_t launch_dc_classify(cudaStream_t st, int N, const float* sc, DensityPtrs d, float threshold,
                               float size_thr);
cudaError_t launch_dc_expand(cudaStream_t st, int N, int n_c, int n_s, ModelPtrs m, int mc3, DensityPtrs d,
                             ModelPtrs t, unsigned long long rng0, float log_factor);
cudaError_t launch_dc_keep(cudaStream_t st, int M, int N, ModelPtrs t, DensityPtrs d, float min_opacity,
                           int max_screen_size, float world_thr);
cudaError_t launch_dc_compact(cudaStream_t st, int M, int new_n, ModelPtrs t, int mc3, DensityPtrs d, ModelPtrs out);
cudaError_t launch_fill(cudaStream_t st, float* p, long long n, float v);

// Per-Gaussian arrays of the 3D-evaluation mode (RenderConfig::eval_3D).
constexpr int kE3Rec = 8;   // float4s per raster record
struct E3Ptrs {
    float4* rec;      // [N*kE3Rec] raster record: gauss2screen rows 0, 1, 3; cov3D_inv; mean_offset,
                      // opacity, depth, rgb, alpha threshold; skip box
    float* g2s;       // [N*16] gauss2screen (row-major), zero for culled Gaussians
    float* ci;        // [N*6] inverse 3D covariance (upper triangle)
    float* mo;        // [N*3] position - camera position
    float4* tdir;     // [num_tiles] unit ray through each tile centre, w = 1 when defined
    float* view;      // [17] inverse view-projection (column-major) and its validity flag
};

struct ScreenArrays {
    float* means2D;
    float* depths;
    float* conics;
    float* opac2d;
    float* rgb;
    int* radii;
    int* tiles;
};

// Gaussian depth-sort input written by a preprocess that does not emit pairs.
struct DepthKeys {
    unsigned* keys;             // [N] depth bits, ~0u for Gaussians without pairs
    unsigned* vals;             // [N] Gaussian index
    bool views24 = false;       // several views: keys = view << 24 | the depth's upper 24 bits
    uint2* rects = nullptr;   // plain preprocess: tile rectangles (xmin | ymin << 16, xmax | ymax << 16), 0 if none
    unsigned long long seg_keys = 0;   // several views: view v's keys at v * seg_keys (padded segments)
};

// Reduced-storage ("chosen") form: positions FP32, the other attributes and the
// SH coefficients 16-bit (BF16 or FP16), Adam moments BF16 (positions: FP32).
struct ChosenPtrs {
    float* pos;     // [N*3]
    void* attr;     // [N*8] 16-bit: raw scale[3], raw opacity, raw rotation[4] (16 bytes per Gaussian)
    void* sh;       // [N*mc3] 16-bit, the reference's basis-interleaved order
    float* m_pos;   // [N*3] Adam moments of the positions
    float* v_pos;
    void* m_attr;   // [N*8] BF16
    void* v_attr;
    void* m_sh;     // [N*mc3] BF16
    void* v_sh;
};

// FP32 raw arrays (reference layout) -> reduced storage (round to nearest) and back.
cudaError_t launch_chosen_from_raw(cudaStream_t st, int N, int mc3, bool fp16, ModelPtrs raw, ChosenPtrs c);
cudaError_t launch_chosen_to_raw(cudaStream_t st, int N, int mc3, bool fp16, ChosenPtrs c, ModelPtrs raw);
// Preprocess of the reduced-storage model: screen records, depth-sort input
// and tile rectangles (the reference's rectangle cut to the box of the
// ellipse where alpha can reach 1/255).
// n_views > 1: sp is the views' parameter array; the outputs hold (view,
// Gaussian) entries view * N + i and, with dk.views24, the 32-bit depth key
// is the view above the depth's upper 24 bits (one 4-pass sort orders every
// entry by (view, depth)).
cudaError_t launch_chosen_preprocess(cudaStream_t st, const StepParams* sp, int N, bool fp16, ChosenPtrs c,
                                     ScreenPtrs s, DepthKeys dk, uint2* rects, Control* ctrl, int n_views = 1);
// Forward rasteriser with the fast-exp blend decision and fused L1
// (loss_later: no loss; launch_l1_loss follows).
cudaError_t launch_raster_fwd_fast(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                                   const unsigned* order, const unsigned* vals, ScreenPtrs s, PixelPtrs px,
                                   Control* ctrl, int ppt = 2, int batch = 128, bool loss_later = false);
// One persistent launch over all tiles of n_views views (views = their
// parameter array, order = all global tiles, heavy first).
cudaError_t launch_raster_fwd_fast_multi(cudaStream_t st, const StepParams* views, int n_views, unsigned n_tiles,
                                         const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                         ScreenPtrs s, PixelPtrs px, Control* ctrl, int ppt = 2, int batch = 128);
cudaError_t launch_raster_bwd_fast_multi(cudaStream_t st, const StepParams* views, int n_views, unsigned n_tiles,
                                         const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                         ScreenPtrs s, PixelPtrs px, RGradPtrs g, Control* ctrl, int ppt = 2,
                                         int batch = 128);
// Backward rasteriser deciding acceptance like launch_raster_fwd_fast.
cudaError_t launch_raster_bwd_fast(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                                   const unsigned* order, const unsigned* vals, ScreenPtrs s, PixelPtrs px,
                                   RGradPtrs g, Control* ctrl, int ppt = 2, int batch = 128);
// Per-Gaussian adjoint fused with Adam (stochastic rounding into the 16-bit
// parameters and BF16 moments); zeroes the screen-gradient accumulators.
// With g.g_pos != NULL the FP32 raw-parameter gradients are stored too.
// n_views > 1: sp is the views' parameter array and rg holds (view, Gaussian)
// entries; each Gaussian's gradient is the sum over the views.
cudaError_t launch_chosen_backward_adam(cudaStream_t st, const StepParams* sp, int N, int mc3, bool fp16,
                                        ChosenPtrs c, RGradPtrs rg, GradPtrs gout, Control* ctrl, int n_views = 1);

// ---- plain FP32 kernels (plain.cu, compiled without FMA contraction) ----
// The rasterisers' ppt (pixels per thread: 1, 2 or 4) sets 256 / ppt threads
// per 16x16 tile; the results do not depend on it (the backward's FP32 sums
// only change order).
// Preprocess; emits the pairs in Gaussian order, or -- when dk.keys != NULL --
// writes the depth-sort input instead (pairs come from launch_emit_ranked).
cudaError_t launch_preprocess_plain(cudaStream_t st, const StepParams* sp, int N, bool train,
                                    bool cache, ModelPtrs m, ScreenPtrs s, PairPtrs pr, Control* ctrl,
                                    DepthKeys dk = DepthKeys{nullptr, nullptr});
// Emits the pairs of the Gaussians in the order rank_gid lists them
// (depth order), with the same scan / look-back as the preprocess: tile-only
// keys to pr.tiles32, and the tile-digit histograms into control slots
// kDepthDigits.. for launch_radix_sort32.
// rects (optional): per-Gaussian tile rectangles (xmin | ymin << 16,
// xmax | ymax << 16) written by the reduced-storage preprocess; without them
// the rectangle is recomputed from the stored mean and radius.
// n_per_view > 0: several views; N counts (view, Gaussian) entries
// view * n_per_view + i, and sp is the views' parameter array.  The keys are
// the views' local tile ids with the view above the tile digits: the emission
// order groups the pairs by view, so a stable sort on the tile digits leaves
// every (view, tile) run contiguous (launch_tile_ranges_views).
// hist_parts (optional, zeroed, kHistParts * (kMaxPasses - kDepthDigits) * 256
// counters): the CTAs add their counts into copy (CTA % kHistParts) and one
// more kernel sums the copies into the control slots -- for launches of many
// CTAs, whose adds would otherwise meet on the same 256 * digits addresses.
cudaError_t launch_emit_ranked(cudaStream_t st, const StepParams* sp, int N, const unsigned* rank_gid,
                               ScreenPtrs s, PairPtrs pr, Control* ctrl, const uint2* rects = nullptr,
                               int n_per_view = 0, int hist_slot = kDepthDigits, unsigned* hist_parts = nullptr);
cudaError_t launch_bin_arrays(cudaStream_t st, const StepParams* sp, int N, ScreenArrays a,
                              PairPtrs pr, Control* ctrl);
cudaError_t launch_export_screen(cudaStream_t st, int N, ScreenPtrs s, ScreenArrays a);
// means2D / conics / opac2d / rgb of a caller -> rec0 / rec1 / col_b
cudaError_t launch_import_screen(cudaStream_t st, int N, ScreenArrays a, ScreenPtrs s);
// 3D-evaluation mode: view setup (inverse view-projection, tile rays), the
// fused preprocess + pair emission (raw: activate the device model first;
// filt: per-Gaussian 3D filter or NULL), the emission from host arrays (a.means2D,
// depths, radii, tiles with e.ci / e.mo) and the buffered rasteriser.
cudaError_t launch_e3_view(cudaStream_t st, const StepParams* sp, int num_tiles, E3Ptrs e);
cudaError_t launch_preprocess_e3(cudaStream_t st, const StepParams* sp, int N, bool raw, ModelPtrs m,
                                 const float* filt, ScreenPtrs s, E3Ptrs e, PairPtrs pr, Control* ctrl);
cudaError_t launch_bin_arrays_e3(cudaStream_t st, const StepParams* sp, int N, ScreenArrays a, E3Ptrs e,
                                 PairPtrs pr, Control* ctrl);
cudaError_t launch_raster_e3(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                             const unsigned* order, const unsigned* vals, E3Ptrs e, PixelPtrs px, Control* ctrl);
// order: tile permutation (heavy first) or NULL for row-major
// batch: the records staged per round (64, 128, 256) in the train step's launches (fused loss /
// FROM_SIGN); the stage API's launches stage 128.
// fused_loss && loss_later: a train step's forward without the loss (launch_l1_loss follows).
cudaError_t launch_raster_fwd_plain(cudaStream_t st, const StepParams* sp, int num_tiles, bool fused_loss,
                                    const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                    ScreenPtrs s, PixelPtrs px, Control* ctrl, int ppt = 2, int batch = 128,
                                    bool loss_later = false);
// The train step's L1 over the image of a loss_later forward and the target at
// sp->gt: sign bytes and the loss sum, as the fused forward writes them.
cudaError_t launch_l1_loss(cudaStream_t st, const StepParams* sp, PixelPtrs px, size_t n_pix, Control* ctrl);
cudaError_t launch_raster_bwd_plain(cudaStream_t st, const StepParams* sp, int num_tiles, bool from_sign,
                                    const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                    ScreenPtrs s, PixelPtrs px, RGradPtrs g, Control* ctrl, int ppt = 2,
                                    int batch = 128);
// Stored-list raster backward (memory comparison with the recompute backward):
// each pixel's contributors (Gaussian, alpha bits) are replayed into
// list[offset[pix] .. offset[pix] + n_contrib[pix]), then walked back to front
// with the explicit image gradient px.d_image.
cudaError_t launch_list_fill(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                             const unsigned* vals, ScreenPtrs s, const int* n_contrib, const int* offset,
                             uint2* list);
cudaError_t launch_list_bwd(cudaStream_t st, const StepParams* sp, int num_tiles, ScreenPtrs s, PixelPtrs px,
                            const int* offset, const uint2* list, RGradPtrs g);
// mode: 0 = write GradientOutput (stage API), 1 = fused optimiser, 2 = write
// GradientOutput for a following launch_optimizer_plain and zero the screen
// gradient accumulators (split train step).  mc3 in {3, 12, 27, 48}.
cudaError_t launch_preprocess_bwd_plain(cudaStream_t st, const StepParams* sp, int N, int mc3, int mode,
                                        ModelPtrs raw, AdamPtrs adam, ScreenPtrs s, RGradPtrs rg,
                                        GradPtrs gout, Control* ctrl);
// ctrl != NULL: skip an overflowed / unacknowledged train step.
cudaError_t launch_optimizer_plain(cudaStream_t st, const StepParams* sp, int N, int mc3, ModelPtrs raw,
                                   AdamPtrs adam, GradPtrs g, const Control* ctrl);

// ---- radix sort + ranges (sort.cu) ----
// Sorts (keys, vals) of *P (device) pairs by the low sort_bits key bits with
// 8-bit LSD passes, ping-ponging between buffer 0 and 1.  Returns in *which
// the buffer that holds the result.  desc must hold passes * desc_stride
// descriptors, zeroed by the caller before the call.
cudaError_t launch_radix_sort(cudaStream_t st, const StepParams* sp, int sort_passes,
                              unsigned long long capacity, unsigned long long* keys0, unsigned* vals0,
                              unsigned long long* keys1, unsigned* vals1, unsigned long long* desc,
                              unsigned long long desc_stride, Control* ctrl, int* which,
                              cudaEvent_t after_hist = nullptr, int first_pass = 0,
                              const unsigned long long* count = nullptr);
cudaError_t launch_tile_ranges(cudaStream_t st, unsigned long long capacity,
                               const unsigned long long* keys_sorted, unsigned* ranges, Control* ctrl);

// Stable LSD sort of 32-bit keys over digits [first_digit, digits), control
// slots slot_base..; hist_done: the digit histograms are already in those slots.
// desc holds (digits - first_digit) * desc_stride zeroed descriptors.
// count (optional): device word with the number of keys (default: the pair count).
// first_digit > 0 orders by the key's upper bits only (ties keep input order).
cudaError_t launch_radix_sort32(cudaStream_t st, const StepParams* sp, int digits, int slot_base, bool hist_done,
                                unsigned long long capacity, unsigned* keys0, unsigned* vals0, unsigned* keys1,
                                unsigned* vals1, unsigned long long* desc, unsigned long long desc_stride,
                                Control* ctrl, int* which, cudaEvent_t after_hist = nullptr,
                                const unsigned long long* count = nullptr, int first_digit = 0);
cudaError_t launch_tile_ranges32(cudaStream_t st, unsigned long long capacity, const unsigned* tiles_sorted,
                                 unsigned* ranges, Control* ctrl);
// Stable sort of 32-bit keys in segments of seg_keys keys (a multiple of 8192;
// capacity a multiple of seg_keys), each segment sorted apart, on digits
// [first_digit, first_digit + digits); every slot of the capacity is a key
// (ctrl->gauss_keys = capacity).  seg_hist: digits * 256 zeroed counters per
// segment; desc: digits * desc_stride zeroed descriptors (desc_stride as for
// launch_radix_sort32 over the capacity).  *which: the buffer with the result.
cudaError_t launch_radix_sort32_segmented(cudaStream_t st, const StepParams* sp, int first_digit, int digits,
                                          unsigned long long capacity, unsigned long long seg_keys, unsigned* keys0,
                                          unsigned* vals0, unsigned* keys1, unsigned* vals1,
                                          unsigned long long* desc, unsigned long long desc_stride,
                                          unsigned* seg_hist, Control* ctrl, int* which);
// Ranges of global tile ids (the view's tile_base + local id) over pairs
// sorted stably by local tile id from a view-grouped emission: a key holds the
// local id in its low 8 * (sort_passes - kDepthDigits) bits and the view above.
cudaError_t launch_tile_ranges_views(cudaStream_t st, unsigned long long capacity, const unsigned* tiles_sorted,
                                     const StepParams* views, unsigned* ranges, Control* ctrl);

// Heavy-first permutation of the tiles (by pair count, in power-of-two
// buckets) for the rasterisers.  Above 65536 tiles (several views) it runs as
// two grid-wide kernels with scratch in ctrl->tile_bucket (zeroed with the
// control block at the start of a step).
cudaError_t launch_tile_order(cudaStream_t st, const unsigned* ranges, int num_tiles, unsigned* order,
                              Control* ctrl = nullptr);

// Bounded-wait self-test: desc2 = two zeroed descriptors.
// Zeroes up to four device regions (8-byte aligned, sizes in 8-byte words; a
// null pointer or zero size skips a region) in one launch: the per-step
// clearing of control block, tile ranges and look-back descriptors.
struct ClearRegions {
    unsigned long long* p[4];
    unsigned long long words[4];
};
cudaError_t launch_clear_regions(cudaStream_t st, const ClearRegions& r);
cudaError_t launch_wait_selftest(cudaStream_t st, unsigned long long* desc2, unsigned* status, unsigned spin_limit);

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // keys per onesweep CTA

}  // namespace gs3d
