/*
 * gs3d_cuda.h -- C ABI of the B200 (sm_100a) 3D Gaussian Splatting hot path.
 *
 * One context owns one CUDA stream on one device and every device buffer of
 * the path (model, Adam moments, screen-space records, tile/depth pairs, tile
 * ranges, per-pixel state).  Calls are stream-ordered and synchronous towards
 * the caller: a call that fills host arrays returns once they are filled.
 * A context is not thread-safe; use one per host thread.
 *
 * Every entry point returns a status (GS3DC_OK == 0).  gs3dc_last_error()
 * gives the message of the last failure.  There is no CPU fallback: without a
 * usable sm_100 device gs3dc_create fails.
 *
 * The structs are the reference's own layouts (gs3d_types.h).  Each entry point
 * names the harmonyos_3dgs interface it stands in for; paths are relative to
 * the harmonyos_3dgs project root.
 */
#ifndef GS3D_CUDA_H
#define GS3D_CUDA_H

#include <stddef.h>
#include <stdint.h>
#include "gs3d_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gs3dc_ctx gs3dc_ctx;

/* ---- status codes ---- */
#define GS3DC_OK                 0
#define GS3DC_ERR_INVALID_ARG    1  /* bad size, NULL where required, unsupported config */
#define GS3DC_ERR_CUDA           2  /* a CUDA runtime call failed (message has details) */
#define GS3DC_ERR_PAIR_OVERFLOW  3  /* more tile pairs than the pair capacity could grow to */
#define GS3DC_ERR_DEVICE_TIMEOUT 4  /* a bounded device-side wait gave up (no hang) */
#define GS3DC_ERR_NO_MODEL       5  /* the call needs a model that was not uploaded */
#define GS3DC_ERR_OUT_OF_MEMORY  6  /* device allocation failed */
#define GS3DC_ERR_STATE          7  /* the call needs a stage that has not run */

/* ---- options (gs3dc_set_option) ---- */
#define GS3DC_OPT_PAIR_CAPACITY  1  /* minimum tile-pair capacity to preallocate */
#define GS3DC_OPT_USE_GRAPH      2  /* 1: gs3dc_train_step replays a captured CUDA graph (default 1) */
#define GS3DC_OPT_FORM           3  /* GS3DC_FORM_* precision form of gs3dc_train_step / gs3dc_render */
#define GS3DC_OPT_SPIN_LIMIT     4  /* iterations before a device-side wait gives up (test hook) */
#define GS3DC_OPT_STAGE_TIMING   5  /* 1: train steps run un-captured with CUDA events between stages */
#define GS3DC_OPT_FUSED_ADAM     6  /* 1: optimiser fused into the preprocess backward; 0 (default): split */
#define GS3DC_OPT_SORT           7  /* GS3DC_SORT_*: how gs3dc_train_step orders its pairs (same result) */
#define GS3DC_OPT_KEEP_GRADIENTS 8  /* 1: gs3dc_train_step keeps its raw-parameter gradients (gs3dc_get_gradients) */
#define GS3DC_OPT_AUTOTUNE       9  /* 1: tune the rasterisers online: per workload shape the first 6 train steps try
                                       1 / 2 / 4 pixels per thread (threads per tile 256 / 128 / 64) twice each, the
                                       next 4 the staging batch 64 / 256 against 128 at the fastest ones (timed with
                                       events, un-captured); the fastest forward / backward settings stay;
                                       0 (default): 2 pixels per thread, batch 128 */
#define GS3DC_OPT_DENSITY_SEED  10  /* state of the density controller's split sampler (LCG); 12345 at creation,
                                        like DensityController::rng_state_ (density_controller.h:41) */
#define GS3DC_OPT_RASTER_PPT    11  /* 1, 2 or 4: the rasterisers' pixels per thread in train steps, fixed (the
                                       autotuner then stays off); 0 (default): 2, or the autotuner's pick */
#define GS3DC_OPT_RASTER_BATCH  12  /* 64, 128 or 256: the records the rasterisers stage per round in train steps,
                                       fixed together with GS3DC_OPT_RASTER_PPT; 0 (default): 128 */

/* Depth-first (default): the Gaussians are stably sorted by depth, their pairs
 * emitted in that order and stably sorted by the tile bits alone.  Full key:
 * pairs emitted in Gaussian order and sorted on all tile and depth bits. */
#define GS3DC_SORT_DEPTH_FIRST   0
#define GS3DC_SORT_FULL_KEY      1

#define GS3DC_FORM_PLAIN_FP32    0  /* FP32 everywhere, no FMA contraction: parity form */
/* Reduced storage ("chosen" form) of gs3dc_train_step: positions FP32; raw
 * scales, opacity, rotation and SH coefficients 16-bit; Adam moments BF16 (FP32
 * for positions); FP32 blending and gradients with FMA and fast exp; tile
 * rectangles cut to where alpha can reach 1/255; parameters written back with
 * stochastic rounding.  gs3dc_set_raw_params / gs3dc_get_raw_params convert
 * from / to FP32.  The stage calls (preprocess ... optimizer_step, render)
 * need the plain form.  Changing the form keeps the model (converted) and
 * restarts the optimiser state. */
#define GS3DC_FORM_BF16          1
#define GS3DC_FORM_FP16          2

/* ---- statistics (gs3dc_get_stat) ---- */
#define GS3DC_STAT_TOTAL_PAIRS    1  /* tile pairs of the last forward */
#define GS3DC_STAT_PAIR_CAPACITY  2
#define GS3DC_STAT_KERNELS_LAST   3  /* kernels launched by the last train step / render */
#define GS3DC_STAT_SORT_PASSES    4  /* radix passes of the last sort */
#define GS3DC_STAT_GRAPH_REPLAYS  5  /* train steps replayed from a captured graph */
#define GS3DC_STAT_ADAM_STEP      6  /* Adam step counter (AdamOptimizer::step_count) */
#define GS3DC_STAT_FWD_PPT        7  /* pixels per thread of the forward rasteriser in the last train step */
#define GS3DC_STAT_BWD_PPT        8  /* pixels per thread of the backward rasteriser in the last train step */
#define GS3DC_STAT_NUM_GAUSSIANS  9  /* Gaussians of the device model (changes with density control) */
#define GS3DC_STAT_SCREEN_GAUSSIANS 10 /* Gaussians of the current screen records (the model's, or those of
                                          gs3dc_rasterize_arrays): the length of the raster gradients */
#define GS3DC_STAT_GRAPH_CAPTURES 11 /* train-step graphs captured (one per workload shape that repeats;
                                        the single-view step keeps the graphs of up to 8 shapes) */
#define GS3DC_STAT_FWD_BATCH     12  /* records the forward rasteriser stages per round in the last train step */
#define GS3DC_STAT_BWD_BATCH     13  /* records the backward rasteriser stages per round in the last train step */

/* Host arrays of PreprocessOutput + the per-Gaussian ForwardCache fields
 * (include/types.h:69-82, 97-107).  Any pointer may be NULL (not produced). */
typedef struct gs3dc_screen_arrays {
    float* means2D;       /* [N*2] */
    float* depths;        /* [N] */
    float* conics;        /* [N*3] */
    float* opacities_2d;  /* [N] */
    float* rgb;           /* [N*3] */
    int* radii;           /* [N] */
    int* tiles_touched;   /* [N] */
    float* cov3D;         /* [N*6] */
    float* p_view;        /* [N*3] */
    float* p_hom_w;       /* [N] */
    float* cov2D;         /* [N*3] after the +0.3 filter */
    float* cov2D_det;     /* [N] */
    /* RenderConfig::eval_3D only (PreprocessOutput, include/types.h:77-79):
     * gs3dc_preprocess fills them; gs3dc_bin reads cov3D_inv and mean_offset */
    float* gauss2screen;  /* [N*16] row-major, zero for culled Gaussians */
    float* cov3D_inv;     /* [N*6] inverse 3D covariance, upper triangle */
    float* mean_offset;   /* [N*3] position - camera position */
} gs3dc_screen_arrays;

/* ---- context ---- */
int gs3dc_create(int device, gs3dc_ctx** out);
void gs3dc_destroy(gs3dc_ctx* ctx);
const char* gs3dc_last_error(const gs3dc_ctx* ctx);
const char* gs3dc_status_string(int status);
/* The cudaStream_t every call of this context is ordered on. */
int gs3dc_get_stream(gs3dc_ctx* ctx, void** stream);
int gs3dc_set_option(gs3dc_ctx* ctx, int option, int64_t value);
int gs3dc_get_stat(gs3dc_ctx* ctx, int stat, int64_t* value);

/* ---- model ----
 * gs3dc_set_gaussians: an activated model for rendering (GaussianData,
 *   include/types.h:34-45); replaces the device copy every call.
 * gs3dc_set_raw_params: the trainable model (RawGaussianParams,
 *   include/train_types.h:9-22); zeroes the Adam moments and step counter like
 *   AdamOptimizer::reset (src/optimizer.cpp:45-58).
 * gs3dc_get_raw_params: copies the device parameters into the host arrays of
 *   raw (same count / max_coeffs as uploaded). */
int gs3dc_set_gaussians(gs3dc_ctx* ctx, const gs3d_gaussians* g);
int gs3dc_set_raw_params(gs3dc_ctx* ctx, const gs3d_raw_params* raw);
int gs3dc_get_raw_params(gs3dc_ctx* ctx, gs3d_raw_params* raw);
/* New values for the uploaded raw model (same count / max_coeffs), Adam state
 * kept: the host side of Trainer::step, which reads the caller's parameters on
 * every call (src/trainer.cpp:26-36) while AdamOptimizer keeps its moments
 * unless N changes (src/optimizer.cpp:64-66). */
int gs3dc_update_raw_params(gs3dc_ctx* ctx, const gs3d_raw_params* raw);
/* The H*W*3 image of the last rasterize / render / train step
 * (Trainer::last_rendered, include/trainer.h:32). */
int gs3dc_get_image(gs3dc_ctx* ctx, float* image);

/* ---- forward stages ----
 * Preprocessor::process (include/preprocessor.h:7-12; CPU src/cpu/preprocessor_cpu.cpp:11-268).
 *   Projects the current model (activated, or the raw model activated on the
 *   device), computes radii / tiles_touched, the prefix sum and the tile
 *   pairs.  `out` (may be NULL) receives host copies. */
int gs3dc_preprocess(gs3dc_ctx* ctx, const gs3d_camera* cam, const gs3d_render_config* cfg,
                     const gs3dc_screen_arrays* out);

/* TileBinner::bin (include/tile_binner.h:7-12; src/cpu/tile_binner_cpu.cpp:6-102).
 *   in == NULL: the pairs of the last gs3dc_preprocess.  in != NULL: bins the
 *   host arrays means2D / depths / radii / tiles_touched of N Gaussians
 *   (uploaded first).  Writes the pair count and, if non-NULL, the unsorted
 *   keys ((tile << 32) | depth bits) and values (Gaussian index), Gaussian-major
 *   and row-major inside each rect like the reference. */
int gs3dc_bin(gs3dc_ctx* ctx, int num_gaussians, const gs3dc_screen_arrays* in,
              const gs3d_camera* cam, const gs3d_render_config* cfg, int64_t* total_pairs,
              uint64_t* keys_unsorted, uint32_t* values_unsorted);

/* Sorter::sort (include/sorter.h:7; src/cpu/sorter_cpu.cpp:6-44).
 *   Stable LSD radix sort of the current pairs by key, then tile ranges.
 *   Host outputs may be NULL.  tile_ranges has 2*num_tiles entries
 *   (start, end), zero for empty tiles. */
int gs3dc_sort(gs3dc_ctx* ctx, uint64_t* keys_sorted, uint32_t* values_sorted,
               uint32_t* tile_ranges);

/* Sorter::sort on caller-provided pairs (the SorterCPU unit-test form, where
 * keys need not come from a camera).  Keys' tile fields must be < num_tiles. */
int gs3dc_sort_pairs(gs3dc_ctx* ctx, int64_t total_pairs, const uint64_t* keys,
                     const uint32_t* values, int num_tiles, uint64_t* keys_sorted,
                     uint32_t* values_sorted, uint32_t* tile_ranges);

/* gs3dc_sort_pairs without any device-memory allocation: no counterpart in the
 * reference.  For callers that must not allocate on their path -- code holding
 * no gs3dc context (creating one allocates), frame loops under a fixed
 * device-memory budget, callers that cannot take the device-wide
 * synchronisation of cudaMalloc / cudaFree.
 *   keys, values, keys_sorted, values_sorted (total_pairs entries) and
 *   tile_ranges (2*num_tiles entries) are device memory of the current device;
 *   the inputs are left unchanged, or keys_sorted / values_sorted may be
 *   exactly the keys / values buffers (in place); any other overlap between
 *   the five buffers is refused (GS3DC_ERR_INVALID_ARG).
 *   The scratch is one static device array of about 16 MiB per device, so
 *   total_pairs may not exceed GS3DC_STATIC_SORT_MAX_PAIRS
 *   (GS3DC_ERR_INVALID_ARG otherwise).  All calls on a device share it: calls
 *   that overlap on the GPU race.  Every call looks up the scratch's device
 *   address on the current device, so a device reset leaves nothing stale.
 *   Runs on `stream` (a cudaStream_t, NULL = default stream) and returns once
 *   the sort is done: the call waits for the stream and reads a status word
 *   back, so it cannot be captured into a CUDA graph (on a capturing stream it
 *   returns GS3DC_ERR_INVALID_ARG and does nothing).
 *   err (may be NULL) receives a message of at most err_len bytes on failure. */
#define GS3DC_STATIC_SORT_MAX_PAIRS 1048576
int gs3dc_sort_pairs_static(int64_t total_pairs, const uint64_t* keys, const uint32_t* values,
                            int num_tiles, uint64_t* keys_sorted, uint32_t* values_sorted,
                            uint32_t* tile_ranges, void* stream, char* err, size_t err_len);

/* Rasterizer::rasterize (include/rasterizer.h:7-15; src/cpu/rasterizer_cpu.cpp:38-198).
 *   Front-to-back blend of the sorted pairs.  image is H*W*3 HWC; T_final and
 *   n_contrib (ForwardCache, include/types.h:98-99) may be NULL. */
int gs3dc_rasterize(gs3dc_ctx* ctx, const gs3d_camera* cam, const gs3d_render_config* cfg,
                    float* image, float* T_final, int* n_contrib);

/* Rasterizer::rasterize on a caller's own PreprocessOutput / BinningOutput
 * (include/rasterizer.h:7-15; src/cpu/rasterizer_cpu.cpp:38-198): the screen
 * arrays means2D, conics, opacities_2d, rgb of num_gaussians Gaussians, the
 * sorted values and the 2*num_tiles tile ranges (num_tiles = the camera's
 * 16x16 grid) are uploaded and blended.  Every value must be below
 * num_gaussians and every range inside [0, total_pairs) (checked on the host).
 * gs3dc_raster_backward may follow; gs3dc_preprocess_backward may not (there
 * is no device model behind these records).  The 2D mode only. */
int gs3dc_rasterize_arrays(gs3dc_ctx* ctx, int num_gaussians, const gs3dc_screen_arrays* in,
                           int64_t total_pairs, const uint32_t* values_sorted, int num_tiles,
                           const uint32_t* tile_ranges, const gs3d_camera* cam,
                           const gs3d_render_config* cfg, float* image, float* T_final, int* n_contrib);

/* Renderer::render (include/renderer.h:17-21; src/renderer.cpp:13-39):
 *   g (may be NULL to reuse the uploaded model) -> preprocess -> bin -> sort ->
 *   rasterize -> image (host, H*W*3). */
int gs3dc_render(gs3dc_ctx* ctx, const gs3d_gaussians* g, const gs3d_camera* cam,
                 const gs3d_render_config* cfg, float* image);

/* ---- backward stages ----
 * RasterizerBackwardCPU::backward (src/cpu/rasterizer_backward_cpu.h:7-10;
 *   src/cpu/rasterizer_backward_cpu.cpp:7-138) for the last rasterize, with
 *   d_image given on the host (H*W*3).  Outputs RasterGradOutput
 *   (include/train_types.h:25-32), any may be NULL. */
int gs3dc_raster_backward(gs3dc_ctx* ctx, const gs3d_camera* cam, const gs3d_render_config* cfg,
                          const float* d_image, float* d_means2D, float* d_conics, float* d_rgb,
                          float* d_opacities_2d);

/* The same backward with the reference's stored per-pixel contributor lists
 * (src/cpu/rasterizer_backward_cpu.cpp:40-67: the forward replayed into a list
 * of (Gaussian, alpha) per pixel, walked back to front), kept to measure what
 * the lists cost against gs3dc_raster_backward, which recovers transmittance
 * by division and keeps no list.  The lists live in one device buffer of
 * sum(n_contrib) entries of 8 bytes plus a 4-byte offset per pixel;
 * *list_bytes (may be NULL) receives that size.  Outputs as
 * gs3dc_raster_backward. */
int gs3dc_raster_backward_lists(gs3dc_ctx* ctx, const gs3d_camera* cam, const gs3d_render_config* cfg,
                                const float* d_image, float* d_means2D, float* d_conics, float* d_rgb,
                                float* d_opacities_2d, int64_t* list_bytes);

/* PreprocessorBackwardCPU::backward (src/cpu/preprocessor_backward_cpu.h:7-10;
 *   src/cpu/preprocessor_backward_cpu.cpp:205-645) from the last raster
 *   backward.  With a raw device model the activation is recomputed; with an
 *   activated one (gs3dc_set_gaussians, as a PreprocessorCUDA forward leaves it)
 *   raw_rotations (host, N*4) supplies the unnormalised quaternions the
 *   normalisation backward needs.  Outputs GradientOutput
 *   (include/train_types.h:35-43), any may be NULL. */
int gs3dc_preprocess_backward(gs3dc_ctx* ctx, const gs3d_camera* cam,
                              const gs3d_render_config* cfg, const float* raw_rotations,
                              float* d_raw_positions, float* d_raw_scales, float* d_raw_rotations,
                              float* d_raw_sh_coeffs, float* d_raw_opacities);

/* AdamOptimizer::step / SGDOptimizer::step (src/optimizer.cpp:9-101) with the
 *   gradients of the last gs3dc_preprocess_backward, on the device model. */
int gs3dc_optimizer_step(gs3dc_ctx* ctx, const gs3d_train_config* tc, int iteration);

/* Trainer::step (include/trainer.h:21-23; src/trainer.cpp:7-70) with the
 *   parameters resident on the device: activate, forward, L1 loss, backward,
 *   optimiser, fused into a few kernels and replayed as one CUDA graph.
 *   Graphs are kept per workload shape (camera size, model size, form;
 *   up to 8 shapes, least recently used replaced), so a caller cycling through
 *   cameras of several sizes replays each size's graph.  A shape's first step
 *   runs un-captured and waits for the device (a pair-capacity overflow is
 *   redone at once).
 *   gt is H*W*3 HWC; gt_on_device != 0 means it is a device pointer.  A host
 *   gt is copied on the context's copy stream (pinned memory makes that copy
 *   asynchronous) while the step's preprocess, sort and forward rasteriser
 *   run; the L1 and the backward follow once it has landed.  The host buffer
 *   may be reused when the call returns with a non-NULL loss; with a NULL loss
 *   the copy may still be running, so keep the buffer unchanged until the next
 *   synchronising call.
 *   loss (may be NULL) receives the mean absolute error; a NULL loss also lets
 *   the call return without waiting for the device (the next call, or
 *   gs3dc_get_raw_params, synchronises). */
int gs3dc_train_step(gs3dc_ctx* ctx, const gs3d_camera* cam, const float* gt, int gt_on_device,
                     const gs3d_render_config* cfg, const gs3d_train_config* tc, int iteration,
                     float* loss);

/* One training step over several views at once (no reference counterpart: the
 * reference's Trainer::step takes one camera).  n_views cameras (1..255, any
 * mix of resolutions), gt = their targets concatenated (view-major, each
 * H*W*3 HWC; gt_on_device != 0: a device pointer).  The loss is the mean over
 * the views of each view's L1 mean; one Adam step follows the gradients summed
 * that way.  Runs in the reduced-storage form (GS3DC_FORM_BF16 / _FP16): every
 * (view, Gaussian) is preprocessed, sorted by (view, depth), emitted with
 * global (view, tile) ids and tile-sorted once; persistent rasterisers take the
 * views' tiles heavy-first from a work counter; the whole step is replayed as
 * one CUDA graph once its shape (views' sizes, N) repeats.  loss may be NULL
 * (no wait for the device, as gs3dc_train_step). */
int gs3dc_train_step_batch(gs3dc_ctx* ctx, int n_views, const gs3d_camera* cams, const float* gt,
                           int gt_on_device, const gs3d_render_config* cfg,
                           const gs3d_train_config* tc, int iteration, float* loss);

/* The forward image of view `view` (H*W*3 HWC, that view's camera size) of the
 * last gs3dc_train_step_batch: Trainer::step's rendered image (last_rendered_,
 * src/trainer.cpp:46-48) for each of the step's cameras.  Synchronous. */
int gs3dc_get_batch_image(gs3dc_ctx* ctx, int view, float* image);

/* Device time per stage of the last train step run with GS3DC_OPT_STAGE_TIMING,
 * measured with CUDA events on the context's stream.  ms[k] for k < n_stages,
 * indexed by GS3DC_STAGE_*. */
#define GS3DC_STAGE_MEMSETS        0  /* clearing of the control block, sort scratch, tile ranges (one kernel in the train step) */
#define GS3DC_STAGE_PREPROCESS     1  /* activation + projection + scan + pair emission */
#define GS3DC_STAGE_SORT_HIST      2  /* digit histograms; depth-first: also the Gaussian depth sort + pair emission */
#define GS3DC_STAGE_SORT_PASSES    3  /* all onesweep passes over the pairs together */
#define GS3DC_STAGE_RANGES         4
#define GS3DC_STAGE_RASTER_FWD     5  /* incl. the fused L1 */
#define GS3DC_STAGE_RASTER_BWD     6
#define GS3DC_STAGE_PREPROCESS_BWD 7  /* incl. the fused optimiser */
#define GS3DC_NUM_STAGES           8
int gs3dc_get_stage_times(gs3dc_ctx* ctx, float* ms, int n_stages);

/* Runs one device-side wait on a flag that nothing sets, bounded by spin_limit
 * polls (1..2^24).  Returns GS3DC_ERR_DEVICE_TIMEOUT when the bound works; the
 * context stays usable afterwards.  No reference counterpart: it exercises the
 * bounded-wait failure path that every look-back of this library relies on. */
int gs3dc_selftest_bounded_wait(gs3dc_ctx* ctx, uint32_t spin_limit);

/* The raw-parameter gradients (FP32, reference layouts) of the last
 * gs3dc_train_step run with GS3DC_OPT_KEEP_GRADIENTS.  No reference
 * counterpart: Trainer::step keeps its GradientOutput internal.  Host arrays
 * may be NULL. */
int gs3dc_get_gradients(gs3dc_ctx* ctx, float* d_raw_positions, float* d_raw_scales,
                        float* d_raw_rotations, float* d_raw_sh_coeffs, float* d_raw_opacities);

/* ---- adaptive density control (plain FP32 form, raw model) ----
 * The trainer's DensityController (src/density_controller.h:6-43,
 * density_controller.cpp:9-204), its statistics kept on the device.
 * gs3dc_density_accumulate: DensityController::accumulate_stats.  d_means2D
 *   ([N*2] host) and radii ([N] host, may be NULL); with d_means2D == NULL the
 *   device's d_means2D of the last gs3dc_raster_backward and the radii of the
 *   last gs3dc_preprocess are used.  The statistics restart when N changes
 *   and with every gs3dc_set_raw_params.
 * gs3dc_densify_and_prune: DensityController::densify_and_prune: clone, split
 *   (children appended after the clones, sampled from the controller's LCG,
 *   seed 12345 per context), prune, compact; the Adam moments and step reset
 *   when the count changes, like Trainer::step_with_densify (trainer.cpp:152-163).
 *   *new_count = the new N (read the model with gs3dc_get_raw_params and
 *   GS3DC_STAT_NUM_GAUSSIANS).  Every split child is kept: the reference's
 *   compaction reads its removal mask past the end for them
 *   (density_controller.cpp:78, train_types.h:119-124), so which survive
 *   there depends on heap contents.
 * gs3dc_reset_opacity: DensityController::reset_opacity (all raw opacities =
 *   inverse_sigmoid(0.01)).
 * gs3dc_train_step_densify: Trainer::step_with_densify (trainer.cpp:72-175): a
 *   train step, the statistics pass (forward + raster backward of the updated
 *   model), densify_and_prune on its iterations, opacity reset on its
 *   iterations; *n_gaussians = the count afterwards. */
int gs3dc_density_accumulate(gs3dc_ctx* ctx, const float* d_means2D, const int* radii);
int gs3dc_densify_and_prune(gs3dc_ctx* ctx, const gs3d_densify_config* cfg, float scene_extent, int* new_count);
int gs3dc_reset_opacity(gs3dc_ctx* ctx);
int gs3dc_train_step_densify(gs3dc_ctx* ctx, const gs3d_camera* cam, const float* gt, int gt_on_device,
                             const gs3d_render_config* cfg, const gs3d_train_config* tcfg,
                             const gs3d_densify_config* dcfg, float scene_extent, int iteration, float* loss,
                             int* n_gaussians);

/* ---- on-disk formats of the reference's drivers (host functions, no context) ----
 * gs3dc_ply_info / gs3dc_ply_read: loadPly (src/ply_loader.cpp:31-189): a binary
 *   little-endian 3DGS PLY; SH degree from the f_rest count; SH reordered from
 *   channel-first to basis-interleaved.  activate != 0: the loader's activations
 *   (sigmoid opacity, exp scale, normalised quaternion) -> GaussianData; 0: the
 *   stored values -> the arrays of g (same layout) without activation.
 *   g->count / g->max_coeffs must be gs3dc_ply_info's; g->filter_3D may be NULL.
 * gs3dc_ply_write: savePly of the train driver (src/train_main.cpp:82-138),
 *   byte for byte.
 * gs3dc_raw_from_gaussians: initRawFromGaussianData (src/train_main.cpp:26-65):
 *   log(max(1e-12, scale)), inverse_sigmoid of the clamped opacity.
 * gs3dc_cameras_read: loadCamerasJson (src/train_main.cpp:262-375): every camera
 *   object (fx, fy > 0, with position and camera-to-world rotation) of a 3DGS
 *   cameras.json, in file order, as view / view-projection matrices (znear 0.01,
 *   zfar 100); names (optional) receives img_name, name_len bytes per camera;
 *   *n_cams = cameras found (only the first max_cams are written).
 * gs3dc_ppm_read / gs3dc_ppm_write: readPPM / writePPM (src/image_io.cpp:9-68):
 *   8-bit P6; image == NULL reads the size only.
 * gs3dc_image_resize_nearest: the train driver's target resize
 *   (src/train_main.cpp:536-548).
 * gs3dc_io_last_error: message of the last failed call of this group (per thread). */
int gs3dc_ply_info(const char* path, int* count, int* sh_degree, int* max_coeffs, int* has_filter_3D);
int gs3dc_ply_read(const char* path, int activate, gs3d_gaussians* g);
int gs3dc_ply_write(const char* path, const gs3d_raw_params* raw);
int gs3dc_raw_from_gaussians(const gs3d_gaussians* g, gs3d_raw_params* raw);
int gs3dc_cameras_read(const char* path, gs3d_camera* cams, char* names, int name_len, int max_cams,
                       int* n_cams);
int gs3dc_ppm_read(const char* path, float* image, int* width, int* height);
int gs3dc_ppm_write(const char* path, const float* image, int width, int height);
int gs3dc_image_resize_nearest(const float* src, int src_w, int src_h, float* dst, int dst_w, int dst_h);
const char* gs3dc_io_last_error(void);

/* Checkpoint / resume of the whole training state: the model in its current
 * form's storage (FP32, or the 16-bit arrays), the optimiser moments and the
 * Adam step counter, so that a resumed run continues exactly where the saved
 * one stopped.  No reference counterpart (the reference's train driver saves
 * the parameters only, src/train_main.cpp:670-674).  gs3dc_load_state
 * replaces the model and switches the context to the saved form. */
int gs3dc_save_state(gs3dc_ctx* ctx, const char* path);
int gs3dc_load_state(gs3dc_ctx* ctx, const char* path);

/* Blocks until every call issued on the context's stream has finished and
 * reports any deferred device-side error (pair overflow, timeout). */
int gs3dc_synchronize(gs3dc_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* GS3D_CUDA_H */
