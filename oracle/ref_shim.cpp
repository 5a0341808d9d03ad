// ref_shim.cpp -- TEST INFRASTRUCTURE.  A C ABI over the reference's own CPU
// stage classes (harmonyos_3dgs src/cpu/*, trainer.cpp, renderer.cpp), linked
// with the reference sources compiled where they lie into
// oracle/_ref/libgs3d_ref.so by oracle/Makefile.  Nothing here reimplements
// the reference: every number comes from its classes.
//
//   ref_forward      PreprocessorCPU -> TileBinnerCPU -> SorterCPU -> RasterizerCPU
//                    (the sequence of Renderer::render, renderer.cpp:13-39, with the
//                    ForwardCache of Trainer::step, trainer.cpp:38-48)
//   ref_train_step   Trainer::step's sequence (trainer.cpp:7-70) with every
//                    intermediate copied out, Adam state kept in a handle
//   ref_trainer_*    the unmodified Trainer class (timing baseline)
//   ref_renderer_*   the unmodified Renderer with the CPU stages (timing baseline)
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "types.h"
#include "train_types.h"
#include "renderer.h"
#include "trainer.h"
#include "loss.h"
#include "optimizer.h"
#include "cpu/preprocessor_cpu.h"
#include "cpu/tile_binner_cpu.h"
#include "cpu/sorter_cpu.h"
#include "cpu/rasterizer_cpu.h"
#include "cpu/rasterizer_backward_cpu.h"
#include "cpu/preprocessor_backward_cpu.h"
#include "density_controller.h"

#include "gs3d_oracle.h"

static_assert(sizeof(Camera) == sizeof(gs3d_camera), "Camera layout");
static_assert(sizeof(RenderConfig) == sizeof(gs3d_render_config), "RenderConfig layout");
static_assert(sizeof(GaussianData) == sizeof(gs3d_gaussians), "GaussianData layout");
static_assert(sizeof(TrainConfig) == sizeof(gs3d_train_config), "TrainConfig layout");
static_assert(sizeof(RawGaussianParams) == sizeof(gs3d_raw_params), "RawGaussianParams layout");
static_assert(sizeof(DensifyConfig) == sizeof(gs3d_densify_config), "DensifyConfig layout");
static_assert(offsetof(DensifyConfig, enabled) == offsetof(gs3d_densify_config, enabled), "DensifyConfig layout");

namespace {

void copy_forward(int N, const PreprocessOutput& pre, const ForwardCache& cache,
                  const BinningOutput& bin, int num_pixels, const float* img, orc_step_io* io) {
    std::memcpy(io->means2D, pre.means2D, sizeof(float) * 2 * N);
    std::memcpy(io->depths, pre.depths, sizeof(float) * N);
    std::memcpy(io->conics, pre.conics, sizeof(float) * 3 * N);
    std::memcpy(io->opac2d, pre.opacities_2d, sizeof(float) * N);
    std::memcpy(io->rgb, pre.rgb, sizeof(float) * 3 * N);
    std::memcpy(io->radii, pre.radii, sizeof(int) * N);
    std::memcpy(io->tiles, pre.tiles_touched, sizeof(int) * N);
    if (io->cov3D) {
        std::memcpy(io->cov3D, cache.cov3D, sizeof(float) * 6 * N);
        std::memcpy(io->p_view, cache.p_view, sizeof(float) * 3 * N);
        std::memcpy(io->p_hom_w, cache.p_hom_w, sizeof(float) * N);
        std::memcpy(io->cov2D, cache.cov2D, sizeof(float) * 3 * N);
        std::memcpy(io->det, cache.cov2D_det, sizeof(float) * N);
    }
    int64_t P = bin.total_pairs;
    if (P > 0) {
        std::memcpy(io->keys_unsorted, bin.keys_unsorted, sizeof(uint64_t) * P);
        std::memcpy(io->vals_unsorted, bin.values_unsorted, sizeof(uint32_t) * P);
        std::memcpy(io->keys_sorted, bin.keys_sorted, sizeof(uint64_t) * P);
        std::memcpy(io->vals_sorted, bin.values_sorted, sizeof(uint32_t) * P);
    }
    std::memcpy(io->ranges, bin.tile_ranges, sizeof(uint32_t) * 2 * bin.num_tiles);
    std::memcpy(io->image, img, sizeof(float) * 3 * num_pixels);
    if (io->T_final && cache.T_final) {
        std::memcpy(io->T_final, cache.T_final, sizeof(float) * num_pixels);
        std::memcpy(io->n_contrib, cache.n_contrib, sizeof(int) * num_pixels);
    }
}

// Runs the reference forward with a cache.  Returns 1 if io->pair_capacity is
// too small (io->total_pairs is set), else 0.
int run_forward(const GaussianData& g, const Camera& cam, const RenderConfig& cfg,
                FrameAllocator& alloc, PreprocessOutput& pre, BinningOutput& bin,
                ForwardCache& cache, float*& rendered, orc_step_io* io) {
    PreprocessorCPU pp;
    TileBinnerCPU tb;
    SorterCPU so;
    RasterizerCPU ra;
    cache = ForwardCache{};
    pre = pp.process(g, cam, cfg, alloc, &cache);
    bin = tb.bin(pre, g.count, cam, cfg, alloc);
    io->total_pairs = bin.total_pairs;
    if (bin.total_pairs > io->pair_capacity) return 1;
    if (bin.total_pairs > 0) so.sort(bin, alloc);
    cache.pre = &pre;
    cache.bin = &bin;
    int num_pixels = cam.width * cam.height;
    rendered = alloc.allocate_array<float>(num_pixels * 3);
    ra.rasterize(pre, bin, cam, cfg, rendered, nullptr, &cache, &alloc);
    return 0;
}

size_t arena_bytes(int N, int max_coeffs, int64_t P, int num_pixels) {
    size_t b = (size_t)N * (size_t)(60 + 4 * max_coeffs * 3) * 8 + (size_t)P * 40 +
               (size_t)num_pixels * 64 + (64u << 20);
    return b;
}

struct AdamHandle {
    AdamOptimizer adam;
};

}  // namespace

extern "C" {

int ref_forward(const gs3d_gaussians* gp, const gs3d_camera* camp, const gs3d_render_config* cfgp,
                orc_step_io* io) {
    const GaussianData& g = *reinterpret_cast<const GaussianData*>(gp);
    const Camera& cam = *reinterpret_cast<const Camera*>(camp);
    const RenderConfig& cfg = *reinterpret_cast<const RenderConfig*>(cfgp);
    int num_pixels = cam.width * cam.height;
    FrameAllocator alloc(arena_bytes(g.count, g.max_coeffs, io->pair_capacity, num_pixels));
    PreprocessOutput pre;
    BinningOutput bin;
    ForwardCache cache;
    float* rendered = nullptr;
    if (run_forward(g, cam, cfg, alloc, pre, bin, cache, rendered, io)) return 1;
    copy_forward(g.count, pre, cache, bin, num_pixels, rendered, io);
    return 0;
}

// The forward with cfg.eval_3D set (the reference's AAA-Gaussians mode): the
// same stage sequence, plus the mode's per-Gaussian gauss2screen, cov3D_inv
// and mean_offset arrays.  io->cov3D must be NULL (the mode keeps no 2D cache).
int ref_forward_eval3d(const gs3d_gaussians* gp, const gs3d_camera* camp, const gs3d_render_config* cfgp,
                       orc_step_io* io, float* g2s, float* cov3D_inv, float* mean_offset) {
    const GaussianData& g = *reinterpret_cast<const GaussianData*>(gp);
    const Camera& cam = *reinterpret_cast<const Camera*>(camp);
    const RenderConfig& cfg = *reinterpret_cast<const RenderConfig*>(cfgp);
    if (!cfg.eval_3D || io->cov3D) return 2;
    int num_pixels = cam.width * cam.height;
    FrameAllocator alloc(arena_bytes(g.count, g.max_coeffs, io->pair_capacity, num_pixels) +
                         (size_t)g.count * 25 * sizeof(float));
    PreprocessOutput pre;
    BinningOutput bin;
    ForwardCache cache;
    float* rendered = nullptr;
    if (run_forward(g, cam, cfg, alloc, pre, bin, cache, rendered, io)) return 1;
    copy_forward(g.count, pre, cache, bin, num_pixels, rendered, io);
    std::memcpy(g2s, pre.gauss2screen, sizeof(float) * 16 * (size_t)g.count);
    std::memcpy(cov3D_inv, pre.cov3D_inv, sizeof(float) * 6 * (size_t)g.count);
    std::memcpy(mean_offset, pre.mean_offset, sizeof(float) * 3 * (size_t)g.count);
    return 0;
}

// DensityController with the model it densifies (density_controller.cpp):
// accumulate, densify_and_prune and reset_opacity on an OwnedRawParams.
struct DcHandle {
    DensityController dc;
    OwnedRawParams owned;
};

void* ref_dc_create(void) { return new (std::nothrow) DcHandle(); }
void ref_dc_destroy(void* h) { delete static_cast<DcHandle*>(h); }

void ref_dc_set_model(void* hp, const gs3d_raw_params* rawp) {
    auto* h = static_cast<DcHandle*>(hp);
    const RawGaussianParams& r = *reinterpret_cast<const RawGaussianParams*>(rawp);
    h->owned.sh_degree = r.sh_degree;
    h->owned.max_coeffs = r.max_coeffs;
    const size_t n = (size_t)r.count, mc3 = (size_t)r.max_coeffs * 3;
    h->owned.positions.assign(r.raw_positions, r.raw_positions + 3 * n);
    h->owned.scales.assign(r.raw_scales, r.raw_scales + 3 * n);
    h->owned.rotations.assign(r.raw_rotations, r.raw_rotations + 4 * n);
    h->owned.sh_coeffs.assign(r.raw_sh_coeffs, r.raw_sh_coeffs + mc3 * n);
    h->owned.opacities.assign(r.raw_opacities, r.raw_opacities + n);
    // OwnedRawParams::append (train_types.h:108-116) pushes values read through
    // pointers into the same vectors; a reallocating push_back would leave the
    // rest of those reads dangling.  With room for the largest result
    // (N + clones + 2 x splits <= 3N) no push_back reallocates.
    h->owned.positions.reserve(9 * n);
    h->owned.scales.reserve(9 * n);
    h->owned.rotations.reserve(12 * n);
    h->owned.sh_coeffs.reserve(3 * mc3 * n);
    h->owned.opacities.reserve(3 * n);
}

void ref_dc_accumulate(void* hp, const float* d_means2D, const int* radii, int N) {
    static_cast<DcHandle*>(hp)->dc.accumulate_stats(d_means2D, radii, N);
}

int ref_dc_densify(void* hp, const gs3d_densify_config* cfg, float extent) {
    auto* h = static_cast<DcHandle*>(hp);
    return h->dc.densify_and_prune(h->owned, *reinterpret_cast<const DensifyConfig*>(cfg), extent);
}

void ref_dc_reset_opacity(void* hp) { DensityController::reset_opacity(static_cast<DcHandle*>(hp)->owned); }

// Copies the handle's model out (arrays sized for its count).
int ref_dc_get_model(void* hp, gs3d_raw_params* rawp) {
    auto* h = static_cast<DcHandle*>(hp);
    RawGaussianParams& r = *reinterpret_cast<RawGaussianParams*>(rawp);
    const size_t n = (size_t)h->owned.count(), mc3 = (size_t)h->owned.max_coeffs * 3;
    std::memcpy(r.raw_positions, h->owned.positions.data(), 12 * n);
    std::memcpy(r.raw_scales, h->owned.scales.data(), 12 * n);
    std::memcpy(r.raw_rotations, h->owned.rotations.data(), 16 * n);
    std::memcpy(r.raw_sh_coeffs, h->owned.sh_coeffs.data(), 4 * mc3 * n);
    std::memcpy(r.raw_opacities, h->owned.opacities.data(), 4 * n);
    return (int)n;
}

// RawGaussianParams::activate (train_types.cpp:6-36) into caller arrays.
void ref_activate(const gs3d_raw_params* rawp, gs3d_gaussians* gp) {
    reinterpret_cast<const RawGaussianParams*>(rawp)->activate(*reinterpret_cast<GaussianData*>(gp));
}

void* ref_adam_create(void) { return new (std::nothrow) AdamHandle(); }
void ref_adam_destroy(void* h) { delete static_cast<AdamHandle*>(h); }

// Trainer::step (trainer.cpp:7-70) with every intermediate copied into io.
int ref_train_step(void* adam_handle, gs3d_raw_params* rawp, const gs3d_camera* camp,
                   const float* gt, const gs3d_render_config* cfgp, const gs3d_train_config* tcp,
                   int iteration, orc_step_io* io) {
    RawGaussianParams& params = *reinterpret_cast<RawGaussianParams*>(rawp);
    const Camera& cam = *reinterpret_cast<const Camera*>(camp);
    const RenderConfig& cfg = *reinterpret_cast<const RenderConfig*>(cfgp);
    const TrainConfig& tc = *reinterpret_cast<const TrainConfig*>(tcp);
    int N = params.count, mc3 = params.max_coeffs * 3;
    int num_pixels = cam.width * cam.height;
    FrameAllocator alloc(arena_bytes(N, params.max_coeffs, io->pair_capacity, num_pixels));
    std::vector<float> ap(N * 3), as(N * 3), ar(N * 4), ash((size_t)N * mc3), ao(N);
    GaussianData g;
    g.count = N;
    g.sh_degree = params.sh_degree;
    g.max_coeffs = params.max_coeffs;
    g.positions = ap.data();
    g.scales = as.data();
    g.rotations = ar.data();
    g.sh_coeffs = ash.data();
    g.opacities = ao.data();
    g.filter_3D = nullptr;
    params.activate(g);
    PreprocessOutput pre;
    BinningOutput bin;
    ForwardCache cache;
    float* rendered = nullptr;
    if (run_forward(g, cam, cfg, alloc, pre, bin, cache, rendered, io)) return 1;
    copy_forward(N, pre, cache, bin, num_pixels, rendered, io);
    float* d_image = alloc.allocate_array<float>(num_pixels * 3);
    io->loss = l1_loss(rendered, gt, cam.height, cam.width, d_image);
    io->loss_acc64 = l1_loss_double(rendered, gt, cam.height, cam.width, d_image);
    std::memcpy(io->d_image, d_image, sizeof(float) * 3 * num_pixels);
    RasterGradOutput rgrad;
    rgrad.allocate_and_zero(alloc, N);
    RasterizerBackwardCPU rbw;
    rbw.backward(pre, bin, cam, cfg, cache, d_image, rgrad);
    std::memcpy(io->d_means2D, rgrad.d_means2D, sizeof(float) * 2 * N);
    std::memcpy(io->d_conics, rgrad.d_conics, sizeof(float) * 3 * N);
    std::memcpy(io->d_rgb, rgrad.d_rgb, sizeof(float) * 3 * N);
    std::memcpy(io->d_opac, rgrad.d_opacities_2d, sizeof(float) * N);
    GradientOutput grads;
    grads.allocate_and_zero(alloc, N, params.max_coeffs);
    PreprocessorBackwardCPU pbw;
    pbw.backward(g, cam, cfg, cache, rgrad, params, grads);
    std::memcpy(io->g_pos, grads.d_raw_positions, sizeof(float) * 3 * N);
    std::memcpy(io->g_sc, grads.d_raw_scales, sizeof(float) * 3 * N);
    std::memcpy(io->g_rot, grads.d_raw_rotations, sizeof(float) * 4 * N);
    std::memcpy(io->g_sh, grads.d_raw_sh_coeffs, sizeof(float) * (size_t)mc3 * N);
    std::memcpy(io->g_op, grads.d_raw_opacities, sizeof(float) * N);
    if (tc.use_adam) {
        static_cast<AdamHandle*>(adam_handle)->adam.step(params, grads, tc, iteration);
    } else {
        SGDOptimizer sgd;
        sgd.step(params, grads, tc, iteration);
    }
    return 0;
}

// The unmodified Trainer (trainer.h:14-50), for timing.
void* ref_trainer_create(size_t arena_bytes_) {
    try {
        return new Trainer(arena_bytes_);
    } catch (...) {
        return nullptr;
    }
}
void ref_trainer_destroy(void* t) { delete static_cast<Trainer*>(t); }
int ref_trainer_step(void* t, gs3d_raw_params* rawp, const gs3d_camera* camp, const float* gt,
                     const gs3d_render_config* cfgp, const gs3d_train_config* tcp, int iteration,
                     float* loss_out) {
    try {
        auto r = static_cast<Trainer*>(t)->step(*reinterpret_cast<RawGaussianParams*>(rawp),
                                                *reinterpret_cast<const Camera*>(camp), gt,
                                                *reinterpret_cast<const RenderConfig*>(cfgp),
                                                *reinterpret_cast<const TrainConfig*>(tcp), iteration);
        if (loss_out) *loss_out = r.loss;
        return 0;
    } catch (...) {
        return 1;
    }
}

// The unmodified Renderer with the CPU stages (renderer.h:9-29), for timing.
void* ref_renderer_create(size_t arena_bytes_) {
    try {
        return new Renderer(std::make_unique<PreprocessorCPU>(), std::make_unique<TileBinnerCPU>(),
                            std::make_unique<SorterCPU>(), std::make_unique<RasterizerCPU>(),
                            arena_bytes_);
    } catch (...) {
        return nullptr;
    }
}
void ref_renderer_destroy(void* r) { delete static_cast<Renderer*>(r); }
int ref_renderer_render(void* r, const gs3d_gaussians* gp, const gs3d_camera* camp,
                        const gs3d_render_config* cfgp, float* img) {
    try {
        static_cast<Renderer*>(r)->render(*reinterpret_cast<const GaussianData*>(gp),
                                          *reinterpret_cast<const Camera*>(camp),
                                          *reinterpret_cast<const RenderConfig*>(cfgp), img, nullptr);
        return 0;
    } catch (...) {
        return 1;
    }
}

}  // extern "C"
