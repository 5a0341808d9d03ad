// gs3d_stages_cuda.cpp -- the CUDA stage adapters (see gs3d_stages_cuda.hpp).
#include "gs3d_stages_cuda.hpp"

#include <cstddef>
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

static_assert(sizeof(GaussianData) == sizeof(gs3d_gaussians), "GaussianData layout");
static_assert(offsetof(GaussianData, filter_3D) == offsetof(gs3d_gaussians, filter_3D), "GaussianData layout");
static_assert(sizeof(Camera) == sizeof(gs3d_camera), "Camera layout");
static_assert(offsetof(Camera, height) == offsetof(gs3d_camera, height), "Camera layout");
static_assert(sizeof(RenderConfig) == sizeof(gs3d_render_config), "RenderConfig layout");
static_assert(offsetof(RenderConfig, tile_h) == offsetof(gs3d_render_config, tile_h), "RenderConfig layout");
static_assert(sizeof(RawGaussianParams) == sizeof(gs3d_raw_params), "RawGaussianParams layout");
static_assert(sizeof(TrainConfig) == sizeof(gs3d_train_config), "TrainConfig layout");
static_assert(offsetof(TrainConfig, adam_eps) == offsetof(gs3d_train_config, adam_eps), "TrainConfig layout");

namespace {

const gs3d_camera* C(const Camera& c) { return reinterpret_cast<const gs3d_camera*>(&c); }
const gs3d_render_config* C(const RenderConfig& c) { return reinterpret_cast<const gs3d_render_config*>(&c); }
const gs3d_gaussians* C(const GaussianData& g) { return reinterpret_cast<const gs3d_gaussians*>(&g); }
gs3d_raw_params* C(RawGaussianParams& r) { return reinterpret_cast<gs3d_raw_params*>(&r); }
const gs3d_train_config* C(const TrainConfig& t) { return reinterpret_cast<const gs3d_train_config*>(&t); }

int num_tiles(const Camera& cam, const RenderConfig& cfg) {
    return ((cam.width + cfg.tile_w - 1) / cfg.tile_w) * ((cam.height + cfg.tile_h - 1) / cfg.tile_h);
}

}  // namespace

CudaDevice::CudaDevice(int device) {
    const int rc = gs3dc_create(device, &ctx_);
    if (rc != GS3DC_OK)
        throw std::runtime_error(std::string("gs3dc_create: ") + gs3dc_status_string(rc) +
                                 " (a B200-class sm_100 GPU is required; there is no CPU fallback)");
}

CudaDevice::~CudaDevice() { gs3dc_destroy(ctx_); }

void CudaDevice::check(int status, const char* what) const {
    if (status != GS3DC_OK)
        throw std::runtime_error(std::string(what) + ": " + gs3dc_status_string(status) + ": " +
                                 gs3dc_last_error(ctx_));
}

// Preprocessor::process (src/cpu/preprocessor_cpu.cpp:11-268)
PreprocessOutput PreprocessorCUDA::process(const GaussianData& g, const Camera& cam, const RenderConfig& cfg,
                                           FrameAllocator& alloc, ForwardCache* cache) {
    dev_->check(gs3dc_set_gaussians(dev_->ctx(), C(g)), "upload model");
    const int N = g.count;
    PreprocessOutput out{};
    out.means2D = alloc.allocate_array<float>((size_t)N * 2);
    out.depths = alloc.allocate_array<float>(N);
    out.conics = alloc.allocate_array<float>((size_t)N * 3);
    out.opacities_2d = alloc.allocate_array<float>(N);
    out.rgb = alloc.allocate_array<float>((size_t)N * 3);
    out.radii = alloc.allocate_array<int>(N);
    out.tiles_touched = alloc.allocate_array<int>(N);
    out.gauss2screen = out.cov3D_inv = out.mean_offset = nullptr;
    out.eval_3D = cfg.eval_3D;
    gs3dc_screen_arrays a{};
    if (cfg.eval_3D) {   // the 3D mode's arrays (preprocessor_cpu.cpp:25-29); it keeps no 2D cache
        out.gauss2screen = alloc.allocate_array<float>((size_t)N * 16);
        out.cov3D_inv = alloc.allocate_array<float>((size_t)N * 6);
        out.mean_offset = alloc.allocate_array<float>((size_t)N * 3);
        a.gauss2screen = out.gauss2screen;
        a.cov3D_inv = out.cov3D_inv;
        a.mean_offset = out.mean_offset;
        cache = nullptr;
    }
    a.means2D = out.means2D;
    a.depths = out.depths;
    a.conics = out.conics;
    a.opacities_2d = out.opacities_2d;
    a.rgb = out.rgb;
    a.radii = out.radii;
    a.tiles_touched = out.tiles_touched;
    if (cache) {
        cache->cov3D = alloc.allocate_array<float>((size_t)N * 6);
        cache->p_view = alloc.allocate_array<float>((size_t)N * 3);
        cache->p_hom_w = alloc.allocate_array<float>(N);
        cache->cov2D = alloc.allocate_array<float>((size_t)N * 3);
        cache->cov2D_det = alloc.allocate_array<float>(N);
        a.cov3D = cache->cov3D;
        a.p_view = cache->p_view;
        a.p_hom_w = cache->p_hom_w;
        a.cov2D = cache->cov2D;
        a.cov2D_det = cache->cov2D_det;
    }
    dev_->check(gs3dc_preprocess(dev_->ctx(), C(cam), C(cfg), &a), "preprocess");
    out.device_data = dev_->ctx();
    return out;
}

// TileBinner::bin (src/cpu/tile_binner_cpu.cpp:6-102)
BinningOutput TileBinnerCUDA::bin(const PreprocessOutput& pre, int N, const Camera& cam, const RenderConfig& cfg,
                                  FrameAllocator& alloc) {
    BinningOutput out{};
    out.num_tiles = num_tiles(cam, cfg);
    int64_t P = 0;
    const bool on_device = pre.device_data == dev_->ctx();
    gs3dc_screen_arrays a{};
    if (!on_device) {
        a.means2D = pre.means2D;
        a.depths = pre.depths;
        a.radii = pre.radii;
        a.tiles_touched = pre.tiles_touched;
        a.cov3D_inv = pre.cov3D_inv;
        a.mean_offset = pre.mean_offset;
        int64_t total = 0;
        for (int i = 0; i < N; i++) total += pre.tiles_touched[i];
        out.keys_unsorted = total ? alloc.allocate_array<uint64_t>((size_t)total) : nullptr;
        out.values_unsorted = total ? alloc.allocate_array<uint32_t>((size_t)total) : nullptr;
        dev_->check(gs3dc_bin(dev_->ctx(), N, &a, C(cam), C(cfg), &P, out.keys_unsorted, out.values_unsorted),
                    "bin");
    } else {
        dev_->check(gs3dc_bin(dev_->ctx(), N, nullptr, C(cam), C(cfg), &P, nullptr, nullptr), "bin");
        if (P > 0 && host_keys_) {
            out.keys_unsorted = alloc.allocate_array<uint64_t>((size_t)P);
            out.values_unsorted = alloc.allocate_array<uint32_t>((size_t)P);
            dev_->check(gs3dc_bin(dev_->ctx(), N, nullptr, C(cam), C(cfg), &P, out.keys_unsorted,
                                  out.values_unsorted),
                        "bin (download)");
        }
    }
    if (P > 0x7fffffff) throw std::runtime_error("bin: more tile pairs than BinningOutput::total_pairs can hold");
    out.total_pairs = (int)P;
    if (P > 0) {
        out.keys_sorted = alloc.allocate_array<uint64_t>((size_t)P);
        out.values_sorted = alloc.allocate_array<uint32_t>((size_t)P);
    }
    out.tile_ranges = alloc.allocate_array<uint32_t>((size_t)out.num_tiles * 2);
    std::memset(out.tile_ranges, 0, sizeof(uint32_t) * 2 * out.num_tiles);
    out.device_data = dev_->ctx();
    return out;
}

// Sorter::sort (src/cpu/sorter_cpu.cpp:6-44)
void SorterCUDA::sort(BinningOutput& bin, FrameAllocator&) {
    if (bin.device_data == dev_->ctx()) {
        dev_->check(gs3dc_sort(dev_->ctx(), host_keys_ ? bin.keys_sorted : nullptr,
                               host_keys_ ? bin.values_sorted : nullptr, bin.tile_ranges),
                    "sort");
    } else {
        dev_->check(gs3dc_sort_pairs(dev_->ctx(), bin.total_pairs, bin.keys_unsorted, bin.values_unsorted,
                                     bin.num_tiles, bin.keys_sorted, bin.values_sorted, bin.tile_ranges),
                    "sort");
        bin.device_data = dev_->ctx();
    }
}

// Rasterizer::rasterize (src/cpu/rasterizer_cpu.cpp:9-203)
void RasterizerCUDA::rasterize(const PreprocessOutput& pre, const BinningOutput& bin, const Camera& cam,
                               const RenderConfig& cfg, float* img, float* depth, ForwardCache* cache,
                               FrameAllocator* alloc) {
    if (depth) throw std::runtime_error("rasterize: the inverse-depth output is not produced by the CUDA backend");
    float* T = nullptr;
    int* nc = nullptr;
    if (cache && alloc) {
        const size_t np = (size_t)cam.width * cam.height;
        cache->T_final = alloc->allocate_array<float>(np);
        cache->n_contrib = alloc->allocate_array<int>(np);
        T = cache->T_final;
        nc = cache->n_contrib;
    }
    if (pre.device_data == dev_->ctx() && bin.device_data == dev_->ctx()) {
        dev_->check(gs3dc_rasterize(dev_->ctx(), C(cam), C(cfg), img, T, nc), "rasterize");
        return;
    }
    // a caller's own screen arrays and sorted pairs (the reference's unit-test form)
    gs3dc_screen_arrays a{};
    a.means2D = pre.means2D;
    a.conics = pre.conics;
    a.opacities_2d = pre.opacities_2d;
    a.rgb = pre.rgb;
    int n = 0;
    for (uint32_t j = 0; j < (uint32_t)bin.total_pairs; j++)
        n = std::max(n, (int)bin.values_sorted[j] + 1);   // the arrays cover every Gaussian a pair names
    dev_->check(gs3dc_rasterize_arrays(dev_->ctx(), n, &a, bin.total_pairs, bin.values_sorted, bin.num_tiles,
                                       bin.tile_ranges, C(cam), C(cfg), img, T, nc),
                "rasterize (host arrays)");
}

// RasterizerBackwardCPU::backward (src/cpu/rasterizer_backward_cpu.cpp:7-138)
void RasterizerBackwardCUDA::backward(const PreprocessOutput&, const BinningOutput&, const Camera& cam,
                                      const RenderConfig& cfg, const ForwardCache&, const float* d_image,
                                      RasterGradOutput& rg) {
    dev_->check(gs3dc_raster_backward(dev_->ctx(), C(cam), C(cfg), d_image, rg.d_means2D, rg.d_conics, rg.d_rgb,
                                      rg.d_opacities_2d),
                "raster backward");
}

// PreprocessorBackwardCPU::backward (src/cpu/preprocessor_backward_cpu.cpp:205-645)
void PreprocessorBackwardCUDA::backward(const GaussianData&, const Camera& cam, const RenderConfig& cfg,
                                        const ForwardCache&, const RasterGradOutput&, const RawGaussianParams& raw,
                                        GradientOutput& gr) {
    dev_->check(gs3dc_preprocess_backward(dev_->ctx(), C(cam), C(cfg), raw.raw_rotations, gr.d_raw_positions,
                                          gr.d_raw_scales, gr.d_raw_rotations, gr.d_raw_sh_coeffs,
                                          gr.d_raw_opacities),
                "preprocess backward");
}

void TrainerCUDA::ensure_uploaded(RawGaussianParams& params, bool always) {
    if (params.count != n_ || params.max_coeffs != mc_) {
        dev_->check(gs3dc_set_raw_params(dev_->ctx(), C(params)), "upload parameters");   // resets Adam
        n_ = params.count;
        mc_ = params.max_coeffs;
    } else if (always) {
        dev_->check(gs3dc_update_raw_params(dev_->ctx(), C(params)), "update parameters");
    }
}

// Trainer::step (src/trainer.cpp:7-70)
TrainerCUDA::StepResult TrainerCUDA::step(RawGaussianParams& params, const Camera& cam, const float* gt,
                                          const RenderConfig& cfg, const TrainConfig& tc, int iteration) {
    ensure_uploaded(params, true);
    float loss = 0.0f;
    dev_->check(gs3dc_train_step(dev_->ctx(), C(cam), gt, 0, C(cfg), C(tc), iteration, &loss), "train step");
    dev_->check(gs3dc_get_raw_params(dev_->ctx(), C(params)), "download parameters");
    width_ = cam.width;
    height_ = cam.height;
    rendered_.clear();
    return {loss, iteration, params.count};
}

TrainerCUDA::StepResult TrainerCUDA::step_resident(RawGaussianParams& params, const Camera& cam, const float* gt,
                                                   const RenderConfig& cfg, const TrainConfig& tc, int iteration) {
    ensure_uploaded(params, false);
    float loss = 0.0f;
    dev_->check(gs3dc_train_step(dev_->ctx(), C(cam), gt, 0, C(cfg), C(tc), iteration, &loss), "train step");
    width_ = cam.width;
    height_ = cam.height;
    rendered_.clear();
    return {loss, iteration, params.count};
}

void TrainerCUDA::download_params(RawGaussianParams& params) const {
    dev_->check(gs3dc_get_raw_params(dev_->ctx(), C(params)), "download parameters");
}

const float* TrainerCUDA::last_rendered() {
    if (width_ <= 0) return nullptr;
    if (rendered_.empty()) {
        rendered_.resize((size_t)width_ * height_ * 3);
        dev_->check(gs3dc_get_image(dev_->ctx(), rendered_.data()), "download image");
    }
    return rendered_.data();
}
