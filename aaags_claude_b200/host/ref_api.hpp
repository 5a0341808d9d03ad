// ref_api.hpp -- the harmonyos_3dgs stage interfaces and buffer types, restated
// for builds outside the reference tree.
//
// The CUDA stage adapters (gs3d_stages_cuda.hpp) derive from the reference's
// abstract Preprocessor / TileBinner / Sorter / Rasterizer classes.  Compiled
// inside the reference build (-DGS3D_WITH_REFERENCE_HEADERS) they use its own
// headers; everywhere else this file provides the same names, member layouts and
// virtual signatures:
//   FrameAllocator, GaussianData, Camera, RenderConfig,
//   PreprocessOutput, BinningOutput, ForwardCache      include/types.h:8-107
//   RawGaussianParams, RasterGradOutput, GradientOutput,
//   TrainConfig                                        include/train_types.h:9-60
//   Preprocessor, TileBinner, Sorter, Rasterizer       include/{preprocessor,tile_binner,sorter,rasterizer}.h
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>

// Arena allocator reset once per frame (include/types.h:8-31): bump pointer,
// 64-byte default alignment, throws when the arena is exhausted.
class FrameAllocator {
public:
    explicit FrameAllocator(size_t capacity) : capacity_((capacity + 63) & ~size_t(63)), offset_(0) {
        buffer_ = static_cast<char*>(std::aligned_alloc(64, capacity_ ? capacity_ : 64));
        if (!buffer_) throw std::bad_alloc();
    }
    ~FrameAllocator() { std::free(buffer_); }
    FrameAllocator(const FrameAllocator&) = delete;
    FrameAllocator& operator=(const FrameAllocator&) = delete;

    void* allocate(size_t bytes, size_t alignment = 64) {
        const size_t start = (offset_ + alignment - 1) & ~(alignment - 1);
        if (start + bytes > capacity_) throw std::runtime_error("FrameAllocator out of memory");
        offset_ = start + bytes;
        return buffer_ + start;
    }
    template <typename T>
    T* allocate_array(size_t count) {
        return static_cast<T*>(allocate(count * sizeof(T)));
    }
    void reset() { offset_ = 0; }
    size_t used() const { return offset_; }
    size_t capacity() const { return capacity_; }

private:
    char* buffer_;
    size_t capacity_;
    size_t offset_;
};

struct GaussianData {
    int count;
    int sh_degree;
    int max_coeffs;
    float* positions;
    float* sh_coeffs;
    float* scales;
    float* rotations;
    float* opacities;
    float* filter_3D;
};

struct Camera {
    float view_matrix[16];
    float viewproj_matrix[16];
    float cam_pos[3];
    float tan_fovx, tan_fovy;
    int width, height;
};

struct RenderConfig {
    float bg_color[3] = {0, 0, 0};
    float scale_modifier = 1.0f;
    bool antialiasing = false;
    bool eval_3D = false;
    bool training = false;
    int sh_degree = 3;
    int tile_w = 16;
    int tile_h = 16;
};

struct PreprocessOutput {
    float* means2D;
    float* depths;
    float* conics;
    float* opacities_2d;
    float* rgb;
    int* radii;
    int* tiles_touched;
    float* gauss2screen;
    float* cov3D_inv;
    float* mean_offset;
    bool eval_3D = false;
    void* device_data = nullptr;
};

struct BinningOutput {
    int total_pairs;
    uint64_t* keys_unsorted;
    uint32_t* values_unsorted;
    uint64_t* keys_sorted;
    uint32_t* values_sorted;
    int num_tiles;
    uint32_t* tile_ranges;
    void* device_data = nullptr;
};

struct ForwardCache {
    float* T_final;
    int* n_contrib;
    float* cov2D;
    float* cov2D_det;
    float* cov3D;
    float* p_view;
    float* p_hom_w;
    PreprocessOutput* pre;
    BinningOutput* bin;
};

struct RawGaussianParams {
    int count;
    int sh_degree;
    int max_coeffs;
    float* raw_positions;
    float* raw_scales;
    float* raw_rotations;
    float* raw_sh_coeffs;
    float* raw_opacities;

    // exp scales, unit quaternions (length clamped at 1e-12), sigmoid opacities
    void activate(GaussianData& g) const {
        const int N = count;
        std::memcpy(g.positions, raw_positions, sizeof(float) * 3 * N);
        for (int i = 0; i < N * 3; i++) g.scales[i] = std::exp(raw_scales[i]);
        for (int i = 0; i < N; i++) {
            const float* q = raw_rotations + 4 * i;
            float len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
            if (len < 1e-12f) len = 1e-12f;
            const float inv = 1.0f / len;
            for (int k = 0; k < 4; k++) g.rotations[4 * i + k] = q[k] * inv;
        }
        std::memcpy(g.sh_coeffs, raw_sh_coeffs, sizeof(float) * (size_t)N * max_coeffs * 3);
        for (int i = 0; i < N; i++) g.opacities[i] = 1.0f / (1.0f + std::exp(-raw_opacities[i]));
    }
};

struct RasterGradOutput {
    float* d_means2D;
    float* d_conics;
    float* d_rgb;
    float* d_opacities_2d;

    void allocate_and_zero(FrameAllocator& alloc, int N) {
        d_means2D = alloc.allocate_array<float>(N * 2);
        d_conics = alloc.allocate_array<float>(N * 3);
        d_rgb = alloc.allocate_array<float>(N * 3);
        d_opacities_2d = alloc.allocate_array<float>(N);
        std::memset(d_means2D, 0, sizeof(float) * 2 * N);
        std::memset(d_conics, 0, sizeof(float) * 3 * N);
        std::memset(d_rgb, 0, sizeof(float) * 3 * N);
        std::memset(d_opacities_2d, 0, sizeof(float) * N);
    }
};

struct GradientOutput {
    float* d_raw_positions;
    float* d_raw_scales;
    float* d_raw_rotations;
    float* d_raw_sh_coeffs;
    float* d_raw_opacities;

    void allocate_and_zero(FrameAllocator& alloc, int N, int max_coeffs) {
        d_raw_positions = alloc.allocate_array<float>(N * 3);
        d_raw_scales = alloc.allocate_array<float>(N * 3);
        d_raw_rotations = alloc.allocate_array<float>(N * 4);
        d_raw_sh_coeffs = alloc.allocate_array<float>((size_t)N * max_coeffs * 3);
        d_raw_opacities = alloc.allocate_array<float>(N);
        std::memset(d_raw_positions, 0, sizeof(float) * 3 * N);
        std::memset(d_raw_scales, 0, sizeof(float) * 3 * N);
        std::memset(d_raw_rotations, 0, sizeof(float) * 4 * N);
        std::memset(d_raw_sh_coeffs, 0, sizeof(float) * (size_t)N * max_coeffs * 3);
        std::memset(d_raw_opacities, 0, sizeof(float) * N);
    }
};

struct TrainConfig {
    float lr_position_init = 0.00016f;
    float lr_position_final = 0.0000016f;
    float lr_feature = 0.0025f;
    float lr_opacity = 0.025f;
    float lr_scaling = 0.005f;
    float lr_rotation = 0.001f;
    int max_steps = 30000;
    bool use_adam = false;
    float adam_beta1 = 0.9f;
    float adam_beta2 = 0.999f;
    float adam_eps = 1e-8f;
};

class Preprocessor {
public:
    virtual ~Preprocessor() = default;
    virtual PreprocessOutput process(const GaussianData& gaussians, const Camera& camera, const RenderConfig& config,
                                     FrameAllocator& allocator, ForwardCache* cache = nullptr) = 0;
};

class TileBinner {
public:
    virtual ~TileBinner() = default;
    virtual BinningOutput bin(const PreprocessOutput& preprocess, int num_gaussians, const Camera& camera,
                              const RenderConfig& config, FrameAllocator& allocator) = 0;
};

class Sorter {
public:
    virtual ~Sorter() = default;
    virtual void sort(BinningOutput& binning, FrameAllocator& allocator) = 0;
};

class Rasterizer {
public:
    virtual ~Rasterizer() = default;
    virtual void rasterize(const PreprocessOutput& preprocess, const BinningOutput& binning, const Camera& camera,
                           const RenderConfig& config, float* output_image, float* output_depth = nullptr,
                           ForwardCache* cache = nullptr, FrameAllocator* allocator = nullptr) = 0;
};
