// gs3d_stages_cuda.hpp -- CUDA (sm_100a) implementations of the harmonyos_3dgs
// stage interfaces, over the gs3dc_* C ABI (include/gs3d_cuda.h).
//
// Drop-in counterparts of the reference's CPU / OpenCL stage classes:
//   PreprocessorCUDA          : Preprocessor   (src/cpu/preprocessor_cpu.h, src/gpu/preprocessor_gpu.h)
//   TileBinnerCUDA            : TileBinner     (src/cpu/tile_binner_cpu.h, src/gpu/tile_binner_gpu.h)
//   SorterCUDA                : Sorter         (src/cpu/sorter_cpu.h, src/gpu/sorter_gpu.h)
//   RasterizerCUDA            : Rasterizer     (src/cpu/rasterizer_cpu.h, src/gpu/rasterizer_gpu.h)
//   RasterizerBackwardCUDA    (src/cpu/rasterizer_backward_cpu.h)
//   PreprocessorBackwardCUDA  (src/cpu/preprocessor_backward_cpu.h)
//   TrainerCUDA               (include/trainer.h: Trainer::step)
// All stages of one pipeline share a CudaDevice (one gs3dc context = one CUDA
// stream + the device buffers).  Device results flow between stages through the
// outputs' device_data handle, as in the reference's OpenCL backend; host arrays
// are filled from the caller's FrameAllocator exactly like the CPU stages.
// Failures throw std::runtime_error (the reference's CL_CHECK convention).
#pragma once

#ifdef GS3D_WITH_REFERENCE_HEADERS
#include "preprocessor.h"
#include "rasterizer.h"
#include "sorter.h"
#include "tile_binner.h"
#include "train_types.h"
#include "types.h"
#else
#include "ref_api.hpp"
#endif

#include <memory>
#include <vector>

#include "gs3d_cuda.h"

class CudaDevice {
public:
    explicit CudaDevice(int device = 0);
    ~CudaDevice();
    CudaDevice(const CudaDevice&) = delete;
    CudaDevice& operator=(const CudaDevice&) = delete;
    gs3dc_ctx* ctx() const { return ctx_; }
    // Throws std::runtime_error("<what>: <gs3dc message>") when status != GS3DC_OK.
    void check(int status, const char* what) const;

private:
    gs3dc_ctx* ctx_ = nullptr;
};

class PreprocessorCUDA : public Preprocessor {
public:
    explicit PreprocessorCUDA(std::shared_ptr<CudaDevice> dev) : dev_(std::move(dev)) {}
    PreprocessOutput process(const GaussianData& gaussians, const Camera& camera, const RenderConfig& config,
                             FrameAllocator& allocator, ForwardCache* cache = nullptr) override;

private:
    std::shared_ptr<CudaDevice> dev_;
};

class TileBinnerCUDA : public TileBinner {
public:
    // host_keys: also copy the unsorted keys / values to the host arrays (the
    // reference's OpenCL binner leaves them NULL, src/gpu/tile_binner_gpu.cpp:384-389)
    explicit TileBinnerCUDA(std::shared_ptr<CudaDevice> dev, bool host_keys = true)
        : dev_(std::move(dev)), host_keys_(host_keys) {}
    BinningOutput bin(const PreprocessOutput& preprocess, int num_gaussians, const Camera& camera,
                      const RenderConfig& config, FrameAllocator& allocator) override;

private:
    std::shared_ptr<CudaDevice> dev_;
    bool host_keys_;
};

class SorterCUDA : public Sorter {
public:
    explicit SorterCUDA(std::shared_ptr<CudaDevice> dev, bool host_keys = true)
        : dev_(std::move(dev)), host_keys_(host_keys) {}
    void sort(BinningOutput& binning, FrameAllocator& allocator) override;

private:
    std::shared_ptr<CudaDevice> dev_;
    bool host_keys_;
};

class RasterizerCUDA : public Rasterizer {
public:
    explicit RasterizerCUDA(std::shared_ptr<CudaDevice> dev) : dev_(std::move(dev)) {}
    // output_depth (inverse-depth image) is not produced by this backend and must be NULL.
    void rasterize(const PreprocessOutput& preprocess, const BinningOutput& binning, const Camera& camera,
                   const RenderConfig& config, float* output_image, float* output_depth = nullptr,
                   ForwardCache* cache = nullptr, FrameAllocator* allocator = nullptr) override;

private:
    std::shared_ptr<CudaDevice> dev_;
};

class RasterizerBackwardCUDA {
public:
    explicit RasterizerBackwardCUDA(std::shared_ptr<CudaDevice> dev) : dev_(std::move(dev)) {}
    void backward(const PreprocessOutput& pre, const BinningOutput& bin, const Camera& cam, const RenderConfig& cfg,
                  const ForwardCache& cache, const float* d_image, RasterGradOutput& rgrad);

private:
    std::shared_ptr<CudaDevice> dev_;
};

class PreprocessorBackwardCUDA {
public:
    explicit PreprocessorBackwardCUDA(std::shared_ptr<CudaDevice> dev) : dev_(std::move(dev)) {}
    void backward(const GaussianData& g, const Camera& cam, const RenderConfig& cfg, const ForwardCache& cache,
                  const RasterGradOutput& rgrad, const RawGaussianParams& raw, GradientOutput& grads);

private:
    std::shared_ptr<CudaDevice> dev_;
};

// Trainer::step on the device: activation, forward, L1, backward and the
// optimiser in one CUDA-graph replay.
//   step()          keeps Trainer::step's contract: the caller's parameters are
//                   read at the start of every call and updated in place at the
//                   end (two parameter-sized PCIe copies per step);
//   step_resident() keeps the parameters on the device between calls (upload on
//                   the first call or when N / SH size change); read them back
//                   with download_params().
// Adam moments reset when N or the SH size changes, like AdamOptimizer.
class TrainerCUDA {
public:
    struct StepResult {
        float loss;
        int iteration;
        int n_gaussians;
    };
    explicit TrainerCUDA(std::shared_ptr<CudaDevice> dev) : dev_(std::move(dev)) {}
    StepResult step(RawGaussianParams& params, const Camera& camera, const float* gt_image, const RenderConfig& cfg,
                    const TrainConfig& train_cfg, int iteration);
    StepResult step_resident(RawGaussianParams& params, const Camera& camera, const float* gt_image,
                             const RenderConfig& cfg, const TrainConfig& train_cfg, int iteration);
    void download_params(RawGaussianParams& params) const;
    // Host copy of the last rendered image (H*W*3); valid until the next step.
    const float* last_rendered();

private:
    void ensure_uploaded(RawGaussianParams& params, bool always);

    std::shared_ptr<CudaDevice> dev_;
    int n_ = -1, mc_ = -1;
    int width_ = 0, height_ = 0;
    std::vector<float> rendered_;
};
