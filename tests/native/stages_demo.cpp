// stages_demo.cpp -- drives the CUDA stage adapters through the reference's
// abstract interfaces, the way Renderer::render (src/renderer.cpp:13-39) and
// Trainer::step (src/trainer.cpp:7-70) compose them.  Used by the GPU tests.
//
//   stages_demo <dir>
//
// <dir> holds the inputs (raw_positions.bin, raw_scales.bin, raw_rotations.bin,
// raw_sh_coeffs.bin, raw_opacities.bin, camera.bin, render_config.bin,
// train_config.bin, gt_image.bin, meta.txt = "N sh_degree max_coeffs steps")
// as raw little-endian arrays; the outputs are written next to them.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "gs3d_stages_cuda.hpp"

namespace {

template <class T>
std::vector<T> read_vec(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot read " + path);
    const std::streamsize n = f.tellg();
    f.seekg(0);
    std::vector<T> v((size_t)n / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), n);
    return v;
}

template <class T>
void write_vec(const std::string& path, const T* p, size_t n) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(p), (std::streamsize)(n * sizeof(T)));
}

template <class T>
T read_pod(const std::string& path) {
    auto v = read_vec<unsigned char>(path);
    if (v.size() != sizeof(T)) throw std::runtime_error("size mismatch in " + path);
    T t;
    std::memcpy(&t, v.data(), sizeof(T));
    return t;
}

// L1 loss gradient (src/loss.cpp:4-16)
float l1(const float* img, const float* gt, size_t n, float* d) {
    const float inv_n = 1.0f / (float)n;
    float sum = 0.0f;
    for (size_t i = 0; i < n; i++) {
        const float diff = img[i] - gt[i];
        sum += std::abs(diff);
        d[i] = diff > 0.0f ? inv_n : (diff < 0.0f ? -inv_n : 0.0f);
    }
    return sum * inv_n;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <dir>\n", argv[0]);
        return 2;
    }
    const std::string d = argv[1];
    try {
        int N = 0, deg = 0, mc = 0, steps = 0;
        {
            std::ifstream m(d + "/meta.txt");
            m >> N >> deg >> mc >> steps;
        }
        auto pos = read_vec<float>(d + "/raw_positions.bin");
        auto sc = read_vec<float>(d + "/raw_scales.bin");
        auto rot = read_vec<float>(d + "/raw_rotations.bin");
        auto sh = read_vec<float>(d + "/raw_sh_coeffs.bin");
        auto op = read_vec<float>(d + "/raw_opacities.bin");
        auto gt = read_vec<float>(d + "/gt_image.bin");
        const Camera cam = read_pod<Camera>(d + "/camera.bin");
        const RenderConfig cfg = read_pod<RenderConfig>(d + "/render_config.bin");
        const TrainConfig tc = read_pod<TrainConfig>(d + "/train_config.bin");
        const size_t np = (size_t)cam.width * cam.height;

        RawGaussianParams raw{N, deg, mc, pos.data(), sc.data(), rot.data(), sh.data(), op.data()};
        std::vector<float> ap(3 * N), as(3 * N), ar(4 * N), ash((size_t)N * mc * 3), ao(N);
        GaussianData g{N, deg, mc, ap.data(), ash.data(), as.data(), ar.data(), ao.data(), nullptr};
        raw.activate(g);

        auto dev = std::make_shared<CudaDevice>(0);
        std::unique_ptr<Preprocessor> pp = std::make_unique<PreprocessorCUDA>(dev);
        std::unique_ptr<TileBinner> tb = std::make_unique<TileBinnerCUDA>(dev);
        std::unique_ptr<Sorter> so = std::make_unique<SorterCUDA>(dev);
        std::unique_ptr<Rasterizer> ra = std::make_unique<RasterizerCUDA>(dev);
        FrameAllocator alloc(size_t(512) << 20);

        // ---- forward through the stage interfaces, with the ForwardCache of training ----
        ForwardCache cache{};
        PreprocessOutput pre = pp->process(g, cam, cfg, alloc, &cache);
        BinningOutput bin = tb->bin(pre, N, cam, cfg, alloc);
        if (bin.total_pairs > 0) so->sort(bin, alloc);
        cache.pre = &pre;
        cache.bin = &bin;
        std::vector<float> img(np * 3);
        ra->rasterize(pre, bin, cam, cfg, img.data(), nullptr, &cache, &alloc);
        write_vec(d + "/out_radii.bin", pre.radii, N);
        write_vec(d + "/out_tiles.bin", pre.tiles_touched, N);
        write_vec(d + "/out_keys_unsorted.bin", bin.keys_unsorted, bin.total_pairs);
        write_vec(d + "/out_vals_unsorted.bin", bin.values_unsorted, bin.total_pairs);
        write_vec(d + "/out_keys_sorted.bin", bin.keys_sorted, bin.total_pairs);
        write_vec(d + "/out_vals_sorted.bin", bin.values_sorted, bin.total_pairs);
        write_vec(d + "/out_ranges.bin", bin.tile_ranges, (size_t)bin.num_tiles * 2);
        write_vec(d + "/out_image.bin", img.data(), np * 3);
        write_vec(d + "/out_T_final.bin", cache.T_final, np);
        write_vec(d + "/out_n_contrib.bin", cache.n_contrib, np);

        // ---- stage-level backward (RasterizerBackward + PreprocessorBackward) ----
        std::vector<float> d_image(np * 3);
        const float loss = l1(img.data(), gt.data(), np * 3, d_image.data());
        RasterGradOutput rg;
        rg.allocate_and_zero(alloc, N);
        RasterizerBackwardCUDA(dev).backward(pre, bin, cam, cfg, cache, d_image.data(), rg);
        GradientOutput gr;
        gr.allocate_and_zero(alloc, N, mc);
        PreprocessorBackwardCUDA(dev).backward(g, cam, cfg, cache, rg, raw, gr);
        write_vec(d + "/out_g_pos.bin", gr.d_raw_positions, (size_t)N * 3);
        write_vec(d + "/out_g_sc.bin", gr.d_raw_scales, (size_t)N * 3);
        write_vec(d + "/out_g_rot.bin", gr.d_raw_rotations, (size_t)N * 4);
        write_vec(d + "/out_g_sh.bin", gr.d_raw_sh_coeffs, (size_t)N * mc * 3);
        write_vec(d + "/out_g_op.bin", gr.d_raw_opacities, (size_t)N);

        // ---- Trainer::step with the caller's parameters updated in place ----
        TrainerCUDA trainer(dev);
        std::vector<float> losses;
        for (int it = 0; it < steps; it++) losses.push_back(trainer.step(raw, cam, gt.data(), cfg, tc, it).loss);
        write_vec(d + "/out_losses.bin", losses.data(), losses.size());
        write_vec(d + "/out_params_pos.bin", pos.data(), pos.size());
        write_vec(d + "/out_params_sc.bin", sc.data(), sc.size());
        write_vec(d + "/out_params_rot.bin", rot.data(), rot.size());
        write_vec(d + "/out_params_sh.bin", sh.data(), sh.size());
        write_vec(d + "/out_params_op.bin", op.data(), op.size());
        write_vec(d + "/out_last_rendered.bin", trainer.last_rendered(), np * 3);
        std::printf("stages_demo ok: N=%d pairs=%d loss=%.7f\n", N, bin.total_pairs, loss);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "stages_demo: %s\n", e.what());
        return 1;
    }
}
