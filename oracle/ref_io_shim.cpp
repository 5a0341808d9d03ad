// ref_io_shim.cpp -- TEST INFRASTRUCTURE.  The reference's file-format helpers
// for the tests: loadPly / readPPM / writePPM (src/ply_loader.cpp,
// src/image_io.cpp, linked), and the train driver's static savePly,
// initRawFromGaussianData and loadCamerasJson, reached by compiling the
// driver's own source (src/train_main.cpp, where it lies, found through the
// include path) inside this translation unit with its main() renamed.
#include "gs3d_oracle.h"

#define main gs3d_ref_train_main
#include "train_main.cpp"
#undef main

extern "C" {

// loadPly into caller arrays sized by ref_io_ply_count / the model's shape.
int ref_io_ply_count(const char* path, int* count, int* sh_degree, int* max_coeffs, int* has_filter) {
    LoadedModel m = loadPly(path);
    *count = m.data.count;
    *sh_degree = m.data.sh_degree;
    *max_coeffs = m.data.max_coeffs;
    *has_filter = m.data.filter_3D ? 1 : 0;
    m.free();
    return 0;
}

int ref_io_ply_load(const char* path, gs3d_gaussians* out) {
    LoadedModel m = loadPly(path);
    const size_t n = (size_t)m.data.count, mc3 = (size_t)m.data.max_coeffs * 3;
    std::memcpy(out->positions, m.data.positions, 12 * n);
    std::memcpy(out->scales, m.data.scales, 12 * n);
    std::memcpy(out->rotations, m.data.rotations, 16 * n);
    std::memcpy(out->sh_coeffs, m.data.sh_coeffs, 4 * mc3 * n);
    std::memcpy(out->opacities, m.data.opacities, 4 * n);
    if (out->filter_3D && m.data.filter_3D) std::memcpy(out->filter_3D, m.data.filter_3D, 4 * n);
    m.free();
    return 0;
}

int ref_io_ply_save(const char* path, const gs3d_raw_params* raw) {
    return savePly(path, *reinterpret_cast<const RawGaussianParams*>(raw)) ? 0 : 1;
}

void ref_io_raw_from_gaussians(const gs3d_gaussians* g, gs3d_raw_params* out) {
    RawGaussianParams r = initRawFromGaussianData(*reinterpret_cast<const GaussianData*>(g));
    const size_t n = (size_t)r.count, mc3 = (size_t)r.max_coeffs * 3;
    std::memcpy(out->raw_positions, r.raw_positions, 12 * n);
    std::memcpy(out->raw_scales, r.raw_scales, 12 * n);
    std::memcpy(out->raw_rotations, r.raw_rotations, 16 * n);
    std::memcpy(out->raw_sh_coeffs, r.raw_sh_coeffs, 4 * mc3 * n);
    std::memcpy(out->raw_opacities, r.raw_opacities, 4 * n);
    freeRawParams(r);
}

// loadCamerasJson: the cameras (up to max) and their image names (name_len bytes each).
int ref_io_cameras(const char* path, gs3d_camera* cams, char* names, int name_len, int max) {
    std::vector<CameraWithImage> v = loadCamerasJson(path);
    const int n = (int)v.size();
    for (int i = 0; i < n && i < max; i++) {
        std::memcpy(&cams[i], &v[i].cam, sizeof(Camera));
        std::strncpy(names + (size_t)i * name_len, v[i].img_name.c_str(), (size_t)name_len - 1);
        names[(size_t)i * name_len + name_len - 1] = '\0';
    }
    return n;
}

int ref_io_ppm_read(const char* path, float* image, int* w, int* h) {
    std::vector<float> img = readPPM(path, *w, *h);
    if (img.empty()) return 1;
    if (image) std::memcpy(image, img.data(), img.size() * sizeof(float));
    return 0;
}

int ref_io_ppm_write(const char* path, const float* image, int w, int h) { return writePPM(path, image, w, h) ? 0 : 1; }

}  // extern "C"
