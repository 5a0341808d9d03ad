// io.cpp -- the on-disk formats of the reference's render / train drivers:
// 3DGS PLY models, cameras.json view lists and binary PPM images, plus the
// conversion of a loaded (activated) model into trainable raw parameters.
// Host code, compiled with -ffp-contract=off: every float value is computed
// with the reference's operations and libm calls, so models, cameras and
// images come out bit for bit as the reference's loaders produce them.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/gs3d_cuda.h"

namespace {

// ---------------- PLY ----------------

struct PlyLayout {
    int count = 0;
    size_t header_bytes = 0;
    int props = 0;                       // float properties per vertex
    std::unordered_map<std::string, int> index;
    int sh_degree = 0, max_coeffs = 1, rest_per_channel = 0;
    bool has_filter = false;
};

bool read_all(const char* path, std::string& out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, n);
    std::fclose(f);
    return true;
}

// Header of a binary little-endian 3DGS PLY (ply_loader.cpp:37-118): vertex
// count, the float properties in order, SH degree from the f_rest count
// (45 / 24 / 9 -> 3 / 2 / 1, else 0).
int parse_ply_header(const std::string& data, PlyLayout& L, std::string& err) {
    size_t pos = 0;
    auto next_line = [&](std::string& line) -> bool {
        if (pos >= data.size()) return false;
        size_t e = data.find('\n', pos);
        if (e == std::string::npos) e = data.size();
        line = data.substr(pos, e - pos);
        if (!line.empty() && line.back() == '\r') line.pop_back();
        pos = e + 1;
        return true;
    };
    std::string line;
    if (!next_line(line) || line != "ply") {
        err = "not a PLY file";
        return GS3DC_ERR_INVALID_ARG;
    }
    bool in_vertex = false, ended = false;
    std::vector<std::string> names;
    while (next_line(line)) {
        if (line == "end_header") {
            ended = true;
            break;
        }
        if (line.rfind("format ", 0) == 0 && line.find("binary_little_endian") == std::string::npos) {
            err = "only binary_little_endian PLY files are supported";
            return GS3DC_ERR_INVALID_ARG;
        }
        if (line.rfind("element ", 0) == 0) {
            in_vertex = line.rfind("element vertex ", 0) == 0;
            if (in_vertex) L.count = std::atoi(line.c_str() + 15);
            else if (L.count > 0) {
                err = "PLY elements after the vertices are not supported";
                return GS3DC_ERR_INVALID_ARG;
            }
            continue;
        }
        if (in_vertex && line.rfind("property ", 0) == 0) {
            if (line.rfind("property float ", 0) != 0) {
                err = "vertex property '" + line + "' is not a float";
                return GS3DC_ERR_INVALID_ARG;
            }
            names.push_back(line.substr(15));
        }
    }
    if (!ended || L.count <= 0) {
        err = "PLY header: no end_header or no vertex count";
        return GS3DC_ERR_INVALID_ARG;
    }
    L.header_bytes = pos;
    L.props = (int)names.size();
    for (int i = 0; i < L.props; i++) L.index[names[i]] = i;
    static const char* required[] = {"x",       "y",       "z",       "f_dc_0", "f_dc_1", "f_dc_2", "opacity",
                                     "scale_0", "scale_1", "scale_2", "rot_0",  "rot_1",  "rot_2",  "rot_3"};
    for (const char* r : required)
        if (!L.index.count(r)) {
            err = std::string("PLY missing required property: ") + r;
            return GS3DC_ERR_INVALID_ARG;
        }
    int rest = 0;
    while (L.index.count("f_rest_" + std::to_string(rest))) rest++;
    if (rest >= 45) L.sh_degree = 3, L.rest_per_channel = 15;
    else if (rest >= 24) L.sh_degree = 2, L.rest_per_channel = 8;
    else if (rest >= 9) L.sh_degree = 1, L.rest_per_channel = 3;
    L.max_coeffs = (L.sh_degree + 1) * (L.sh_degree + 1);
    L.has_filter = L.index.count("filter_3D") > 0;
    if (data.size() < L.header_bytes + (size_t)L.count * L.props * sizeof(float)) {
        err = "PLY: failed to read all vertex data";
        return GS3DC_ERR_INVALID_ARG;
    }
    return GS3DC_OK;
}

thread_local std::string g_io_error;

int io_fail(int status, const std::string& msg) {
    g_io_error = msg;
    return status;
}

// ---------------- cameras.json ----------------

// A small JSON reader for the cameras.json of 3DGS (an array of objects).
struct Json {
    enum Kind { NUL, NUM, STR, ARR, OBJ, BOOL } kind = NUL;
    double num = 0.0;
    std::string str;
    std::vector<Json> items;
    std::vector<std::pair<std::string, Json>> fields;
    const Json* get(const char* k) const {
        for (auto& f : fields)
            if (f.first == k) return &f.second;
        return nullptr;
    }
};

struct JsonParser {
    const char* p;
    const char* end;
    int depth = 0;
    void ws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    }
    bool value(Json& v) {
        ws();
        if (p >= end || ++depth > 64) return false;
        bool ok = false;
        if (*p == '{') ok = object(v);
        else if (*p == '[') ok = array(v);
        else if (*p == '"') {
            v.kind = Json::STR;
            ok = string(v.str);
        } else if (!std::strncmp(p, "true", 4) || !std::strncmp(p, "false", 5)) {
            v.kind = Json::BOOL;
            v.num = *p == 't' ? 1.0 : 0.0;
            p += *p == 't' ? 4 : 5;
            ok = true;
        } else if (!std::strncmp(p, "null", 4)) {
            p += 4;
            ok = true;
        } else {
            // numbers: strtod, the parser behind the reference's std::stod
            char* q = nullptr;
            errno = 0;
            v.num = std::strtod(p, &q);
            ok = q != p;
            v.kind = Json::NUM;
            p = q;
        }
        depth--;
        return ok;
    }
    bool string(std::string& s) {
        if (*p != '"') return false;
        p++;
        while (p < end && *p != '"') {
            if (*p == '\\' && p + 1 < end) {
                p++;
                const char c = *p;
                s.push_back(c == 'n' ? '\n' : c == 't' ? '\t' : c);
            } else {
                s.push_back(*p);
            }
            p++;
        }
        if (p >= end) return false;
        p++;
        return true;
    }
    bool array(Json& v) {
        v.kind = Json::ARR;
        p++;
        ws();
        if (p < end && *p == ']') {
            p++;
            return true;
        }
        while (p < end) {
            v.items.emplace_back();
            if (!value(v.items.back())) return false;
            ws();
            if (p < end && *p == ',') {
                p++;
                continue;
            }
            if (p < end && *p == ']') {
                p++;
                return true;
            }
            return false;
        }
        return false;
    }
    bool object(Json& v) {
        v.kind = Json::OBJ;
        p++;
        ws();
        if (p < end && *p == '}') {
            p++;
            return true;
        }
        while (p < end) {
            ws();
            std::string k;
            if (!string(k)) return false;
            ws();
            if (p >= end || *p != ':') return false;
            p++;
            v.fields.emplace_back(k, Json());
            if (!value(v.fields.back().second)) return false;
            ws();
            if (p < end && *p == ',') {
                p++;
                continue;
            }
            if (p < end && *p == '}') {
                p++;
                return true;
            }
            return false;
        }
        return false;
    }
};

// Column-major 4x4 product summed from zero (main.cpp:77-85)
void mat4mul(const float A[16], const float B[16], float out[16]) {
    for (int col = 0; col < 4; col++)
        for (int row = 0; row < 4; row++) {
            float sum = 0;
            for (int k = 0; k < 4; k++) sum += A[k * 4 + row] * B[col * 4 + k];
            out[col * 4 + row] = sum;
        }
}

// Projection of the drivers, znear 0.01, zfar 100 (main.cpp:66-74)
void perspective(float tan_fovx, float tan_fovy, float znear, float zfar, float proj[16]) {
    std::memset(proj, 0, 16 * sizeof(float));
    proj[0] = 1.0f / tan_fovx;
    proj[5] = 1.0f / tan_fovy;
    proj[10] = zfar / (zfar - znear);
    proj[11] = 1.0f;
    proj[14] = -(zfar * znear) / (zfar - znear);
}

// One cameras.json entry as the train driver reads it (train_main.cpp:320-370):
// false for an entry that is not a camera (fx or fy <= 0, or no position /
// rotation).  The stored rotation is camera-to-world: the view matrix holds its
// transpose and -R^T c.
bool camera_from(const Json& o, gs3d_camera& cam, std::string& name) {
    auto num = [&](const char* k) -> double {
        const Json* j = o.get(k);
        return j && j->kind == Json::NUM ? j->num : 0.0;
    };
    std::memset(&cam, 0, sizeof(cam));
    cam.width = (int)num("width");
    cam.height = (int)num("height");
    const float fx = (float)num("fx"), fy = (float)num("fy");
    if (fx <= 0 || fy <= 0) return false;
    const Json* P = o.get("position");
    const Json* Rj = o.get("rotation");
    if (!P || P->kind != Json::ARR || P->items.size() < 3 || !Rj || Rj->kind != Json::ARR || Rj->items.size() < 3)
        return false;
    cam.tan_fovx = (float)cam.width / (2.0f * fx);
    cam.tan_fovy = (float)cam.height / (2.0f * fy);
    for (int k = 0; k < 3; k++) cam.cam_pos[k] = (float)P->items[k].num;
    float R[3][3];
    for (int r = 0; r < 3; r++) {
        const Json& row = Rj->items[r];
        if (row.kind != Json::ARR || row.items.size() < 3) return false;
        for (int c = 0; c < 3; c++) R[r][c] = (float)row.items[c].num;
    }
    const float* p = cam.cam_pos;
    const float t[3] = {-(R[0][0] * p[0] + R[1][0] * p[1] + R[2][0] * p[2]),
                        -(R[0][1] * p[0] + R[1][1] * p[1] + R[2][1] * p[2]),
                        -(R[0][2] * p[0] + R[1][2] * p[1] + R[2][2] * p[2])};
    float* v = cam.view_matrix;
    v[0] = R[0][0]; v[1] = R[0][1]; v[2] = R[0][2]; v[3] = 0;
    v[4] = R[1][0]; v[5] = R[1][1]; v[6] = R[1][2]; v[7] = 0;
    v[8] = R[2][0]; v[9] = R[2][1]; v[10] = R[2][2]; v[11] = 0;
    v[12] = t[0]; v[13] = t[1]; v[14] = t[2]; v[15] = 1;
    float proj[16];
    perspective(cam.tan_fovx, cam.tan_fovy, 0.01f, 100.0f, proj);
    mat4mul(proj, cam.view_matrix, cam.viewproj_matrix);
    const Json* nm = o.get("img_name");
    name = nm && nm->kind == Json::STR ? nm->str : std::string();
    return true;
}

}  // namespace

extern "C" {

const char* gs3dc_io_last_error(void) { return g_io_error.c_str(); }

int gs3dc_ply_info(const char* path, int* count, int* sh_degree, int* max_coeffs, int* has_filter_3D) {
    if (!path) return io_fail(GS3DC_ERR_INVALID_ARG, "NULL path");
    std::string data, err;
    if (!read_all(path, data)) return io_fail(GS3DC_ERR_INVALID_ARG, std::string("cannot open ") + path);
    PlyLayout L;
    if (int rc = parse_ply_header(data, L, err)) return io_fail(rc, err);
    if (count) *count = L.count;
    if (sh_degree) *sh_degree = L.sh_degree;
    if (max_coeffs) *max_coeffs = L.max_coeffs;
    if (has_filter_3D) *has_filter_3D = L.has_filter ? 1 : 0;
    return GS3DC_OK;
}

int gs3dc_ply_read(const char* path, int activate, gs3d_gaussians* g) {
    if (!path || !g) return io_fail(GS3DC_ERR_INVALID_ARG, "NULL argument");
    std::string data, err;
    if (!read_all(path, data)) return io_fail(GS3DC_ERR_INVALID_ARG, std::string("cannot open ") + path);
    PlyLayout L;
    if (int rc = parse_ply_header(data, L, err)) return io_fail(rc, err);
    if (g->count != L.count || g->max_coeffs != L.max_coeffs)
        return io_fail(GS3DC_ERR_INVALID_ARG, "arrays sized for another model (use gs3dc_ply_info)");
    if (!g->positions || !g->scales || !g->rotations || !g->sh_coeffs || !g->opacities)
        return io_fail(GS3DC_ERR_INVALID_ARG, "model arrays must be non-NULL");
    g->sh_degree = L.sh_degree;
    const int N = L.count, mc3 = L.max_coeffs * 3, rpc = L.rest_per_channel;
    auto ix = [&](const std::string& k) { return L.index.at(k); };
    const int ipx = ix("x"), ipy = ix("y"), ipz = ix("z"), idc0 = ix("f_dc_0"), idc1 = ix("f_dc_1"),
              idc2 = ix("f_dc_2"), iop = ix("opacity"), is0 = ix("scale_0"), is1 = ix("scale_1"),
              is2 = ix("scale_2"), ir0 = ix("rot_0"), ir1 = ix("rot_1"), ir2 = ix("rot_2"), ir3 = ix("rot_3");
    std::vector<int> irest((size_t)3 * rpc);
    for (int k = 0; k < 3 * rpc; k++) irest[k] = ix("f_rest_" + std::to_string(k));
    const int ifl = L.has_filter ? ix("filter_3D") : -1;
    std::vector<float> row(L.props);
    for (int i = 0; i < N; i++) {
        std::memcpy(row.data(), data.data() + L.header_bytes + (size_t)i * L.props * 4, (size_t)L.props * 4);
        const float* v = row.data();
        g->positions[3 * i] = v[ipx];
        g->positions[3 * i + 1] = v[ipy];
        g->positions[3 * i + 2] = v[ipz];
        // SH: channel-first in the file, basis-interleaved in memory (ply_loader.cpp:153-166)
        float* sh = g->sh_coeffs + (size_t)i * mc3;
        std::memset(sh, 0, sizeof(float) * mc3);
        sh[0] = v[idc0];
        sh[1] = v[idc1];
        sh[2] = v[idc2];
        for (int k = 0; k < rpc; k++)
            for (int c = 0; c < 3; c++) sh[3 + 3 * k + c] = v[irest[(size_t)c * rpc + k]];
        float r0 = v[ir0], r1 = v[ir1], r2 = v[ir2], r3 = v[ir3];
        if (activate) {
            // activations of the loader (ply_loader.cpp:168-185)
            g->opacities[i] = 1.0f / (1.0f + std::exp(-v[iop]));
            g->scales[3 * i] = std::exp(v[is0]);
            g->scales[3 * i + 1] = std::exp(v[is1]);
            g->scales[3 * i + 2] = std::exp(v[is2]);
            const float len = std::sqrt(r0 * r0 + r1 * r1 + r2 * r2 + r3 * r3);
            if (len > 0.0f) {
                const float inv = 1.0f / len;
                r0 *= inv;
                r1 *= inv;
                r2 *= inv;
                r3 *= inv;
            }
        } else {
            g->opacities[i] = v[iop];
            g->scales[3 * i] = v[is0];
            g->scales[3 * i + 1] = v[is1];
            g->scales[3 * i + 2] = v[is2];
        }
        g->rotations[4 * i] = r0;
        g->rotations[4 * i + 1] = r1;
        g->rotations[4 * i + 2] = r2;
        g->rotations[4 * i + 3] = r3;
        if (g->filter_3D) g->filter_3D[i] = ifl >= 0 ? v[ifl] : 0.0f;
    }
    return GS3DC_OK;
}

int gs3dc_ply_write(const char* path, const gs3d_raw_params* r) {
    if (!path || !r) return io_fail(GS3DC_ERR_INVALID_ARG, "NULL argument");
    const int N = r->count, mc3 = r->max_coeffs * 3, rpc = r->max_coeffs - 1;
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_fail(GS3DC_ERR_INVALID_ARG, std::string("cannot write ") + path);
    // header and vertex layout of the train driver's saver (train_main.cpp:82-138)
    std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(N) + "\n";
    for (const char* p : {"x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"}) h += std::string("property float ") + p + "\n";
    for (int i = 0; i < 3 * rpc; i++) h += "property float f_rest_" + std::to_string(i) + "\n";
    for (const char* p : {"opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"})
        h += std::string("property float ") + p + "\n";
    h += "end_header\n";
    bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
    const int props = 6 + 3 * rpc + 8;
    std::vector<float> v(props);
    for (int i = 0; i < N && ok; i++) {
        int k = 0;
        for (int j = 0; j < 3; j++) v[k++] = r->raw_positions[3 * i + j];
        const float* sh = r->raw_sh_coeffs + (size_t)i * mc3;
        for (int j = 0; j < 3; j++) v[k++] = sh[j];
        for (int c = 0; c < 3; c++)
            for (int b = 0; b < rpc; b++) v[k++] = sh[3 + 3 * b + c];
        v[k++] = r->raw_opacities[i];
        for (int j = 0; j < 3; j++) v[k++] = r->raw_scales[3 * i + j];
        for (int j = 0; j < 4; j++) v[k++] = r->raw_rotations[4 * i + j];
        ok = std::fwrite(v.data(), sizeof(float), props, f) == (size_t)props;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? GS3DC_OK : io_fail(GS3DC_ERR_INVALID_ARG, std::string("write to ") + path + " failed");
}

int gs3dc_raw_from_gaussians(const gs3d_gaussians* g, gs3d_raw_params* r) {
    if (!g || !r || r->count != g->count || r->max_coeffs != g->max_coeffs)
        return io_fail(GS3DC_ERR_INVALID_ARG, "raw arrays must match the model's count and SH width");
    // initRawFromGaussianData (train_main.cpp:26-65): log scales, inverse-sigmoid
    // opacities clamped to [1e-6, 1 - 1e-6], positions / rotations / SH as they are
    const size_t N = (size_t)g->count, mc3 = (size_t)g->max_coeffs * 3;
    r->sh_degree = g->sh_degree;
    std::memcpy(r->raw_positions, g->positions, N * 12);
    for (size_t i = 0; i < 3 * N; i++) {
        const float s = g->scales[i];
        r->raw_scales[i] = std::log(1e-12f < s ? s : 1e-12f);
    }
    std::memcpy(r->raw_rotations, g->rotations, N * 16);
    std::memcpy(r->raw_sh_coeffs, g->sh_coeffs, N * mc3 * 4);
    for (size_t i = 0; i < N; i++) {
        float y = g->opacities[i];
        y = 1e-6f < ((y < 1.0f - 1e-6f) ? y : 1.0f - 1e-6f) ? ((y < 1.0f - 1e-6f) ? y : 1.0f - 1e-6f) : 1e-6f;
        r->raw_opacities[i] = std::log(y / (1.0f - y));
    }
    return GS3DC_OK;
}

int gs3dc_cameras_read(const char* path, gs3d_camera* cams, char* names, int name_len, int max_cams,
                       int* n_cams) {
    if (!path || !n_cams) return io_fail(GS3DC_ERR_INVALID_ARG, "NULL argument");
    std::string data;
    if (!read_all(path, data)) return io_fail(GS3DC_ERR_INVALID_ARG, std::string("cannot open ") + path);
    JsonParser jp{data.data(), data.data() + data.size()};
    Json root;
    if (!jp.value(root) || (root.kind != Json::ARR && root.kind != Json::OBJ))
        return io_fail(GS3DC_ERR_INVALID_ARG, std::string("not a cameras.json array: ") + path);
    const std::vector<Json> single = root.kind == Json::OBJ ? std::vector<Json>{root} : std::vector<Json>{};
    const std::vector<Json>& items = root.kind == Json::ARR ? root.items : single;
    int n = 0;
    for (const Json& o : items) {
        if (o.kind != Json::OBJ || !o.get("id")) continue;
        gs3d_camera cam;
        std::string nm;
        if (!camera_from(o, cam, nm)) continue;
        if (cams && n < max_cams) {
            cams[n] = cam;
            if (names && name_len > 0) {
                char* dst = names + (size_t)n * name_len;
                std::strncpy(dst, nm.c_str(), (size_t)name_len - 1);
                dst[name_len - 1] = '\0';
            }
        }
        n++;
    }
    *n_cams = n;
    return GS3DC_OK;
}

int gs3dc_ppm_read(const char* path, float* image, int* width, int* height) {
    if (!path || !width || !height) return io_fail(GS3DC_ERR_INVALID_ARG, "NULL argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return io_fail(GS3DC_ERR_INVALID_ARG, std::string("cannot open ") + path);
    // P6, comments before the size, one whitespace byte after maxval (image_io.cpp:24-68)
    char magic[3] = {};
    int w = 0, h = 0, maxval = 0, ch;
    bool ok = std::fscanf(f, "%2s", magic) == 1 && std::strcmp(magic, "P6") == 0;
    while (ok && (ch = std::fgetc(f)) != EOF) {
        if (ch == '#') {
            while ((ch = std::fgetc(f)) != EOF && ch != '\n') {
            }
        } else if (ch > ' ') {
            std::ungetc(ch, f);
            break;
        }
    }
    ok = ok && std::fscanf(f, "%d %d %d", &w, &h, &maxval) == 3 && w > 0 && h > 0 && maxval > 0 && maxval < 256;
    if (!ok) {
        std::fclose(f);
        return io_fail(GS3DC_ERR_INVALID_ARG, std::string("not an 8-bit binary PPM (P6): ") + path);
    }
    std::fgetc(f);
    *width = w;
    *height = h;
    if (!image) {
        std::fclose(f);
        return GS3DC_OK;
    }
    std::vector<unsigned char> raw((size_t)w * h * 3);
    const size_t got = std::fread(raw.data(), 1, raw.size(), f);
    std::fclose(f);
    if (got != raw.size()) return io_fail(GS3DC_ERR_INVALID_ARG, std::string("PPM pixel data cut short: ") + path);
    const float scale = 1.0f / (float)maxval;
    for (size_t i = 0; i < raw.size(); i++) image[i] = (float)raw[i] * scale;
    return GS3DC_OK;
}

int gs3dc_ppm_write(const char* path, const float* image, int width, int height) {
    if (!path || !image || width <= 0 || height <= 0) return io_fail(GS3DC_ERR_INVALID_ARG, "bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_fail(GS3DC_ERR_INVALID_ARG, std::string("cannot write ") + path);
    std::fprintf(f, "P6\n%d %d\n255\n", width, height);
    // clamp to [0, 1], x 255, round half up (image_io.cpp:9-21)
    std::vector<unsigned char> px((size_t)width * height * 3);
    for (size_t i = 0; i < px.size(); i++) {
        const float c = image[i];
        const float v = 0.0f < (c < 1.0f ? c : 1.0f) ? (c < 1.0f ? c : 1.0f) : 0.0f;
        px[i] = (unsigned char)(v * 255.0f + 0.5f);
    }
    bool ok = std::fwrite(px.data(), 1, px.size(), f) == px.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? GS3DC_OK : io_fail(GS3DC_ERR_INVALID_ARG, std::string("write to ") + path + " failed");
}

int gs3dc_image_resize_nearest(const float* src, int sw, int sh, float* dst, int dw, int dh) {
    if (!src || !dst || sw <= 0 || sh <= 0 || dw <= 0 || dh <= 0) return io_fail(GS3DC_ERR_INVALID_ARG, "bad size");
    // the train driver's target resize (train_main.cpp:536-548)
    for (int y = 0; y < dh; y++) {
        const int sy = (int)((long long)y * sh / dh);
        for (int x = 0; x < dw; x++) {
            const int sx = (int)((long long)x * sw / dw);
            for (int c = 0; c < 3; c++) dst[((size_t)y * dw + x) * 3 + c] = src[((size_t)sy * sw + sx) * 3 + c];
        }
    }
    return GS3DC_OK;
}

}  // extern "C"
