// ref_math.cuh -- the reference's per-Gaussian arithmetic, restated for the
// device in the reference's operation order: activation (train_types.cpp:6-36),
// projection / EWA / SH (preprocessor_cpu.cpp:186-265, math_utils.cpp:8-144,
// sh_eval.cpp:24-89), the adjoint chain (preprocessor_backward_cpu.cpp:8-645)
// and the Adam element update (optimizer.cpp:32-43).
//
// Included by plain.cu, compiled without FMA contraction and with IEEE
// division / square root -- which makes its results round like the
// reference's -- and by the reduced-storage form's unit, compiled with FMA
// contraction, where the same code runs faster and rounds differently.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "raster_common.cuh"

namespace gs3d {
namespace {

__device__ __forceinline__ float ldf(float x) { return x; }
__device__ __forceinline__ float ldf(__half x) { return __half2float(x); }
__device__ __forceinline__ float ldf(__nv_bfloat16 x) { return __bfloat162float(x); }

// ---------------- reference math (float, reference operation order) ----------------

// math_utils.cpp:8-12
__device__ __forceinline__ void xform4x3(const float p[3], const float* m, float o[3]) {
    o[0] = m[0] * p[0] + m[4] * p[1] + m[8] * p[2] + m[12];
    o[1] = m[1] * p[0] + m[5] * p[1] + m[9] * p[2] + m[13];
    o[2] = m[2] * p[0] + m[6] * p[1] + m[10] * p[2] + m[14];
}
// math_utils.cpp:14-19 (w component only; x,y are what the projection uses too)
__device__ __forceinline__ void xform4x4(const float p[3], const float* m, float o[4]) {
    o[0] = m[0] * p[0] + m[4] * p[1] + m[8] * p[2] + m[12];
    o[1] = m[1] * p[0] + m[5] * p[1] + m[9] * p[2] + m[13];
    o[2] = m[2] * p[0] + m[6] * p[1] + m[10] * p[2] + m[14];
    o[3] = m[3] * p[0] + m[7] * p[1] + m[11] * p[2] + m[15];
}

// math_utils.cpp:21-28
__device__ __forceinline__ void tile_rect(float px, float py, int r, int gx, int gy, int tw, int th,
                                          int rmn[2], int rmx[2]) {
    const float fr = (float)r, ftw = (float)tw, fth = (float)th;
    rmn[0] = min(gx, max(0, (int)((px - fr) / ftw)));
    rmn[1] = min(gy, max(0, (int)((py - fr) / fth)));
    rmx[0] = min(gx, max(0, (int)((px + fr + ftw - 1.0f) / ftw)));
    rmx[1] = min(gy, max(0, (int)((py + fr + fth - 1.0f) / fth)));
}

__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }  // std::max

// math_utils.cpp:38-42
__device__ __forceinline__ void quat_to_R(float r, float x, float y, float z, float R[3][3]) {
    R[0][0] = 1.f - 2.f * (y * y + z * z);
    R[0][1] = 2.f * (x * y + r * z);
    R[0][2] = 2.f * (x * z - r * y);
    R[1][0] = 2.f * (x * y - r * z);
    R[1][1] = 1.f - 2.f * (x * x + z * z);
    R[1][2] = 2.f * (y * z + r * x);
    R[2][0] = 2.f * (x * z + r * y);
    R[2][1] = 2.f * (y * z - r * x);
    R[2][2] = 1.f - 2.f * (x * x + y * y);
}

// math_utils.cpp:30-62
__device__ __forceinline__ void cov3d(const float s_in[3], float mod, const float q[4], float cov[6]) {
    const float s[3] = {mod * s_in[0], mod * s_in[1], mod * s_in[2]};
    float R[3][3], M[3][3];
    quat_to_R(q[0], q[1], q[2], q[3], R);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) M[i][j] = s[i] * R[i][j];
    cov[0] = M[0][0] * M[0][0] + M[1][0] * M[1][0] + M[2][0] * M[2][0];
    cov[1] = M[0][0] * M[0][1] + M[1][0] * M[1][1] + M[2][0] * M[2][1];
    cov[2] = M[0][0] * M[0][2] + M[1][0] * M[1][2] + M[2][0] * M[2][2];
    cov[3] = M[0][1] * M[0][1] + M[1][1] * M[1][1] + M[2][1] * M[2][1];
    cov[4] = M[0][1] * M[0][2] + M[1][1] * M[1][2] + M[2][1] * M[2][2];
    cov[5] = M[0][2] * M[0][2] + M[1][2] * M[1][2] + M[2][2] * M[2][2];
}

// Clamped view point and T = W J of the EWA projection, [col][row] as in
// math_utils.cpp:64-110.  txtz / tytz are the unclamped ratios.
struct Ewa {
    float t[3];
    float txtz, tytz, limx, limy;
    float J[3][3], W[3][3], T[3][3];
};

__device__ __forceinline__ void ewa_setup(const float pos[3], const float* vm, float fx, float fy,
                                          float tanx, float tany, Ewa& e) {
    float t[3];
    xform4x3(pos, vm, t);
    e.limx = 1.3f * tanx;
    e.limy = 1.3f * tany;
    e.txtz = t[0] / t[2];
    e.tytz = t[1] / t[2];
    t[0] = fmin_ref(e.limx, fmax_ref(-e.limx, e.txtz)) * t[2];
    t[1] = fmin_ref(e.limy, fmax_ref(-e.limy, e.tytz)) * t[2];
    e.t[0] = t[0];
    e.t[1] = t[1];
    e.t[2] = t[2];
    e.J[0][0] = fx / t[2]; e.J[0][1] = 0.0f; e.J[0][2] = -(fx * t[0]) / (t[2] * t[2]);
    e.J[1][0] = 0.0f; e.J[1][1] = fy / t[2]; e.J[1][2] = -(fy * t[1]) / (t[2] * t[2]);
    e.J[2][0] = 0.0f; e.J[2][1] = 0.0f; e.J[2][2] = 0.0f;
    e.W[0][0] = vm[0]; e.W[0][1] = vm[4]; e.W[0][2] = vm[8];
    e.W[1][0] = vm[1]; e.W[1][1] = vm[5]; e.W[1][2] = vm[9];
    e.W[2][0] = vm[2]; e.W[2][1] = vm[6]; e.W[2][2] = vm[10];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; k++) acc += e.W[k][r] * e.J[c][k];
            e.T[c][r] = acc;
        }
}

// math_utils.cpp:111-143
__device__ __forceinline__ void cov2d(const Ewa& e, const float c3[6], float out[3]) {
    const float V[3][3] = {{c3[0], c3[1], c3[2]}, {c3[1], c3[3], c3[4]}, {c3[2], c3[4], c3[5]}};
    float tmp[3][3];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; k++) acc += V[r][k] * e.T[c][k];
            tmp[c][r] = acc;
        }
    float res00 = 0.0f, res10 = 0.0f, res11 = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; k++) res00 += e.T[0][k] * tmp[0][k];
#pragma unroll
    for (int k = 0; k < 3; k++) res10 += e.T[0][k] * tmp[1][k];
#pragma unroll
    for (int k = 0; k < 3; k++) res11 += e.T[1][k] * tmp[1][k];
    out[0] = res00;
    out[1] = res10;
    out[2] = res11;
}

// SH constants, sh_eval.cpp:5-22
#define SH_C0 0.28209479177387814f
#define SH_C1 0.4886025119029199f
#define SH_C20 1.0925484305920792f
#define SH_C21 -1.0925484305920792f
#define SH_C22 0.31539156525252005f
#define SH_C23 -1.0925484305920792f
#define SH_C24 0.5462742152960396f
#define SH_C30 -0.5900435899266435f
#define SH_C31 2.890611442640554f
#define SH_C32 -0.4570457994644658f
#define SH_C33 0.3731763325901154f
#define SH_C34 -0.4570457994644658f
#define SH_C35 1.445305721320277f
#define SH_C36 -0.5900435899266435f

// Normalised view direction (sh_eval.cpp:31-35); returns |pos - cam|.
__device__ __forceinline__ float view_dir(const float p[3], const float* cam, float d[3]) {
    const float dx = p[0] - cam[0], dy = p[1] - cam[1], dz = p[2] - cam[2];
    const float len = sqrtf(dx * dx + dy * dy + dz * dz);
    d[0] = dx / len;
    d[1] = dy / len;
    d[2] = dz / len;
    return len;
}

// Pre-clamp SH colour of one channel (sh_eval.cpp:38-81). sh points at this
// Gaussian's coefficients; stride 3 between bases.
template <typename S>
__device__ __forceinline__ float sh_channel(int deg, const S* __restrict__ sh, int c, float x, float y, float z) {
    float v = SH_C0 * ldf(sh[c]);
    if (deg > 0) {
        v += -SH_C1 * y * ldf(sh[3 + c]) + SH_C1 * z * ldf(sh[6 + c]) + -SH_C1 * x * ldf(sh[9 + c]);
        if (deg > 1) {
            const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            v += SH_C20 * xy * ldf(sh[12 + c]) + SH_C21 * yz * ldf(sh[15 + c]) +
                 SH_C22 * (2.0f * zz - xx - yy) * ldf(sh[18 + c]) + SH_C23 * xz * ldf(sh[21 + c]) +
                 SH_C24 * (xx - yy) * ldf(sh[24 + c]);
            if (deg > 2) {
                v += SH_C30 * y * (3.0f * xx - yy) * ldf(sh[27 + c]) + SH_C31 * xy * z * ldf(sh[30 + c]) +
                     SH_C32 * y * (4.0f * zz - xx - yy) * ldf(sh[33 + c]) +
                     SH_C33 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy) * ldf(sh[36 + c]) +
                     SH_C34 * x * (4.0f * zz - xx - yy) * ldf(sh[39 + c]) + SH_C35 * z * (xx - yy) * ldf(sh[42 + c]) +
                     SH_C36 * x * (xx - 3.0f * yy) * ldf(sh[45 + c]);
            }
        }
    }
    return v;
}

// Activation of one Gaussian (train_types.cpp:6-36): exp scales, unit
// quaternion (length clamped to 1e-12), sigmoid opacity.
__device__ __forceinline__ void activate_one(const float rsc[3], const float rq[4], float rop, float sc[3],
                                             float q[4], float* op) {
#pragma unroll
    for (int k = 0; k < 3; k++) sc[k] = exp_ref(rsc[k]);
    float len = sqrtf(rq[0] * rq[0] + rq[1] * rq[1] + rq[2] * rq[2] + rq[3] * rq[3]);
    if (len < 1e-12f) len = 1e-12f;
    const float inv = 1.0f / len;
#pragma unroll
    for (int k = 0; k < 4; k++) q[k] = rq[k] * inv;
    *op = 1.0f / (1.0f + exp_ref(-rop));
}

// ---------------- per-Gaussian forward (preprocessor_cpu.cpp:186-265) ----------------

struct Proj {
    float px, py, depth, con[3], opac, rgb[3];
    int radius, rmn[2], rmx[2];
    float cov3[6], pv[3], phw, cov2[3], det;
};

// Returns false when the Gaussian is culled.
// S: element type of the SH coefficients (float here; 16-bit in the
// reduced-storage form).  c3_in (optional): the Gaussian's cov3D, computed once
// by a caller that projects it into several cameras.
template <typename S>
__device__ __forceinline__ bool project_one(const StepParams& sp, const float p[3], const float sc[3],
                                            const float q[4], float op, const S* __restrict__ sh, Proj& r,
                                            const float* c3_in = nullptr) {
    const gs3d_camera& cam = sp.cam;
    float pv[3];
    xform4x3(p, cam.view_matrix, pv);
    if (pv[2] <= 0.2f) return false;
    float ph[4];
    xform4x4(p, cam.viewproj_matrix, ph);
    const float pw = 1.0f / (ph[3] + 1e-7f);
    const float ndc_x = ph[0] * pw, ndc_y = ph[1] * pw;
    const float pix_x = ((ndc_x + 1.0f) * (float)cam.width - 1.0f) * 0.5f;
    const float pix_y = ((ndc_y + 1.0f) * (float)cam.height - 1.0f) * 0.5f;

    float c3[6];
    if (c3_in) {
#pragma unroll
        for (int k = 0; k < 6; k++) c3[k] = c3_in[k];
    } else {
        cov3d(sc, sp.cfg.scale_modifier, q, c3);
    }
    Ewa e;
    ewa_setup(p, cam.view_matrix, sp.focal_x, sp.focal_y, cam.tan_fovx, cam.tan_fovy, e);
    float c2[3];
    cov2d(e, c3, c2);
    const float det_cov = c2[0] * c2[2] - c2[1] * c2[1];
    c2[0] += 0.3f;
    c2[2] += 0.3f;
    const float det = c2[0] * c2[2] - c2[1] * c2[1];
    float hconv = 1.0f;
    if (sp.cfg.antialiasing) hconv = sqrtf(fmax_ref(0.000025f, det_cov / det));
    if (det == 0.0f) return false;
    const float dinv = 1.0f / det;
    const float mid = 0.5f * (c2[0] + c2[2]);
    const float l1 = mid + sqrtf(fmax_ref(0.1f, mid * mid - det));
    const float l2 = mid - sqrtf(fmax_ref(0.1f, mid * mid - det));
    const int radius = (int)ceilf(3.0f * sqrtf(fmax_ref(l1, l2)));
    if (radius > max(cam.width, cam.height)) return false;
    tile_rect(pix_x, pix_y, radius, sp.grid_x, sp.grid_y, sp.cfg.tile_w, sp.cfg.tile_h, r.rmn, r.rmx);
    if ((r.rmx[0] - r.rmn[0]) * (r.rmx[1] - r.rmn[1]) == 0) return false;

    float d[3];
    view_dir(p, cam.cam_pos, d);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float v = fmax_ref(0.0f, sh_channel(sp.sh_deg_fwd, sh, c, d[0], d[1], d[2]) + 0.5f);
        if (!sp.cfg.training) v = fmin_ref(1.0f, v);
        r.rgb[c] = v;
    }
    r.px = pix_x;
    r.py = pix_y;
    r.depth = pv[2];
    r.con[0] = c2[2] * dinv;
    r.con[1] = -c2[1] * dinv;
    r.con[2] = c2[0] * dinv;
    r.opac = op * hconv;
    r.radius = radius;
#pragma unroll
    for (int k = 0; k < 6; k++) r.cov3[k] = c3[k];
#pragma unroll
    for (int k = 0; k < 3; k++) r.pv[k] = pv[k];
    r.phw = ph[3];
#pragma unroll
    for (int k = 0; k < 3; k++) r.cov2[k] = c2[k];
    r.det = det;
    return true;
}

// Adam element update (optimizer.cpp:32-43), same rounding sequence.
__device__ __forceinline__ float adam_elem(float p, float& m, float& v, float g, float lr, float b1, float b2,
                                           float eps, float bc1, float bc2) {
    m = b1 * m + (1.0f - b1) * g;
    v = b2 * v + (1.0f - b2) * g * g;
    const float mh = m * bc1;
    const float vh = v * bc2;
    return p - lr * mh / (sqrtf(vh) + eps);
}

__device__ __forceinline__ void apply_update(const StepParams& sp, float* p, float* m, float* v, float g,
                                             float lr) {
    if (sp.use_adam) {
        float mm = *m, vv = *v;
        *p = adam_elem(*p, mm, vv, g, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
        *m = mm;
        *v = vv;
    } else {
        *p = *p - lr * g;  // SGD, optimizer.cpp:14-25
    }
}

// Inputs of one Gaussian's backward: raw parameters and its screen-space gradients.
struct BwdIn {
    float p[3], rsc[3], rq[4], rop;
    const float* act;  // non-NULL: activated (scale[3], rot[4], opacity) of an activated model; rq stays raw
    const float* sh;   // this Gaussian's SH coefficients, basis-major with stride 3
    float dm[2], dcn[3], drgb[3], dop;
};

// Gradients w.r.t. the raw parameters; the SH gradient is basis[k] * geff[c].
struct BwdOut {
    float gp[3], gs[3], gq[4], gop, geff[3], basis[16];
};

// The view-dependent part of one Gaussian's adjoint of
// PreprocessorBackwardCPU::backward (preprocessor_backward_cpu.cpp:205-645)
// for one camera: the SH chain (:8-203) into o.geff, o.basis and the position;
// then, when the recomputed 2D covariance is not degenerate, chains 1a-1b
// (conic -> cov2D -> cov3D, :243-380) into dcov, path A (:536-597) and chain 4
// (:609-643) into the position.  c3 is the forward's cov3D (cov3d of the
// activated scale and rotation), sc / q the activated scale and rotation.
// Returns false for det == 0, where the reference stops (dcov untouched).
// Every output is linear in the screen gradients of `in`, so the gradients of
// several cameras are the sums of their parts.
__device__ __forceinline__ bool backward_view(const StepParams& sp, const float p[3], const float c3[6],
                                              const float* shp, const BwdIn& in, BwdOut& o, float dcov[6]) {
    const gs3d_camera& cam = sp.cam;
    const int deg = sp.sh_deg_model;
    // ---- chain 2: SH (:8-203) ----
    float d[3];
    const float len = view_dir(p, cam.cam_pos, d);
    const float x = d[0], y = d[1], z = d[2];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float rawc = sh_channel(deg, shp, c, x, y, z);
        o.geff[c] = in.drgb[c] * ((rawc + 0.5f >= 0.0f) ? 1.0f : 0.0f);
    }
    o.basis[0] = SH_C0;
    if (deg > 0) {
        o.basis[1] = -SH_C1 * y;
        o.basis[2] = SH_C1 * z;
        o.basis[3] = -SH_C1 * x;
        if (deg > 1) {
            const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            o.basis[4] = SH_C20 * xy;
            o.basis[5] = SH_C21 * yz;
            o.basis[6] = SH_C22 * (2.0f * zz - xx - yy);
            o.basis[7] = SH_C23 * xz;
            o.basis[8] = SH_C24 * (xx - yy);
            if (deg > 2) {
                o.basis[9] = SH_C30 * y * (3.0f * xx - yy);
                o.basis[10] = SH_C31 * xy * z;
                o.basis[11] = SH_C32 * y * (4.0f * zz - xx - yy);
                o.basis[12] = SH_C33 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
                o.basis[13] = SH_C34 * x * (4.0f * zz - xx - yy);
                o.basis[14] = SH_C35 * z * (xx - yy);
                o.basis[15] = SH_C36 * x * (xx - 3.0f * yy);
            }
        }
        // d colour / d dir (:129-189)
        float dd0[3] = {0.f, 0.f, 0.f}, dd1[3] = {0.f, 0.f, 0.f}, dd2[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dd0[c] += -SH_C1 * shp[9 + c];
            dd1[c] += -SH_C1 * shp[3 + c];
            dd2[c] += SH_C1 * shp[6 + c];
        }
        if (deg > 1) {
            const float xx = x * x, yy = y * y, zz = z * z;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float s4 = shp[12 + c], s5 = shp[15 + c], s6 = shp[18 + c], s7 = shp[21 + c], s8 = shp[24 + c];
                dd0[c] += SH_C20 * y * s4 - 2.0f * SH_C22 * x * s6 + SH_C23 * z * s7 + 2.0f * SH_C24 * x * s8;
                dd1[c] += SH_C20 * x * s4 + SH_C21 * z * s5 - 2.0f * SH_C22 * y * s6 - 2.0f * SH_C24 * y * s8;
                dd2[c] += SH_C21 * y * s5 + 4.0f * SH_C22 * z * s6 + SH_C23 * x * s7;
            }
            if (deg > 2) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float s9 = shp[27 + c], s10 = shp[30 + c], s11 = shp[33 + c], s12 = shp[36 + c];
                    const float s13 = shp[39 + c], s14 = shp[42 + c], s15 = shp[45 + c];
                    dd0[c] += SH_C30 * 6.0f * x * y * s9 + SH_C31 * y * z * s10 + SH_C32 * (-2.0f * x * y) * s11 +
                              SH_C33 * (-6.0f * x * z) * s12 + SH_C34 * (4.0f * zz - 3.0f * xx - yy) * s13 +
                              SH_C35 * 2.0f * x * z * s14 + SH_C36 * (3.0f * xx - 3.0f * yy) * s15;
                    dd1[c] += SH_C30 * (3.0f * xx - 3.0f * yy) * s9 + SH_C31 * x * z * s10 +
                              SH_C32 * (4.0f * zz - xx - 3.0f * yy) * s11 + SH_C33 * (-6.0f * y * z) * s12 +
                              SH_C34 * (-2.0f * x * y) * s13 - SH_C35 * 2.0f * y * z * s14 +
                              SH_C36 * (-6.0f * x * y) * s15;
                    dd2[c] += SH_C31 * x * y * s10 + SH_C32 * 8.0f * y * z * s11 +
                              SH_C33 * (6.0f * zz - 3.0f * xx - 3.0f * yy) * s12 + SH_C34 * 8.0f * x * z * s13 +
                              SH_C35 * (xx - yy) * s14;
                }
            }
        }
        float ddir0 = 0.f, ddir1 = 0.f, ddir2 = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) ddir0 += o.geff[c] * dd0[c];
#pragma unroll
        for (int c = 0; c < 3; c++) ddir1 += o.geff[c] * dd1[c];
#pragma unroll
        for (int c = 0; c < 3; c++) ddir2 += o.geff[c] * dd2[c];
        const float inv_len = 1.0f / len;
        const float dot = ddir0 * x + ddir1 * y + ddir2 * z;
        o.gp[0] += (ddir0 - x * dot) * inv_len;
        o.gp[1] += (ddir1 - y * dot) * inv_len;
        o.gp[2] += (ddir2 - z * dot) * inv_len;
    }
    // ---- forward recompute (the ForwardCache of preprocessor_cpu.cpp:254-264) ----
    Ewa e;
    ewa_setup(p, cam.view_matrix, sp.focal_x, sp.focal_y, cam.tan_fovx, cam.tan_fovy, e);
    float c2[3];
    cov2d(e, c3, c2);
    c2[0] += 0.3f;
    c2[2] += 0.3f;
    const float det = c2[0] * c2[2] - c2[1] * c2[1];
    if (det == 0.0f) return false;
    float ph[4];
    xform4x4(p, cam.viewproj_matrix, ph);
    // ---- chain 1a: conic -> cov2D (:243-306) ----
    const float a = c2[0], b = c2[1], c = c2[2];
    const float inv_det = 1.0f / det;
    const float id2 = inv_det * inv_det;
    const float* dcn = in.dcn;
    const float d_a = dcn[0] * (-c * c * id2) + dcn[1] * (b * c * id2) + dcn[2] * (-b * b * id2);
    const float d_b = dcn[0] * (2.0f * b * c * id2) + dcn[1] * (-(a * c + b * b) * id2) + dcn[2] * (2.0f * a * b * id2);
    const float d_c = dcn[0] * (-b * b * id2) + dcn[1] * (a * b * id2) + dcn[2] * (-a * a * id2);
    // ---- chain 1b: cov2D -> cov3D (:316-380) ----
    float dV[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            dV[k][j] = d_a * e.T[0][k] * e.T[0][j] + d_b * e.T[0][k] * e.T[1][j] + d_c * e.T[1][k] * e.T[1][j];
    dcov[0] = dV[0][0];
    dcov[1] = dV[0][1] + dV[1][0];
    dcov[2] = dV[0][2] + dV[2][0];
    dcov[3] = dV[1][1];
    dcov[4] = dV[1][2] + dV[2][1];
    dcov[5] = dV[2][2];
    // ---- path A: cov2D -> T -> J -> p_view -> position (:536-597) ----
    const float V[3][3] = {{c3[0], c3[1], c3[2]}, {c3[1], c3[3], c3[4]}, {c3[2], c3[4], c3[5]}};
    float VT[2][3];
#pragma unroll
    for (int col = 0; col < 2; col++)
#pragma unroll
        for (int row = 0; row < 3; row++) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; k++) acc += V[row][k] * e.T[col][k];
            VT[col][row] = acc;
        }
    float dT[2][3];
#pragma unroll
    for (int qq = 0; qq < 3; qq++) {
        dT[0][qq] = 2.0f * d_a * VT[0][qq] + d_b * VT[1][qq];
        dT[1][qq] = d_b * VT[0][qq] + 2.0f * d_c * VT[1][qq];
    }
    float dJ[2][3];
#pragma unroll
    for (int col = 0; col < 2; col++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float acc = 0.0f;
#pragma unroll
            for (int row = 0; row < 3; row++) acc += dT[col][row] * e.W[k][row];
            dJ[col][k] = acc;
        }
    const float* t = e.t;
    const float tz2 = t[2] * t[2];
    const float tz3 = tz2 * t[2];
    const float fx = sp.focal_x, fy = sp.focal_y;
    float dt0 = dJ[0][2] * (-fx / tz2);
    float dt1 = dJ[1][2] * (-fy / tz2);
    const float dt2 = dJ[0][0] * (-fx / tz2) + dJ[1][1] * (-fy / tz2) + dJ[0][2] * (2.0f * fx * t[0] / tz3) +
                      dJ[1][2] * (2.0f * fy * t[1] / tz3);
    if (fabsf(e.txtz) >= e.limx) dt0 = 0.0f;
    if (fabsf(e.tytz) >= e.limy) dt1 = 0.0f;
    const float* vm = cam.view_matrix;
#pragma unroll
    for (int col = 0; col < 3; col++) {
        o.gp[col] += dt0 * vm[col * 4 + 0];
        o.gp[col] += dt1 * vm[col * 4 + 1];
        o.gp[col] += dt2 * vm[col * 4 + 2];
    }
    // ---- chain 4: means2D -> ndc -> p_hom -> position (:609-643) ----
    // means2D recomputed exactly as the forward wrote it (preprocessor_cpu.cpp:195-203)
    const float pw = 1.0f / (ph[3] + 1e-7f);
    const float pix_x = ((ph[0] * pw + 1.0f) * (float)cam.width - 1.0f) * 0.5f;
    const float pix_y = ((ph[1] * pw + 1.0f) * (float)cam.height - 1.0f) * 0.5f;
    const float dndx = in.dm[0] * (float)cam.width * 0.5f;
    const float dndy = in.dm[1] * (float)cam.height * 0.5f;
    const float wh = ph[3] + 1e-7f;
    const float iw = 1.0f / wh;
    const float ndc_x = (2.0f * pix_x + 1.0f) / (float)cam.width - 1.0f;
    const float ndc_y = (2.0f * pix_y + 1.0f) / (float)cam.height - 1.0f;
    const float dph0 = dndx * iw, dph1 = dndy * iw, dph2 = 0.0f;
    const float dph3 = -(ndc_x * dndx + ndc_y * dndy) * iw;
    const float* VP = cam.viewproj_matrix;
#pragma unroll
    for (int dim = 0; dim < 3; dim++)
        o.gp[dim] += VP[dim * 4 + 0] * dph0 + VP[dim * 4 + 1] * dph1 + VP[dim * 4 + 2] * dph2 + VP[dim * 4 + 3] * dph3;
    return true;
}

// The view-independent part: a cov3D gradient through M = S R (chain 1c,
// :395-442) and the rotation matrix into the unit quaternion (:455-498), then
// the quaternion normalisation (:503-519) against the raw quaternion rq, into
// o.gs and o.gq.  mod = RenderConfig::scale_modifier.
__device__ __forceinline__ void backward_cov3d(float mod, const float sc[3], const float q[4], const float rq[4],
                                               const float dcov[6], BwdOut& o) {
    // ---- chain 1c: cov3D -> M -> scale, R (:395-442) ----
    const float sv[3] = {mod * sc[0], mod * sc[1], mod * sc[2]};
    const float rr = q[0], xq = q[1], yq = q[2], zq = q[3];
    float R[3][3], M[3][3];
    quat_to_R(rr, xq, yq, zq, R);
#pragma unroll
    for (int ii = 0; ii < 3; ii++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) M[ii][jj] = sv[ii] * R[ii][jj];
    float dR[3][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float dM0 = 2.0f * dcov[0] * M[k][0] + dcov[1] * M[k][1] + dcov[2] * M[k][2];
        const float dM1 = dcov[1] * M[k][0] + 2.0f * dcov[3] * M[k][1] + dcov[4] * M[k][2];
        const float dM2 = dcov[2] * M[k][0] + dcov[4] * M[k][1] + 2.0f * dcov[5] * M[k][2];
        float ds = 0.0f;
        ds += dM0 * R[k][0];
        ds += dM1 * R[k][1];
        ds += dM2 * R[k][2];
        dR[k][0] = dM0 * sv[k];
        dR[k][1] = dM1 * sv[k];
        dR[k][2] = dM2 * sv[k];
        o.gs[k] = ds * mod * sc[k];
    }
    // ---- d R -> d unit quaternion (:455-498) ----
    float dq0 = 0.f, dq1 = 0.f, dq2 = 0.f, dq3 = 0.f;
    dq2 += dR[0][0] * (-4.0f * yq);
    dq3 += dR[0][0] * (-4.0f * zq);
    dq0 += dR[0][1] * 2.0f * zq; dq1 += dR[0][1] * 2.0f * yq;
    dq2 += dR[0][1] * 2.0f * xq; dq3 += dR[0][1] * 2.0f * rr;
    dq0 += dR[0][2] * (-2.0f * yq); dq1 += dR[0][2] * 2.0f * zq;
    dq2 += dR[0][2] * (-2.0f * rr); dq3 += dR[0][2] * 2.0f * xq;
    dq0 += dR[1][0] * (-2.0f * zq); dq1 += dR[1][0] * 2.0f * yq;
    dq2 += dR[1][0] * 2.0f * xq; dq3 += dR[1][0] * (-2.0f * rr);
    dq1 += dR[1][1] * (-4.0f * xq);
    dq3 += dR[1][1] * (-4.0f * zq);
    dq0 += dR[1][2] * 2.0f * xq; dq1 += dR[1][2] * 2.0f * rr;
    dq2 += dR[1][2] * 2.0f * zq; dq3 += dR[1][2] * 2.0f * yq;
    dq0 += dR[2][0] * 2.0f * yq; dq1 += dR[2][0] * 2.0f * zq;
    dq2 += dR[2][0] * 2.0f * rr; dq3 += dR[2][0] * 2.0f * xq;
    dq0 += dR[2][1] * (-2.0f * xq); dq1 += dR[2][1] * (-2.0f * rr);
    dq2 += dR[2][1] * 2.0f * zq; dq3 += dR[2][1] * 2.0f * yq;
    dq1 += dR[2][2] * (-4.0f * xq);
    dq2 += dR[2][2] * (-4.0f * yq);
    // ---- normalisation backward (:503-519) ----
    float qlen = sqrtf(rq[0] * rq[0] + rq[1] * rq[1] + rq[2] * rq[2] + rq[3] * rq[3]);
    if (qlen < 1e-12f) qlen = 1e-12f;
    const float il = 1.0f / qlen;
    const float dot = dq0 * rr + dq1 * xq + dq2 * yq + dq3 * zq;
    o.gq[0] = (dq0 - rr * dot) * il;
    o.gq[1] = (dq1 - xq * dot) * il;
    o.gq[2] = (dq2 - yq * dot) * il;
    o.gq[3] = (dq3 - zq * dot) * il;
}

// The whole per-Gaussian adjoint chain of PreprocessorBackwardCPU::backward
// (preprocessor_backward_cpu.cpp:205-645) for a visible Gaussian, with the
// forward quantities (activation, p_view, cov3D, cov2D, det, means2D)
// recomputed bit-identically instead of read from a cache.
__device__ __forceinline__ void backward_one(const StepParams& sp, const BwdIn& in, BwdOut& o) {
    float sc[3], q[4], op;
    if (in.act) {
#pragma unroll
        for (int k = 0; k < 3; k++) sc[k] = in.act[k];
#pragma unroll
        for (int k = 0; k < 4; k++) q[k] = in.act[3 + k];
        op = in.act[7];
    } else {
        activate_one(in.rsc, in.rq, in.rop, sc, q, &op);
    }
    // ---- chain 3: sigmoid (:231-232) ----
    o.gop = in.dop * op * (1.0f - op);
    float c3[6];
    cov3d(sc, sp.cfg.scale_modifier, q, c3);
    float dcov[6];
    if (backward_view(sp, in.p, c3, in.sh, in, o, dcov)) backward_cov3d(sp.cfg.scale_modifier, sc, q, in.rq, dcov, o);
}


}  // namespace
}  // namespace gs3d
