// eval3d.cuh -- the reference's 3D-evaluation render mode (RenderConfig::eval_3D,
// "AAA-Gaussians") for sm_100a.  Included by plain.cu, so it is compiled with
// the plain form's flags (-fmad=false, IEEE division and square root) and
// every float operation below rounds like the reference's x86 build; the
// operation order follows harmonyos_3dgs src/math_utils.cpp:152-696,
// src/cpu/preprocessor_cpu.cpp:64-187, src/cpu/tile_binner_cpu.cpp:16-20,59-99
// and src/cpu/rasterizer_cpu.cpp:15-21,61-135.
//
// Kernels:
//   k_e3_view        the inverse view-projection (computed on the device, in
//                    the reference's cofactor order) and the unit ray through
//                    every tile centre;
//   k_preprocess_e3  one thread per Gaussian: gauss2screen with the 3D mip
//                    filter, whole-screen frustum culling by the maximum
//                    contribution, screen (or view) bounding box, inverse 3D
//                    covariance, SH colour; then the block scan + look-back
//                    emission of the pairs, each key carrying the Gaussian's
//                    depth along its tile's centre ray;
//   k_bin_arrays_e3  the same emission from host-provided arrays;
//   k_raster_e3      one CTA per 16x16 tile, one thread per pixel: exact ray
//                    maximum of every Gaussian of the tile, accepted ones
//                    kept in a 16-entry buffer sorted by depth along the
//                    pixel's ray (a ring in shared memory), blended front to
//                    back when it overflows and flushed at the end.
#pragma once

#include <climits>

namespace gs3d {
namespace {

constexpr float kE3Pi = 3.14159265358979323846f;   // (float)M_PI
constexpr int kKBuf = 16;                           // StopThePop buffer (rasterizer_cpu.cpp:63)
constexpr int kE3Batch = 64;                        // records staged per batch
constexpr int kE3Threads = 256;                     // one thread per pixel of a 16x16 tile

// x86 float -> int32 truncation (cvttss2si): NaN and out-of-range give INT_MIN.
__device__ __forceinline__ int cvt_trunc_x86(float f) {
    return (f >= -2147483648.0f && f < 2147483648.0f) ? (int)f : INT_MIN;
}

// getRect (math_utils.cpp:21-28) with the x86 conversions.
__device__ __forceinline__ void tile_rect_x86(float px, float py, int r, int gx, int gy, int tw, int th, int rmn[2],
                                              int rmx[2]) {
    const float fr = (float)r, ftw = (float)tw, fth = (float)th;
    rmn[0] = min(gx, max(0, cvt_trunc_x86((px - fr) / ftw)));
    rmn[1] = min(gy, max(0, cvt_trunc_x86((py - fr) / fth)));
    rmx[0] = min(gx, max(0, cvt_trunc_x86((px + fr + ftw - 1.0f) / ftw)));
    rmx[1] = min(gy, max(0, cvt_trunc_x86((py + fr + fth - 1.0f) / fth)));
}

// Correctly rounded float results of the libm functions the mode calls (the
// reference's glibc atan2f / tanf / logf differ from these by one ulp on a
// small share of inputs).
__device__ __forceinline__ float atan2_ref(float y, float x) { return (float)atan2((double)y, (double)x); }
__device__ __forceinline__ float tan_ref(float x) { return (float)tan((double)x); }
__device__ __forceinline__ float log_ref(float x) { return (float)log((double)x); }

// math_utils.cpp:158-163 (the transpose of computeCov3D's layout)
__device__ __forceinline__ void quat2mat_e3(const float q[4], float R[3][3]) {
    const float r = q[0], x = q[1], y = q[2], z = q[3];
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

// out = A * B, column-major, every sum started from zero (math_utils.cpp:166-174)
__device__ __forceinline__ void mat4mul_e3(const float A[16], const float B[16], float out[16]) {
#pragma unroll
    for (int col = 0; col < 4; col++)
#pragma unroll
        for (int row = 0; row < 4; row++) {
            float s = 0.0f;
#pragma unroll
            for (int k = 0; k < 4; k++) s += A[k * 4 + row] * B[col * 4 + k];
            out[col * 4 + row] = s;
        }
}

// Squared Mahalanobis distance of the line where two Gaussian-space planes
// meet (math_utils.cpp:186-207); mp = its closest point.
__device__ __forceinline__ float ray_max_e3(const float a[4], const float b[4], float mp[4]) {
    const float dx = a[1] * b[2] - a[2] * b[1];
    const float dy = a[2] * b[0] - a[0] * b[2];
    const float dz = a[0] * b[1] - a[1] * b[0];
    const float mx = a[3] * b[0] - a[0] * b[3];
    const float my = a[3] * b[1] - a[1] * b[3];
    const float mz = a[3] * b[2] - a[2] * b[3];
    const float dd = dx * dx + dy * dy + dz * dz;
    const float q0 = mx / dd, q1 = my / dd, q2 = mz / dd;
    mp[0] = dy * q2 - dz * q1;
    mp[1] = dz * q0 - dx * q2;
    mp[2] = dx * q1 - dy * q0;
    mp[3] = 1.0f;
    return mx * q0 + my * q1 + mz * q2;
}

// The same distance alone (the rasteriser does not use the point).
__device__ __forceinline__ float ray_dist_e3(const float a[4], const float b[4]) {
    const float dx = a[1] * b[2] - a[2] * b[1];
    const float dy = a[2] * b[0] - a[0] * b[2];
    const float dz = a[0] * b[1] - a[1] * b[0];
    const float mx = a[3] * b[0] - a[0] * b[3];
    const float my = a[3] * b[1] - a[1] * b[3];
    const float mz = a[3] * b[2] - a[2] * b[3];
    const float dd = dx * dx + dy * dy + dz * dz;
    return mx * (mx / dd) + my * (my / dd) + mz * (mz / dd);
}

// g2s^T v for row-major g2s, sums from zero (math_utils.cpp:216-220, 243-247)
__device__ __forceinline__ void to_screen_e3(const float g2s[16], const float v[4], float out[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; j++) s += g2s[j * 4 + i] * v[j];
        out[i] = s;
    }
}

// math_utils.cpp:210-222
__device__ __forceinline__ float plane_max_e3(const float pl[4], const float g2s[16], float mps[4]) {
    const float norm = pl[3] / (pl[0] * pl[0] + pl[1] * pl[1] + pl[2] * pl[2]);
    const float mpg[4] = {-pl[0] * norm, -pl[1] * norm, -pl[2] * norm, -pl[3] * norm};
    to_screen_e3(g2s, mpg, mps);
    return -mpg[3];
}

// math_utils.cpp:225-234
__device__ __forceinline__ bool in_range_e3(const float ps[4], const float from[3], const float ext[3], int dim,
                                            float& d) {
    d = ps[dim] - from[dim] * ps[3];
    return d > 0.0f && d < ext[dim] * ps[3];
}
__device__ __forceinline__ bool in_range_e3(const float ps[4], const float from[3], const float ext[3], int dim) {
    float d;
    return in_range_e3(ps, from, ext, dim, d);
}

// 0.5 x the minimum squared distance over the screen rectangle's frustum
// (math_utils.cpp:253-340): the mean when inside, else the closer side
// planes, their intersection and the two mixed intersections, in that order.
__device__ float frustum_max_e3(float x0, float y0, float x1, float y1, const float g2s[16]) {
    float best = 1e30f;
    const float from[3] = {x0, y0, -1.0f};
    const float ext[3] = {x1 - x0, y1 - y0, 1.0f - -1.0f};
    const float mean[4] = {g2s[3], g2s[7], g2s[11], g2s[15]};
    float d[3];
    const bool bx = in_range_e3(mean, from, ext, 0, d[0]);
    const bool by = in_range_e3(mean, from, ext, 1, d[1]);
    const bool bz = in_range_e3(mean, from, ext, 2, d[2]);
    if (bx && by && bz) return 0.0f;   // 0.5 * 0
    const float sx = (d[0] - (ext[0] * 0.5f * mean[3])) >= 0 ? ext[0] * 0.5f : -ext[0] * 0.5f;
    const float sy = (d[1] - (ext[1] * 0.5f * mean[3])) >= 0 ? ext[1] * 0.5f : -ext[1] * 0.5f;
    const float cx = from[0] + ext[0] * 0.5f + sx;
    const float cy = from[1] + ext[1] * 0.5f + sy;
    float px[4], py[4], ps[4], mg[4], c;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        px[i] = g2s[i] - g2s[12 + i] * cx;
        py[i] = g2s[4 + i] - g2s[12 + i] * cy;
    }
    c = plane_max_e3(px, g2s, ps);
    if (c < best && in_range_e3(ps, from, ext, 1) && in_range_e3(ps, from, ext, 2)) best = c;
    c = plane_max_e3(py, g2s, ps);
    if (c < best && in_range_e3(ps, from, ext, 0) && in_range_e3(ps, from, ext, 2)) best = c;
    c = ray_max_e3(px, py, mg);
    to_screen_e3(g2s, mg, ps);
    if (c < best && in_range_e3(ps, from, ext, 2)) best = c;
    float o[4];
    const float ocy = from[1] + ext[1] * 0.5f - sy;
#pragma unroll
    for (int i = 0; i < 4; i++) o[i] = g2s[4 + i] - g2s[12 + i] * ocy;
    c = ray_max_e3(px, o, mg);
    to_screen_e3(g2s, mg, ps);
    if (c < best && in_range_e3(ps, from, ext, 2)) best = c;
    const float ocx = from[0] + ext[0] * 0.5f - sx;
#pragma unroll
    for (int i = 0; i < 4; i++) o[i] = g2s[i] - g2s[12 + i] * ocx;
    c = ray_max_e3(o, py, mg);
    to_screen_e3(g2s, mg, ps);
    if (c < best && in_range_e3(ps, from, ext, 2)) best = c;
    return 0.5f * best;
}

// Screen-space bounding box of the cutoff ellipsoid (math_utils.cpp:342-389).
__device__ bool aabb_screen_e3(const float g2s[16], float cutoff, float ext[2]) {
    const float t[4] = {cutoff, cutoff, cutoff, -1.0f};
    const float *r0 = g2s, *r1 = g2s + 4, *r2 = g2s + 8, *r3 = g2s + 12;
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; k++) s += t[k] * r3[k] * r3[k];
    if (s >= 0.0f) return false;
    float f[4];
#pragma unroll
    for (int k = 0; k < 4; k++) f[k] = t[k] / s;
    float p[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        p[0] += f[k] * r0[k] * r3[k];
        p[1] += f[k] * r1[k] * r3[k];
        p[2] += f[k] * r2[k] * r3[k];
    }
    float h[3] = {p[0] * p[0], p[1] * p[1], p[2] * p[2]};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        h[0] -= f[k] * r0[k] * r0[k];
        h[1] -= f[k] * r1[k] * r1[k];
        h[2] -= f[k] * r2[k] * r2[k];
    }
    const float ez = sqrtf(fmax_ref(0.0f, h[2]));
    const float zlo = p[2] - ez, zhi = p[2] + ez;
    if (zlo < -1.0f || zhi > 1.0f) return false;
    ext[0] = sqrtf(fmax_ref(0.0f, h[0]));
    ext[1] = sqrtf(fmax_ref(0.0f, h[1]));
    return true;
}

// math_utils.cpp:391-396
__device__ __forceinline__ float norm_angle_e3(float th) {
    th = fmodf(th, 2.0f * kE3Pi);
    if (th > kE3Pi) th -= 2.0f * kE3Pi;
    if (th <= -kE3Pi) th += 2.0f * kE3Pi;
    return th;
}

// Tangents of the view-space angles bounding the ellipsoid about one image
// axis (math_utils.cpp:408-456).  The angle rotations are bounded loops (the
// reference's while loops run at most a few times for finite angles).
__device__ void theta_e3(const float g2v[16], const float vd[3], float cutoff, int axis, float& lo_t, float& hi_t) {
    const float t[4] = {cutoff, cutoff, cutoff, -1.0f};
    const float mu = atan2_ref(axis == 0 ? vd[0] : vd[1], vd[2]);
    const float* Ta = g2v + axis * 4;
    const float* T2 = g2v + 8;
    float sa = 0.0f, sz = 0.0f, mv = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        sa += t[i] * Ta[i] * Ta[i];
        sz += t[i] * T2[i] * T2[i];
        mv += t[i] * Ta[i] * T2[i];
    }
    const float inside = mv * mv - sz * sa;
    float lo = -(kE3Pi / 2.0f - 1e-5f);
    float hi = kE3Pi / 2.0f - 1e-5f;
    if (inside > 0.0f) {
        const float sq = sqrtf(inside);
        float a0 = atan2_ref(-(mv + sq), -sz);
        float a1 = atan2_ref(-(mv - sq), -sz);
        for (int it = 0; it < 64 && a0 > mu; it++) a0 -= kE3Pi;
        for (int it = 0; it < 64 && a0 < (mu - kE3Pi); it++) a0 += kE3Pi;
        for (int it = 0; it < 64 && a1 < mu; it++) a1 += kE3Pi;
        for (int it = 0; it < 64 && a1 > (mu + kE3Pi); it++) a1 -= kE3Pi;
        const float n0 = norm_angle_e3(a0);
        const float n1 = norm_angle_e3(a1);
        if (mu < 0.0f && fabsf(n0) < fabsf(n1)) {
            a0 += 2.0f * kE3Pi;
            a1 += 2.0f * kE3Pi;
        } else if (mu > 0.0f && fabsf(n1) < fabsf(n0)) {
            a0 -= 2.0f * kE3Pi;
            a1 -= 2.0f * kE3Pi;
        }
        lo = fmax_ref(lo, a0);
        hi = fmin_ref(hi, a1);
    }
    lo_t = tan_ref(lo);
    hi_t = tan_ref(hi);
}

// View-space bounding box, the fallback (math_utils.cpp:398-472).
__device__ void aabb_view_e3(const float g2v[16], const float mv[3], float fx, float fy, float W, float H,
                             float cutoff, float ext[2]) {
    const float vlen = sqrtf(mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2]);
    const float vd[3] = {mv[0] / vlen, mv[1] / vlen, mv[2] / vlen};
    float bxl, bxh, byl, byh;
    theta_e3(g2v, vd, cutoff, 0, bxl, bxh);
    theta_e3(g2v, vd, cutoff, 1, byl, byh);
    const float xl = W / 2.0f + fx * bxl, xh = W / 2.0f + fx * bxh;
    const float yl = H / 2.0f + fy * byl, yh = H / 2.0f + fy * byh;
    ext[0] = (xh - xl) / 2.0f;
    ext[1] = (yh - yl) / 2.0f;
}

// gauss2screen / gauss2view, row-major, with the mip-filter dilation; returns
// the opacity's dilation factor (math_utils.cpp:474-584, kernel_size > 0).
__device__ float gauss2screen_e3(const float mean[3], const float scale[3], const float rot[4], float mod,
                                 const float cam_pos[3], const float* vp_m, const float* view_m, float focal,
                                 float kernel, float filt, int W, int H, float g2s[16], float g2v[16]) {
    float R[3][3];
    quat2mat_e3(rot, R);
    float vr[3] = {mean[0] - cam_pos[0], mean[1] - cam_pos[1], mean[2] - cam_pos[2]};
    const float vl = sqrtf(vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]);
    vr[0] /= vl;
    vr[1] /= vl;
    vr[2] /= vl;
    float vg[3];
#pragma unroll
    for (int i = 0; i < 3; i++) vg[i] = R[i][0] * vr[0] + R[i][1] * vr[1] + R[i][2] * vr[2];
    const float rs[3] = {vg[0] * vg[0], vg[1] * vg[1], vg[2] * vg[2]};
    float mvw[3];
    xform4x3(mean, view_m, mvw);
    const float q = mvw[2] / focal;
    float mip = q * q * kernel;
    mip = fmax_ref(filt * filt, mip);
    float sd3[3];
#pragma unroll
    for (int j = 0; j < 3; j++) sd3[j] = sqrtf(scale[j] * scale[j] + mip);
    const float s[3] = {scale[0] * scale[0], scale[1] * scale[1], scale[2] * scale[2]};
    const float sdl[3] = {sd3[0] * sd3[0], sd3[1] * sd3[1], sd3[2] * sd3[2]};
    const float dm = rs[0] * (s[1] * s[2]) + rs[1] * (s[2] * s[0]) + rs[2] * (s[0] * s[1]);
    const float dmd = rs[0] * (sdl[1] * sdl[2]) + rs[1] * (sdl[2] * sdl[0]) + rs[2] * (sdl[0] * sdl[1]);
    const float dil = sqrtf(dm / dmd);
    const float sm = sqrtf(mod);
    const float sd[3] = {sd3[0] * sm, sd3[1] * sm, sd3[2] * sm};
    float g2w[16];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        // L[row][c] = sd[c] * R[c][row]
        g2w[c * 4 + 0] = sd[c] * R[c][0];
        g2w[c * 4 + 1] = sd[c] * R[c][1];
        g2w[c * 4 + 2] = sd[c] * R[c][2];
        g2w[c * 4 + 3] = 0.0f;
    }
    g2w[12] = mean[0];
    g2w[13] = mean[1];
    g2w[14] = mean[2];
    g2w[15] = 1.0f;
    float vpt[16];
#pragma unroll
    for (int k = 0; k < 16; k++) vpt[k] = 0.0f;
    vpt[0] = (float)W / 2.0f;
    vpt[5] = (float)H / 2.0f;
    vpt[10] = 1.0f;
    vpt[15] = 1.0f;
    vpt[12] = (float)W / 2.0f - 0.5f;
    vpt[13] = (float)H / 2.0f - 0.5f;
    float w2s[16], cm[16];
    mat4mul_e3(vpt, vp_m, w2s);
    mat4mul_e3(w2s, g2w, cm);
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) g2s[r * 4 + c] = cm[c * 4 + r];
    mat4mul_e3(view_m, g2w, cm);
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) g2v[r * 4 + c] = cm[c * 4 + r];
    return dil;
}

// Upper triangle of R^T diag(1/sd^2) R (math_utils.cpp:590-614)
__device__ __forceinline__ void cov3d_inv_e3(const float sdil[3], float mod, const float rot[4], float ci[6]) {
    float R[3][3];
    quat2mat_e3(rot, R);
    const float sm = sqrtf(mod);
    float is2[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const float s = sdil[j] * sm;
        is2[j] = 1.0f / (s * s);
    }
    int idx = 0;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = r; c < 3; c++) {
            float v = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; k++) v += R[k][r] * is2[k] * R[k][c];
            ci[idx++] = v;
        }
}

// Distance along the unit ray vd of the Gaussian's maximum (math_utils.cpp:616-630)
__device__ __forceinline__ float depth_along_ray_e3(const float ci[6], const float mo[3], const float vd[3]) {
    const float S0 = ci[0] * vd[0] + ci[1] * vd[1] + ci[2] * vd[2];
    const float S1 = ci[1] * vd[0] + ci[3] * vd[1] + ci[4] * vd[2];
    const float S2 = ci[2] * vd[0] + ci[4] * vd[1] + ci[5] * vd[2];
    const float num = mo[0] * S0 + mo[1] * S1 + mo[2] * S2;
    const float den = vd[0] * S0 + vd[1] * S1 + vd[2] * S2;
    if (fabsf(den) < 1e-10f) return sqrtf(mo[0] * mo[0] + mo[1] * mo[1] + mo[2] * mo[2]);
    return num / den;
}

// Unit world direction through pixel (px, py) (math_utils.cpp:632-651)
__device__ __forceinline__ void pixel_dir_e3(float px, float py, int w, int h, const float ivp[16],
                                             const float cam_pos[3], float d[3]) {
    const float nx = (2.0f * px + 1.0f) / (float)w - 1.0f;
    const float ny = (2.0f * py + 1.0f) / (float)h - 1.0f;
    float wp[4];
#pragma unroll
    for (int i = 0; i < 4; i++) wp[i] = ivp[i] * nx + ivp[4 + i] * ny + ivp[8 + i] * 0.0f + ivp[12 + i] * 1.0f;
    const float wi = 1.0f / (wp[3] + 1e-10f);
    d[0] = wp[0] * wi - cam_pos[0];
    d[1] = wp[1] * wi - cam_pos[1];
    d[2] = wp[2] * wi - cam_pos[2];
    const float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len > 1e-10f) {
        d[0] /= len;
        d[1] /= len;
        d[2] /= len;
    }
}

// Column-major 4x4 inverse by cofactors (math_utils.cpp:653-696); false when
// |det| < 1e-12.
__device__ bool invert4_e3(const float* m, float inv[16]) {
    const float a00 = m[0], a10 = m[1], a20 = m[2], a30 = m[3];
    const float a01 = m[4], a11 = m[5], a21 = m[6], a31 = m[7];
    const float a02 = m[8], a12 = m[9], a22 = m[10], a32 = m[11];
    const float a03 = m[12], a13 = m[13], a23 = m[14], a33 = m[15];
    const float b00 = a00 * a11 - a01 * a10, b01 = a00 * a12 - a02 * a10, b02 = a00 * a13 - a03 * a10;
    const float b03 = a01 * a12 - a02 * a11, b04 = a01 * a13 - a03 * a11, b05 = a02 * a13 - a03 * a12;
    const float b06 = a20 * a31 - a21 * a30, b07 = a20 * a32 - a22 * a30, b08 = a20 * a33 - a23 * a30;
    const float b09 = a21 * a32 - a22 * a31, b10 = a21 * a33 - a23 * a31, b11 = a22 * a33 - a23 * a32;
    const float det = b00 * b11 - b01 * b10 + b02 * b09 + b03 * b08 - b04 * b07 + b05 * b06;
    if (fabsf(det) < 1e-12f) return false;
    const float id = 1.0f / det;
    inv[0] = (a11 * b11 - a12 * b10 + a13 * b09) * id;
    inv[1] = (-a10 * b11 + a12 * b08 - a13 * b07) * id;
    inv[2] = (a10 * b10 - a11 * b08 + a13 * b06) * id;
    inv[3] = (-a10 * b09 + a11 * b07 - a12 * b06) * id;
    inv[4] = (-a01 * b11 + a02 * b10 - a03 * b09) * id;
    inv[5] = (a00 * b11 - a02 * b08 + a03 * b07) * id;
    inv[6] = (-a00 * b10 + a01 * b08 - a03 * b06) * id;
    inv[7] = (a00 * b09 - a01 * b07 + a02 * b06) * id;
    inv[8] = (a31 * b05 - a32 * b04 + a33 * b03) * id;
    inv[9] = (-a30 * b05 + a32 * b02 - a33 * b01) * id;
    inv[10] = (a30 * b04 - a31 * b02 + a33 * b00) * id;
    inv[11] = (-a30 * b03 + a31 * b01 - a32 * b00) * id;
    inv[12] = (-a21 * b05 + a22 * b04 - a23 * b03) * id;
    inv[13] = (a20 * b05 - a22 * b02 + a23 * b01) * id;
    inv[14] = (-a20 * b04 + a21 * b02 - a23 * b00) * id;
    inv[15] = (a20 * b03 - a21 * b01 + a22 * b00) * id;
    return true;
}

// Conservative pixel box (xmin, xmax, ymin, ymax of pixel indices) outside of
// which no pixel's ray gets within squared distance 2 thr of the Gaussian,
// i.e. where alpha stays below 1/255: the projected bounding box of the
// ellipsoid q <= 2 thr (1 + 1e-4) + 1e-3 (the construction of aabb_screen_e3,
// evaluated in FP64), shifted by the half-pixel of the ray's pixel centre and
// widened by one pixel.  No box (never skipped) when the ellipsoid reaches the
// camera plane.  Used only to skip work: it never changes a result.
__device__ float4 e3_skip_box(const float g2s[16], float thr) {
    const float4 none = make_float4(-1e30f, 1e30f, -1e30f, 1e30f);
    const double c = 2.0 * (double)thr * (1.0 + 1e-4) + 1e-3;
    const double t[4] = {c, c, c, -1.0};
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) s += t[k] * (double)g2s[12 + k] * (double)g2s[12 + k];
    if (!(s < 0.0)) return none;
    double p0 = 0.0, p1 = 0.0, h0 = 0.0, h1 = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double f = t[k] / s, r3 = g2s[12 + k], r0 = g2s[k], r1 = g2s[4 + k];
        p0 += f * r0 * r3;
        p1 += f * r1 * r3;
        h0 += f * r0 * r0;
        h1 += f * r1 * r1;
    }
    const double e0 = sqrt(fmax(0.0, p0 * p0 - h0)), e1 = sqrt(fmax(0.0, p1 * p1 - h1));
    const double x0 = p0 - e0 - 1.5, x1 = p0 + e0 + 0.5, y0 = p1 - e1 - 1.5, y1 = p1 + e1 + 0.5;
    if (!(fabs(x0) < 1e30 && fabs(x1) < 1e30 && fabs(y0) < 1e30 && fabs(y1) < 1e30)) return none;
    return make_float4((float)x0, (float)x1, (float)y0, (float)y1);
}

// ---------------- kernels ----------------

// view[0..15] = inverse view-projection (zero when singular), view[16] = 1 when
// it exists; tdir[t] = (unit ray through tile t's centre, same flag).
__global__ void k_e3_view(const StepParams* __restrict__ spp, float4* __restrict__ tdir, float* __restrict__ view) {
    const StepParams& sp = *spp;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float ivp[16];
    const bool have = invert4_e3(sp.cam.viewproj_matrix, ivp);
    if (!have)
#pragma unroll
        for (int k = 0; k < 16; k++) ivp[k] = 0.0f;
    if (t == 0) {
#pragma unroll
        for (int k = 0; k < 16; k++) view[k] = ivp[k];
        view[16] = have ? 1.0f : 0.0f;
    }
    if (t >= sp.num_tiles) return;
    const int x = t % sp.grid_x, y = t / sp.grid_x;
    float d[3] = {0.0f, 0.0f, 0.0f};
    if (have) {
        // tile_binner_cpu.cpp:82-85: the tile centre in pixels
        const float cx = ((float)x + 0.5f) * (float)sp.cfg.tile_w;
        const float cy = ((float)y + 0.5f) * (float)sp.cfg.tile_h;
        pixel_dir_e3(cx, cy, sp.cam.width, sp.cam.height, ivp, sp.cam.cam_pos, d);
    }
    tdir[t] = make_float4(d[0], d[1], d[2], have ? 1.0f : 0.0f);
}

// Key depth of a pair (tile_binner_cpu.cpp:79-88): the Gaussian's depth
// along the tile-centre ray when positive, else its view depth.
struct RayDepth {
    const float* ci;
    const float* mo;
    const float4* tdir;
    __device__ __forceinline__ unsigned operator()(unsigned dbits, unsigned gid, unsigned tile) const {
        const float4 d4 = tdir[tile];
        if (d4.w == 0.0f) return dbits;
        const float vd[3] = {d4.x, d4.y, d4.z};
        const float c[6] = {ci[6 * gid], ci[6 * gid + 1], ci[6 * gid + 2],
                            ci[6 * gid + 3], ci[6 * gid + 4], ci[6 * gid + 5]};
        const float m[3] = {mo[3 * gid], mo[3 * gid + 1], mo[3 * gid + 2]};
        const float ptd = depth_along_ray_e3(c, m, vd);
        return ptd > 0.0f ? __float_as_uint(ptd) : dbits;
    }
};

// Preprocess of the 3D-evaluation mode (preprocessor_cpu.cpp:64-187) fused
// with the pair emission.  RAW: the device model holds raw parameters
// (activated here, train_types.cpp:6-36).
template <bool RAW>
__global__ void __launch_bounds__(kBlock) k_preprocess_e3(const StepParams* __restrict__ spp, int N, ModelPtrs m,
                                                          const float* __restrict__ filt, ScreenPtrs s, E3Ptrs e,
                                                          PairPtrs pr, Control* ctrl) {
    __shared__ EmitShared<> sm;
    __shared__ int s_blk;
    const StepParams& sp = *spp;
    if (threadIdx.x == 0) s_blk = (int)atomicAdd(&ctrl->tickets[0], 1u);
    __syncthreads();
    const int blk = s_blk;
    const int i = blk * kBlock + threadIdx.x;
    int cnt = 0, rx = 0, ry = 0, rw = 1;
    unsigned dbits = 0;
    if (i < N) {
        const gs3d_camera& cam = sp.cam;
        const float p[3] = {m.pos[3 * i], m.pos[3 * i + 1], m.pos[3 * i + 2]};
        float sc[3], q[4], op;
        if (RAW) {
            const float rsc[3] = {m.sc[3 * i], m.sc[3 * i + 1], m.sc[3 * i + 2]};
            const float rq[4] = {m.rot[4 * i], m.rot[4 * i + 1], m.rot[4 * i + 2], m.rot[4 * i + 3]};
            activate_one(rsc, rq, m.op[i], sc, q, &op);
        } else {
#pragma unroll
            for (int k = 0; k < 3; k++) sc[k] = m.sc[3 * i + k];
#pragma unroll
            for (int k = 0; k < 4; k++) q[k] = m.rot[4 * i + k];
            op = m.op[i];
        }
        bool vis = false;
        float g2s[16], ci[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, mo[3] = {0.f, 0.f, 0.f};
        float pix_x = 0.f, pix_y = 0.f, depth = 0.f, opacity = 0.f, rgb[3] = {0.f, 0.f, 0.f}, thr_k = 0.f;
        int radius = 0, rmn[2] = {0, 0}, rmx[2] = {0, 0};
        float pv[3];
        xform4x3(p, cam.view_matrix, pv);
        do {
            if (pv[2] < 0.2f) break;                                          // :67-68
            opacity = op;
            const float focal = fmax_ref(sp.focal_x, sp.focal_y);
            const float f3 = filt ? filt[i] : 0.0f;
            float g2v[16];
            const float dil = gauss2screen_e3(p, sc, q, sp.cfg.scale_modifier, cam.cam_pos, cam.viewproj_matrix,
                                              cam.view_matrix, focal, 0.3f, f3, cam.width, cam.height, g2s, g2v);
            opacity *= dil;
            if (opacity < kAlphaMin) break;                                   // :82-84
            const float thr = log_ref(opacity / kAlphaMin);
            thr_k = thr;
            const float cutoff = fmin_ref(11.11f, 2.0f * thr);
            float R[3][3];
            quat2mat_e3(q, R);
            const float smod = sqrtf(sp.cfg.scale_modifier);
            float sdil[3], sd[3];
            {                                                                 // :95-101
                float mvw[3];
                xform4x3(p, cam.view_matrix, mvw);
                float mip = (mvw[2] / focal) * (mvw[2] / focal) * 0.3f;
                mip = fmax_ref(f3 * f3, mip);
#pragma unroll
                for (int j = 0; j < 3; j++) sdil[j] = sqrtf(sc[j] * sc[j] + mip);
            }
#pragma unroll
            for (int j = 0; j < 3; j++) sd[j] = sdil[j] * smod;
            cov3d_inv_e3(sdil, sp.cfg.scale_modifier, q, ci);                 // :106-107
#pragma unroll
            for (int k = 0; k < 3; k++) mo[k] = p[k] - cam.cam_pos[k];
            const float diff[3] = {cam.cam_pos[0] - p[0], cam.cam_pos[1] - p[1], cam.cam_pos[2] - p[2]};
            float cg[3];
#pragma unroll
            for (int j = 0; j < 3; j++) cg[j] = (R[j][0] * diff[0] + R[j][1] * diff[1] + R[j][2] * diff[2]) / sd[j];
            const float dist_sq = cg[0] * cg[0] + cg[1] * cg[1] + cg[2] * cg[2];
            if (dist_sq < cutoff) break;                                      // :128-129 camera inside
            const float mc = frustum_max_e3(0.0f, 0.0f, (float)(cam.width - 1), (float)(cam.height - 1), g2s);
            if (mc > thr) break;                                              // :136-137
            float ph[4];
            xform4x4(p, cam.viewproj_matrix, ph);
            const float pwi = 1.0f / (ph[3] + 1e-7f);
            pix_x = ((ph[0] * pwi + 1.0f) * (float)cam.width - 1.0f) * 0.5f;  // ndc2Pix
            pix_y = ((ph[1] * pwi + 1.0f) * (float)cam.height - 1.0f) * 0.5f;
            float ex[2];
            if (!aabb_screen_e3(g2s, cutoff, ex))
                aabb_view_e3(g2v, pv, sp.focal_x, sp.focal_y, (float)cam.width, (float)cam.height, cutoff, ex);
            radius = max(cvt_trunc_x86(ceilf(fmax_ref(ex[0], ex[1]))), 1);
            tile_rect_x86(pix_x, pix_y, radius, sp.grid_x, sp.grid_y, sp.cfg.tile_w, sp.cfg.tile_h, rmn, rmx);
            if ((rmx[0] - rmn[0]) * (rmx[1] - rmn[1]) == 0) break;
            float d[3];
            view_dir(p, cam.cam_pos, d);
            const float* sh = m.sh + (size_t)sp.max_coeffs * 3 * i;
            auto colour = [&](const float* shr) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    float v = fmax_ref(0.0f, sh_channel(sp.sh_deg_fwd, shr, c, d[0], d[1], d[2]) + 0.5f);
                    if (!sp.cfg.training) v = fmin_ref(1.0f, v);
                    rgb[c] = v;
                }
            };
            if (sp.max_coeffs == 16) {
                // degree-3 storage: the 192-byte row (16-byte aligned) as twelve 16-byte loads
                float4 shv[12];
#pragma unroll
                for (int k = 0; k < 12; k++) shv[k] = reinterpret_cast<const float4*>(sh)[k];
                colour(reinterpret_cast<const float*>(shv));
            } else {
                colour(sh);
            }
            depth = pv[2];
            vis = true;
        } while (false);
        if (vis) {
            cnt = (rmx[1] - rmn[1]) * (rmx[0] - rmn[0]);
            rx = rmn[0];
            ry = rmn[1];
            rw = rmx[0] - rmn[0];
            dbits = __float_as_uint(depth);
        } else {
            radius = 0;
            pix_x = pix_y = depth = opacity = 0.0f;
            rgb[0] = rgb[1] = rgb[2] = 0.0f;
#pragma unroll
            for (int k = 0; k < 16; k++) g2s[k] = 0.0f;
        }
        s.rec0[i] = make_float4(pix_x, pix_y, 0.f, 0.f);
        s.rec1[i] = make_float4(0.f, opacity, rgb[0], rgb[1]);
        s.cbt[i] = blue_thr(rgb[2], opacity);
        s.depth[i] = depth;
        s.radius[i] = radius;
        s.tiles[i] = cnt;
        float4* g4 = reinterpret_cast<float4*>(e.g2s) + 4 * (size_t)i;
#pragma unroll
        for (int r = 0; r < 4; r++) g4[r] = make_float4(g2s[4 * r], g2s[4 * r + 1], g2s[4 * r + 2], g2s[4 * r + 3]);
#pragma unroll
        for (int k = 0; k < 6; k++) e.ci[6 * (size_t)i + k] = ci[k];
#pragma unroll
        for (int k = 0; k < 3; k++) e.mo[3 * (size_t)i + k] = mo[k];
        float4* rc = e.rec + (size_t)kE3Rec * i;
        rc[0] = make_float4(g2s[0], g2s[1], g2s[2], g2s[3]);
        rc[1] = make_float4(g2s[4], g2s[5], g2s[6], g2s[7]);
        rc[2] = make_float4(g2s[12], g2s[13], g2s[14], g2s[15]);
        rc[3] = make_float4(ci[0], ci[1], ci[2], ci[3]);
        rc[4] = make_float4(ci[4], ci[5], mo[0], mo[1]);
        rc[5] = make_float4(mo[2], opacity, depth, rgb[0]);
        rc[6] = make_float4(rgb[1], rgb[2], thr_k, 0.f);
        rc[7] = vis ? e3_skip_box(g2s, thr_k) : make_float4(1e30f, -1e30f, 1e30f, -1e30f);
    }
    scan_and_emit(sm, blk, (unsigned)i, cnt, cnt, rx, ry, rw, dbits, sp.grid_x, pr, ctrl, sp.spin_limit, nullptr,
                  nullptr, 0, 0u, -1, RayDepth{e.ci, e.mo, e.tdir});
}

// The emission of the 3D-evaluation mode from host-provided arrays
// (tile_binner_cpu.cpp:59-99 with the per-tile depth keys).
__global__ void __launch_bounds__(kBlock) k_bin_arrays_e3(const StepParams* __restrict__ spp, int N, ScreenArrays a,
                                                          const float* __restrict__ ci, const float* __restrict__ mo,
                                                          const float4* __restrict__ tdir, PairPtrs pr,
                                                          Control* ctrl) {
    __shared__ EmitShared<> sm;
    __shared__ int s_blk;
    const StepParams& sp = *spp;
    if (threadIdx.x == 0) s_blk = (int)atomicAdd(&ctrl->tickets[0], 1u);
    __syncthreads();
    const int blk = s_blk;
    const int i = blk * kBlock + threadIdx.x;
    int cnt = 0, emit = 0, rx = 0, ry = 0, rw = 1;
    unsigned dbits = 0;
    if (i < N) {
        cnt = a.tiles[i];
        if (a.radii[i] > 0) {
            int rmn[2], rmx[2];
            tile_rect_x86(a.means2D[2 * i], a.means2D[2 * i + 1], a.radii[i], sp.grid_x, sp.grid_y, sp.cfg.tile_w,
                          sp.cfg.tile_h, rmn, rmx);
            rx = rmn[0];
            ry = rmn[1];
            rw = max(1, rmx[0] - rmn[0]);
            emit = min(cnt, (rmx[0] - rmn[0]) * (rmx[1] - rmn[1]));
            dbits = __float_as_uint(a.depths[i]);
        }
    }
    scan_and_emit(sm, blk, (unsigned)i, cnt, emit, rx, ry, rw, dbits, sp.grid_x, pr, ctrl, sp.spin_limit, nullptr,
                  nullptr, 0, 0u, -1, RayDepth{ci, mo, tdir});
}

// The per-pixel buffered blend (rasterizer_cpu.cpp:61-135, output :187-198).
// Shared memory (dynamic): the batch's records [kE3Rec][kE3Batch] float4 and
// the pixels' buffers as rings [kKBuf][256] of depth, alpha and index.
__global__ void __launch_bounds__(kE3Threads) k_raster_e3(const StepParams* __restrict__ spp,
                                                          const unsigned* __restrict__ ranges,
                                                          const unsigned* __restrict__ order,
                                                          const unsigned* __restrict__ vals, E3Ptrs e, PixelPtrs px,
                                                          Control* ctrl) {
    extern __shared__ float4 e3_smem[];
    float4* s_rec = e3_smem;                                                   // [kE3Rec][kE3Batch]
    float* s_kd = reinterpret_cast<float*>(e3_smem + kE3Rec * kE3Batch);      // [kKBuf][256]
    float* s_ka = s_kd + kKBuf * kE3Threads;
    unsigned* s_ki = reinterpret_cast<unsigned*>(s_ka + kKBuf * kE3Threads);
    const StepParams& sp = *spp;
    const int tid = threadIdx.x;
    const int tile = order ? (int)order[blockIdx.x] : (int)blockIdx.x;
    const int W = sp.cam.width, H = sp.cam.height;
    const int tx = tile % sp.grid_x, ty = tile / sp.grid_x;
    const int x = tx * kTile + (tid & 15), y = ty * kTile + (tid >> 4);
    const bool inside = x < W && y < H;
    const unsigned rs = ranges[2 * tile], re = ranges[2 * tile + 1];
    float ray[3] = {0.0f, 0.0f, 1.0f};
    if (inside) {
        float ivp[16];
#pragma unroll
        for (int k = 0; k < 16; k++) ivp[k] = e.view[k];
        pixel_dir_e3((float)x + 0.5f, (float)y + 0.5f, W, H, ivp, sp.cam.cam_pos, ray);
    }
    const float fpx = (float)x + 0.5f, fpy = (float)y + 0.5f;
    // this warp's 16x2 strip of pixel indices, for the per-Gaussian skip boxes
    const float wx0 = (float)(tx * kTile), wx1 = wx0 + (float)(kTile - 1);
    const float wy0 = (float)(ty * kTile + 2 * (tid >> 5)), wy1 = wy0 + 1.0f;
    float T = 1.0f, C0 = 0.0f, C1 = 0.0f, C2 = 0.0f;
    int cnt = 0, kc = 0, head = 0;
    bool done = !inside;
    for (unsigned b = rs; b < re; b += kE3Batch) {
        if (__syncthreads_count(done) == kE3Threads) break;
        for (int k = tid; k < kE3Rec * kE3Batch; k += kE3Threads) {
            const int r = k / kE3Rec, f = k - r * kE3Rec;
            const unsigned j = b + (unsigned)r;
            if (j < re) s_rec[f * kE3Batch + r] = e.rec[(size_t)kE3Rec * vals[j] + f];
        }
        __syncthreads();
        const int nb = (int)min((unsigned)kE3Batch, re - b);
        for (int k = 0; k < nb && !done; k++) {
            if (box_misses(s_rec[7 * kE3Batch + k], wx0, wx1, wy0, wy1)) continue;   // warp-uniform
            const float4 r0 = s_rec[k], r1 = s_rec[kE3Batch + k], r3 = s_rec[2 * kE3Batch + k];
            const float plx[4] = {r0.x - r3.x * fpx, r0.y - r3.y * fpx, r0.z - r3.z * fpx, r0.w - r3.w * fpx};
            const float ply[4] = {r1.x - r3.x * fpy, r1.y - r3.y * fpy, r1.z - r3.z * fpy, r1.w - r3.w * fpy};
            {
                // screening: the squared distance with one fast division is within a
                // few ulps of the exact one (all terms are non-negative); beyond
                // 2 thr + 1e-3 alpha is certainly below 1/255
                const float dx = plx[1] * ply[2] - plx[2] * ply[1];
                const float dy = plx[2] * ply[0] - plx[0] * ply[2];
                const float dz = plx[0] * ply[1] - plx[1] * ply[0];
                const float mx = plx[3] * ply[0] - plx[0] * ply[3];
                const float my = plx[3] * ply[1] - plx[1] * ply[3];
                const float mz = plx[3] * ply[2] - plx[2] * ply[3];
                const float dd = dx * dx + dy * dy + dz * dz;
                const float sm = mx * mx + my * my + mz * mz;
                const float lim = 2.0f * s_rec[6 * kE3Batch + k].z + 1e-3f;
                if (sm < 1e30f && dd > 1e-30f && dd < 1e30f && __fdividef(sm, dd) * (1.0f - 1e-5f) > lim) continue;
            }
            const float power = -0.5f * ray_dist_e3(plx, ply);
            if (power > 0.0f) continue;
            const float4 r5 = s_rec[5 * kE3Batch + k];
            const float o = r5.y;
            const float alpha = fmin_ref(0.99f, o * exp_ref(power));
            if (alpha < kAlphaMin) continue;
            const float4 r3c = s_rec[3 * kE3Batch + k], r4 = s_rec[4 * kE3Batch + k];
            const float ci[6] = {r3c.x, r3c.y, r3c.z, r3c.w, r4.x, r4.y};
            const float mo[3] = {r4.z, r4.w, r5.x};
            float pd = r5.z;
            const float ptd = depth_along_ray_e3(ci, mo, ray);
            if (ptd > 0.0f) pd = ptd;
            if (kc >= kKBuf) {   // blend the front entry (rasterizer_cpu.cpp:105-116)
                const int f = head * kE3Threads + tid;
                const float a = s_ka[f];
                const unsigned gid = s_ki[f];
                const float tT = T * (1.0f - a);
                if (tT < kTMin) {
                    done = true;
                    continue;
                }
                const float4 c5 = e.rec[(size_t)kE3Rec * gid + 5], c6 = e.rec[(size_t)kE3Rec * gid + 6];
                C0 += c5.w * a * T;
                C1 += c6.x * a * T;
                C2 += c6.y * a * T;
                T = tT;
                cnt++;
                head = (head + 1) & (kKBuf - 1);
                kc = kKBuf - 1;
            }
            // sorted insertion: entries deeper than pd move back by one
            int pos = kc;
            for (int q = kc - 1; q >= 0; q--) {
                if (s_kd[((head + q) & (kKBuf - 1)) * kE3Threads + tid] > pd) pos = q;
                else break;
            }
            for (int q = kc; q > pos; q--) {
                const int dst = ((head + q) & (kKBuf - 1)) * kE3Threads + tid;
                const int src = ((head + q - 1) & (kKBuf - 1)) * kE3Threads + tid;
                s_kd[dst] = s_kd[src];
                s_ka[dst] = s_ka[src];
                s_ki[dst] = s_ki[src];
            }
            const int at = ((head + pos) & (kKBuf - 1)) * kE3Threads + tid;
            s_kd[at] = pd;
            s_ka[at] = alpha;
            s_ki[at] = vals[b + (unsigned)k];
            kc++;
        }
    }
    // flush front to back (rasterizer_cpu.cpp:124-134)
    for (int q = 0; q < kc && !done; q++) {
        const int f = ((head + q) & (kKBuf - 1)) * kE3Threads + tid;
        const float a = s_ka[f];
        const float tT = T * (1.0f - a);
        if (tT < kTMin) break;
        const unsigned gid = s_ki[f];
        const float4 c5 = e.rec[(size_t)kE3Rec * gid + 5], c6 = e.rec[(size_t)kE3Rec * gid + 6];
        C0 += c5.w * a * T;
        C1 += c6.x * a * T;
        C2 += c6.y * a * T;
        T = tT;
        cnt++;
    }
    if (inside) {
        const size_t pix = (size_t)y * W + x;
        px.image[3 * pix] = C0 + T * sp.cfg.bg_color[0];
        px.image[3 * pix + 1] = C1 + T * sp.cfg.bg_color[1];
        px.image[3 * pix + 2] = C2 + T * sp.cfg.bg_color[2];
        if (px.T_final) px.T_final[pix] = T;
        if (px.n_contrib) px.n_contrib[pix] = cnt;
    }
}

constexpr size_t kE3RasterSmem = sizeof(float4) * kE3Rec * kE3Batch + (size_t)3 * 4 * kKBuf * kE3Threads;

}  // namespace
}  // namespace gs3d
