// raster_common.cuh -- helpers shared by the forward rasteriser (plain.cu,
// no FMA contraction) and the backward (raster_bwd.cu, FMA contraction on).
// Everything here either rounds the same under both builds (power_rn, whose
// operations carry explicit rounding) or is a conservative bound whose margin
// dwarfs any rounding difference (skip_threshold, skip_box).
#pragma once

#include <cuda_runtime.h>

namespace gs3d {

constexpr float kAlphaMin = 1.0f / 255.0f;   // rasterizer_cpu.cpp:150
constexpr float kTMin = 0.0001f;             // rasterizer_cpu.cpp:165

__device__ __forceinline__ float fmin_ref(float a, float b) { return (b < a) ? b : a; }  // std::min

// The Gaussian's exponent at pixel offset (dx, dy) = mean - pixel
// (rasterizer_cpu.cpp:146-148): -0.5 (a dx^2 + c dy^2) - b dx dy, evaluated
// left to right with every product and sum rounded separately, so that it is
// bit-identical in translation units with and without FMA contraction.
__device__ __forceinline__ float power_rn(float4 r0, float4 r1, float dx, float dy) {
    const float adx2 = __fmul_rn(__fmul_rn(r0.z, dx), dx);
    const float cdy2 = __fmul_rn(__fmul_rn(r1.x, dy), dy);
    const float bdxdy = __fmul_rn(__fmul_rn(r0.w, dx), dy);
    return __fsub_rn(__fmul_rn(-0.5f, __fadd_rn(adx2, cdy2)), bdxdy);
}

// A power below this bound gives alpha = o * exp(power) < 1/255 for certain
// (ln(1/(255 o)) less a margin far above the rounding of logf / expf), so the
// blend loops skip such Gaussians without evaluating exp; the skip they take
// is the one the exact alpha test would take.
__device__ __forceinline__ float skip_threshold(float o) { return logf(kAlphaMin / o) - 1e-3f; }

// Axis-aligned box (xmin, xmax, ymin, ymax) in pixels outside of which the
// Gaussian's power is below skip_threshold: the ellipse
// d^T C d <= -2 thr has half extents sqrt(-2 thr * Sigma_xx), sqrt(-2 thr *
// Sigma_yy) with Sigma = C^-1, widened by one pixel for rounding.  A warp
// whose pixels all lie outside it skips the Gaussian without evaluating it.
__device__ __forceinline__ float4 skip_box(float4 r0, float4 r1, float thr) {
    const float t2 = -2.0f * thr;
    const float det = r0.z * r1.x - r0.w * r0.w;   // conic a c - b^2
    if (!(t2 > 0.0f)) return make_float4(1e30f, -1e30f, 1e30f, -1e30f);     // never reaches alpha 1/255
    if (!(det > 0.0f)) return make_float4(-1e30f, 1e30f, -1e30f, 1e30f);    // not positive definite: no culling
    const float ex = sqrtf(t2 * r1.x / det) + 1.0f;
    const float ey = sqrtf(t2 * r0.z / det) + 1.0f;
    return make_float4(r0.x - ex, r0.x + ex, r0.y - ey, r0.y + ey);
}

__device__ __forceinline__ bool box_misses(float4 b, float x0, float x1, float y0, float y1) {
    return b.y < x0 || b.x > x1 || b.w < y0 || b.z > y1;
}

// ---- base-2 exponent of the reduced-storage form ----
// The reduced-storage rasterisers evaluate alpha = o * 2^q with
// q = power * log2(e) written as q = A + dy (B + H dy): A = -0.5 log2(e) a dx^2
// and B = -log2(e) b dx are shared by every pixel of a thread (its pixels share
// the column x, so dx), H = -0.5 log2(e) c by every pixel, leaving two FMAs per
// pixel.  Every operation carries explicit rounding, so the forward and the
// backward (different FMA-contraction settings) get the same q, the same
// 2^q and the same accept decisions.
constexpr float kLog2e = 1.4426950408889634f;

__device__ __forceinline__ float ex2_approx(float q) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(q));
    return r;
}

// skip_threshold in base-2 units: q below it gives alpha < 1/255 for certain
// (the natural bound's 1e-3 margin becomes 1.44e-3, far above rounding).
__device__ __forceinline__ float skip_threshold2(float o) { return __fmul_rn(skip_threshold(o), kLog2e); }

// Per (Gaussian, thread) coefficients of q: x = A, y = B, z = H.
__device__ __forceinline__ float3 q_coeffs(float4 r0, float4 r1, float dx) {
    const float A = __fmul_rn(__fmul_rn(r0.z, -0.5f * kLog2e), __fmul_rn(dx, dx));
    const float B = __fmul_rn(r0.w, __fmul_rn(-kLog2e, dx));
    const float H = __fmul_rn(r1.x, -0.5f * kLog2e);
    return make_float3(A, B, H);
}

__device__ __forceinline__ float q_at(float3 k, float dy) { return __fmaf_rn(dy, __fmaf_rn(k.z, dy, k.y), k.x); }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums eight values over the 32 lanes of a warp with 9 shuffles instead of 40:
// each butterfly stage sends half of the values it still holds to its partner,
// so the set of values a lane carries halves at every step.  On return lane l
// holds the warp total of value ((l>>4)&1)*4 + ((l>>3)&1)*2 + ((l>>2)&1)
// (*idx); lanes with the same bits 2..4 hold the same total.
__device__ __forceinline__ float warp_sum8(const float v[8], int* idx) {
    const unsigned lane = threadIdx.x & 31;
    const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
    float a[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float send = h16 ? v[i] : v[i + 4];
        const float keep = h16 ? v[i + 4] : v[i];
        a[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    float b[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const float send = h8 ? a[i] : a[i + 2];
        const float keep = h8 ? a[i + 2] : a[i];
        b[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    const float send = h4 ? b[0] : b[1];
    float c = (h4 ? b[1] : b[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
    c += __shfl_xor_sync(0xffffffffu, c, 2);
    c += __shfl_xor_sync(0xffffffffu, c, 1);
    *idx = (h16 ? 4 : 0) + (h8 ? 2 : 0) + (h4 ? 1 : 0);
    return c;
}

}  // namespace gs3d
