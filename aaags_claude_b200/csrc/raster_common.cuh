// raster_common.cuh -- helpers shared by the forward rasteriser (plain.cu,
// no FMA contraction) and the backward (raster_bwd.cu, FMA contraction on).
// Everything here either rounds the same under both builds (power_rn, whose
// operations carry explicit rounding) or is a conservative bound whose margin
// dwarfs any rounding difference (skip_threshold, band_rows).
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
// (ln(1/(255 o)) less a margin far above the rounding of log / exp), so the
// blend loops skip such Gaussians without evaluating exp; the skip they take
// is the one the exact alpha test would take.  It is computed from the
// accept threshold thr2 = -log2(255 o) that the preprocess stores per
// Gaussian (blue_thr): ln(1/(255 o)) = ln(2) thr2.  The roundings of log2f and
// of this FMA move the bound by a few 1e-6, far inside the 1e-3 margin.
constexpr float kLn2 = 0.6931471805599453f;
__device__ __forceinline__ float skip_threshold(float thr2) { return fmaf(thr2, kLn2, -1e-3f); }

// Square root from the hardware reciprocal square root (rsqrtf, within 2 ulp),
// for the conservative bounds below; 0 for x <= 0.
__device__ __forceinline__ float sqrt_bound(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }

// Rows of a tile's column band where a Gaussian can reach power >= thr.
// The ellipse E = {d : a dx^2 + 2 b dx dy + c dy^2 <= t2}, t2 = -2 thr, with
// d = mean - pixel and conic (a, b, c) = (r0.z, r0.w, r1.x), is cut by the band
// of pixel columns [x0, x1]; returns the pixel rows [y0, y1] of that cut,
// y0 > y1 when E misses the band (or alpha can never reach 1/255).  Over
// dx in the band the top of E is (-b dx + sqrt(t2 c - det dx^2)) / c, a concave
// function whose maximum is E's topmost point dy = sqrt(t2 a / det) at
// dx = -b dy / a when that lies in the band and a band edge otherwise (the
// bottom likewise); edges outside E's x extent |dx| <= sqrt(t2 c / det) only
// add candidates, which keeps the range conservative.  The rows are widened by
// one pixel plus 1e-3 of the extent, above the FP32 rounding of these steps
// for det >= 1e-3 a c; more elongated conics are not culled.  A pixel outside
// the range has power < thr, so alpha < 1/255 (skip_threshold's margin), and
// the blend would skip it: culling it changes no result.
__device__ __forceinline__ float2 band_rows(float4 r0, float4 r1, float thr, float x0, float x1) {
    const float t2 = -2.0f * thr;
    const float a = r0.z, b = r0.w, c = r1.x;
    if (!(t2 > 0.0f)) return make_float2(1e30f, -1e30f);   // alpha never reaches 1/255
    const float det = fmaf(a, c, -b * b);
    if (!(a > 0.0f) || !(c > 0.0f) || !(det >= 1e-3f * a * c)) return make_float2(-1e30f, 1e30f);
    const float idet = __fdividef(1.0f, det);
    const float xext = sqrt_bound(t2 * c * idet), yext = sqrt_bound(t2 * a * idet);
    const float dlo = r0.x - x1, dhi = r0.x - x0;   // dx over the band
    const float mx = 1.0f + 1e-3f * xext;
    if (dlo > xext + mx || dhi < -xext - mx) return make_float2(1e30f, -1e30f);
    const float ic = __fdividef(1.0f, c);
    const float slo = sqrt_bound(t2 * c - det * dlo * dlo);
    const float shi = sqrt_bound(t2 * c - det * dhi * dhi);
    float up = fmaxf((slo - b * dlo) * ic, (shi - b * dhi) * ic);
    float dn = fminf((-slo - b * dlo) * ic, (-shi - b * dhi) * ic);
    const float xtop = __fdividef(-b * yext, a);    // dx of the topmost point; the bottom is at -xtop
    if (xtop >= dlo && xtop <= dhi) up = yext;
    if (-xtop >= dlo && -xtop <= dhi) dn = -yext;
    const float my = 1.0f + 1e-3f * yext;
    return make_float2(r0.y - up - my, r0.y - dn + my);   // rows y = mean.y - dy
}

// Bit w set when the warp strip of rows [ty0 + ROWS w, ty0 + ROWS w + ROWS - 1]
// meets the rows [yr.x, yr.y].
template <int NW, int ROWS>
__device__ __forceinline__ unsigned strip_mask(float2 yr, float ty0) {
    unsigned m = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const float s0 = ty0 + (float)(ROWS * w), s1 = s0 + (float)(ROWS - 1);
        if (yr.y >= s0 && yr.x <= s1) m |= 1u << w;
    }
    return m;
}

// The entries e < n of a batch whose mask has this warp's bit, in ascending
// order, written to list; returns their number.  Whole warp.
__device__ __forceinline__ int warp_list(const unsigned char* mask, int n, unsigned warp, unsigned char* list) {
    const unsigned lane = threadIdx.x & 31;
    int m = 0;
    for (int c0 = 0; c0 < n; c0 += 32) {
        const int e = c0 + (int)lane;
        const bool mine = e < n && ((mask[e] >> warp) & 1u);
        const unsigned bal = __ballot_sync(0xffffffffu, mine);
        if (mine) list[m + __popc(bal & ((1u << lane) - 1u))] = (unsigned char)e;
        m += __popc(bal);
    }
    __syncwarp();
    return m;
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

// The reduced form's accept test: o 2^q >= 1/255 <=> q >= log2(1 / (255 o)),
// decided on q alone (forward and backward stage the same value), so no
// separate alpha comparison follows.  Culling keeps skip_threshold's margin.
__device__ __forceinline__ float accept_threshold2(float o) { return -log2f(255.0f * o); }

// The screen record's (blue, accept threshold) pair, written by every preprocess.
__device__ __forceinline__ float2 blue_thr(float b, float o) { return make_float2(b, accept_threshold2(o)); }

// The staged record of the reduced form carries the conic pre-scaled for q:
// (x, y, -0.5 log2(e) a, -log2(e) b), (-0.5 log2(e) c, o, r, g).
__device__ __forceinline__ void q_scale(float4& r0, float4& r1) {
    r0.z = __fmul_rn(r0.z, -0.5f * kLog2e);
    r0.w = __fmul_rn(r0.w, -kLog2e);
    r1.x = __fmul_rn(r1.x, -0.5f * kLog2e);
}

// Per (Gaussian, thread) coefficients of q from a pre-scaled record: x = A, y = B, z = H.
__device__ __forceinline__ float3 q_coeffs(float4 r0s, float4 r1s, float dx) {
    return make_float3(__fmul_rn(r0s.z, __fmul_rn(dx, dx)), __fmul_rn(r0s.w, dx), r1s.x);
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
