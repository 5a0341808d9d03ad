// chosen.cu -- the reduced-storage ("chosen") form of the train step.
//
// Storage: positions FP32; raw scales, raw opacity, raw rotation and the SH
// coefficients 16-bit (S = __nv_bfloat16 or __half), 16 bytes of attributes
// plus 2*mc3 bytes of SH per Gaussian; Adam moments BF16 (positions: FP32).
// Arithmetic: FP32 with FMA contraction; blending, transmittance, the screen
// and parameter gradients and the Adam update all in FP32; FP64 only for the
// determinant / inverse of near-degenerate 2D covariances.  Parameters and
// moments are written back with stochastic rounding, so that Adam steps
// smaller than half a 16-bit ulp still move them in expectation.
//
// Against the plain form the preprocess also cuts each Gaussian's tile
// rectangle (the reference's 3-sigma square) to the box of the ellipse where
// alpha can reach 1/255, q = d^T conic d <= 2 ln(255 o): tiles outside it hold
// no pixel the blend would accept, so they get no pair.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"
#include "raster_common.cuh"
#include "ref_math.cuh"

namespace gs3d {
namespace {

// Blend decision of the reduced-storage forward: fast exp, no exact recheck.
struct FastBlend {
    __device__ __forceinline__ static int decide(float power, float o, float T, float& alpha, float& e,
                                                 float& test_T) {
        e = __expf(power);
        alpha = fmin_ref(0.99f, o * e);
        if (alpha < kAlphaMin) return 0;
        test_T = T * (1.0f - alpha);
        if (test_T < kTMin) return 2;
        return 1;
    }
};

}  // namespace
}  // namespace gs3d

#include "raster_fwd.cuh"

namespace gs3d {
namespace {

// ---- 16-bit storage ----

template <typename S>
__device__ __forceinline__ S cvt_rn(float x);
template <>
__device__ __forceinline__ __nv_bfloat16 cvt_rn<__nv_bfloat16>(float x) {
    return __float2bfloat16_rn(x);
}
template <>
__device__ __forceinline__ __half cvt_rn<__half>(float x) {
    return __float2half_rn(x);
}

// 32-bit mixing function (the MurmurHash3 finalizer) of an element index and
// the step seed: the random bits of stochastic rounding.
__device__ __forceinline__ unsigned mix32(unsigned a, unsigned b) {
    unsigned h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u);
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

// Stochastic rounding: x goes to one of its two 16-bit neighbours with
// probability proportional to its distance from the other.
template <typename S>
__device__ __forceinline__ S cvt_sr(float x, unsigned r);
template <>
__device__ __forceinline__ __nv_bfloat16 cvt_sr<__nv_bfloat16>(float x, unsigned r) {
    // BF16 is the top half of the FP32 pattern: add 16 random bits below it, truncate
    unsigned u = __float_as_uint(x);
    if ((u & 0x7f800000u) == 0x7f800000u) return __float2bfloat16_rn(x);   // inf / nan
    u += r & 0xffffu;
    return __ushort_as_bfloat16((unsigned short)(u >> 16));
}
template <>
__device__ __forceinline__ __half cvt_sr<__half>(float x, unsigned r) {
    const __half lo = __float2half_rd(x), hi = __float2half_ru(x);
    const float flo = __half2float(lo), fhi = __half2float(hi);
    if (!(fhi > flo)) return lo;
    const float p = (x - flo) / (fhi - flo);
    return ((float)(r >> 8) * (1.0f / 16777216.0f) < p) ? hi : lo;
}

template <typename S>
__global__ void k_chosen_from_raw(int N, int mc3, ModelPtrs raw, ChosenPtrs c) {
    const long long n_sh = (long long)N * mc3;
    const long long stride = (long long)gridDim.x * blockDim.x;
    S* attr = static_cast<S*>(c.attr);
    S* sh = static_cast<S*>(c.sh);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n_sh; e += stride) sh[e] = cvt_rn<S>(raw.sh[e]);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            c.pos[3 * i + k] = raw.pos[3 * i + k];
            attr[8 * i + k] = cvt_rn<S>(raw.sc[3 * i + k]);
        }
        attr[8 * i + 3] = cvt_rn<S>(raw.op[i]);
#pragma unroll
        for (int k = 0; k < 4; k++) attr[8 * i + 4 + k] = cvt_rn<S>(raw.rot[4 * i + k]);
    }
}

template <typename S>
__global__ void k_chosen_to_raw(int N, int mc3, ChosenPtrs c, ModelPtrs raw) {
    const long long n_sh = (long long)N * mc3;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const S* attr = static_cast<const S*>(c.attr);
    const S* sh = static_cast<const S*>(c.sh);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n_sh; e += stride) raw.sh[e] = ldf(sh[e]);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            raw.pos[3 * i + k] = c.pos[3 * i + k];
            raw.sc[3 * i + k] = ldf(attr[8 * i + k]);
        }
        raw.op[i] = ldf(attr[8 * i + 3]);
#pragma unroll
        for (int k = 0; k < 4; k++) raw.rot[4 * i + k] = ldf(attr[8 * i + 4 + k]);
    }
}

// The 16 attribute bytes of Gaussian i, unpacked.
template <typename S>
__device__ __forceinline__ void load_attr(const void* attr, long long i, float rsc[3], float* rop, float rq[4]) {
    const uint4 raw = reinterpret_cast<const uint4*>(attr)[i];
    const S* a = reinterpret_cast<const S*>(&raw);
#pragma unroll
    for (int k = 0; k < 3; k++) rsc[k] = ldf(a[k]);
    *rop = ldf(a[3]);
#pragma unroll
    for (int k = 0; k < 4; k++) rq[k] = ldf(a[4 + k]);
}

// ---- preprocess ----

template <typename S>
__global__ void __launch_bounds__(kBlock) k_chosen_preprocess(const StepParams* __restrict__ spp, int N, ChosenPtrs c,
                                                              ScreenPtrs s, DepthKeys dk, uint2* __restrict__ rects,
                                                              Control* ctrl) {
    const StepParams& sp = *spp;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) ctrl->gauss_keys = (unsigned long long)N;
    if (i >= N) return;
    const int mc3 = sp.max_coeffs * 3;
    const float p[3] = {c.pos[3 * i], c.pos[3 * i + 1], c.pos[3 * i + 2]};
    float rsc[3], rq[4], rop, sc[3], q[4], op;
    load_attr<S>(c.attr, i, rsc, &rop, rq);
    activate_one(rsc, rq, rop, sc, q, &op);
    Proj r;
    const bool vis = project_one<S>(sp, p, sc, q, op, static_cast<const S*>(c.sh) + (size_t)mc3 * i, r);
    int cnt = 0;
    uint2 rect = make_uint2(0u, 0u);
    unsigned dbits = 0xFFFFFFFFu;
    if (vis) {
        // near-degenerate 2D covariance: determinant and inverse in FP64
        if (r.det < 1e-4f * r.cov2[0] * r.cov2[2]) {
            const double a = r.cov2[0], b = r.cov2[1], cc = r.cov2[2];
            const double det = a * cc - b * b;
            if (det > 0.0) {
                r.con[0] = (float)(cc / det);
                r.con[1] = (float)(-b / det);
                r.con[2] = (float)(a / det);
            }
        }
        // box of the ellipse d^T conic d <= 2 ln(255 o) (with margin), cut from the reference's rectangle
        const float o255 = 255.0f * r.opac;
        if (o255 > 1.0f) {
            const float tau = 2.0f * logf(o255) * 1.001f + 1e-3f;
            const float ex = sqrtf(tau * r.cov2[0]), ey = sqrtf(tau * r.cov2[2]);
            const float tw = (float)sp.cfg.tile_w, th = (float)sp.cfg.tile_h;
            const int x0 = max(r.rmn[0], (int)floorf((r.px - ex) / tw));
            const int x1 = min(r.rmx[0], (int)floorf((r.px + ex) / tw) + 1);
            const int y0 = max(r.rmn[1], (int)floorf((r.py - ey) / th));
            const int y1 = min(r.rmx[1], (int)floorf((r.py + ey) / th) + 1);
            if (x1 > x0 && y1 > y0) {
                cnt = (x1 - x0) * (y1 - y0);
                rect = make_uint2((unsigned)x0 | ((unsigned)y0 << 16), (unsigned)x1 | ((unsigned)y1 << 16));
                dbits = __float_as_uint(r.depth);
            }
        }
        s.rec0[i] = make_float4(r.px, r.py, r.con[0], r.con[1]);
        s.rec1[i] = make_float4(r.con[2], r.opac, r.rgb[0], r.rgb[1]);
        s.col_b[i] = r.rgb[2];
        s.depth[i] = r.depth;
        s.radius[i] = r.radius;
    } else {
        s.rec0[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.rec1[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.col_b[i] = 0.f;
        s.depth[i] = 0.f;
        s.radius[i] = 0;
    }
    s.tiles[i] = cnt;
    rects[i] = rect;
    dk.keys[i] = cnt > 0 ? (unsigned long long)dbits : 0xFFFFFFFFull;
    dk.vals[i] = (unsigned)i;
}

// ---- fused adjoint + Adam ----

// Adam (optimizer.cpp:32-43 in FP32) or SGD on one element; the moments come
// in and go out as floats.
__device__ __forceinline__ float opt_elem(const StepParams& sp, float p, float& m, float& v, float g, float lr) {
    if (sp.use_adam) return adam_elem(p, m, v, g, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
    return p - lr * g;
}

constexpr int kCBwdThreads = 128;

template <typename S>
__global__ void __launch_bounds__(kCBwdThreads) k_chosen_backward_adam(const StepParams* __restrict__ spp, int N,
                                                                       int mc3, ChosenPtrs c, RGradPtrs rg,
                                                                       GradPtrs gout, Control* ctrl) {
    const StepParams& sp = *spp;
    // an overflowed (or timed-out) step, or any step after one the host has not
    // acknowledged yet, updates nothing
    if ((ctrl->status & (kStatusOverflow | kStatusTimeout)) || sp.persist->sticky_overflow) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && sp.use_adam) atomicAdd(&sp.persist->applied_steps, 1ull);
    if (i >= N) return;
    const unsigned seed = sp.seed;

    // screen gradients of this Gaussian; the accumulators restart at zero
    float dm[2] = {rg.dm2[2 * i], rg.dm2[2 * i + 1]};
    float dcn[3] = {rg.dcon[3 * i], rg.dcon[3 * i + 1], rg.dcon[3 * i + 2]};
    float drgb[3] = {rg.drgb[3 * i], rg.drgb[3 * i + 1], rg.drgb[3 * i + 2]};
    const float dop = rg.dop[i];
    rg.dm2[2 * i] = rg.dm2[2 * i + 1] = 0.f;
    rg.dcon[3 * i] = rg.dcon[3 * i + 1] = rg.dcon[3 * i + 2] = 0.f;
    rg.drgb[3 * i] = rg.drgb[3 * i + 1] = rg.drgb[3 * i + 2] = 0.f;
    rg.dop[i] = 0.f;

    BwdIn in;
    BwdOut o;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        in.p[k] = c.pos[3 * i + k];
        o.gp[k] = o.gs[k] = o.geff[k] = 0.f;
        in.dcn[k] = dcn[k];
        in.drgb[k] = drgb[k];
    }
#pragma unroll
    for (int k = 0; k < 4; k++) o.gq[k] = 0.f;
    o.gop = 0.f;
#pragma unroll
    for (int k = 0; k < 16; k++) o.basis[k] = 0.f;
    load_attr<S>(c.attr, i, in.rsc, &in.rop, in.rq);
    in.dm[0] = dm[0];
    in.dm[1] = dm[1];
    in.dop = dop;
    in.act = nullptr;
    const S* shp = static_cast<const S*>(c.sh) + (size_t)mc3 * i;
    float shf[48];
#pragma unroll
    for (int k = 0; k < 48; k++) shf[k] = k < mc3 ? ldf(shp[k]) : 0.f;
    in.sh = shf;
    // every gradient is linear in the screen gradients: a Gaussian without any has none
    const bool any = dm[0] != 0.f || dm[1] != 0.f || dcn[0] != 0.f || dcn[1] != 0.f || dcn[2] != 0.f ||
                     drgb[0] != 0.f || drgb[1] != 0.f || drgb[2] != 0.f || dop != 0.f;
    if (any) backward_one(sp, in, o);
    if (gout.g_pos) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            gout.g_pos[3 * i + k] = o.gp[k];
            gout.g_sc[3 * i + k] = o.gs[k];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) gout.g_rot[4 * i + k] = o.gq[k];
        gout.g_op[i] = o.gop;
        for (int k = 0; k < mc3; k++) gout.g_sh[(size_t)mc3 * i + k] = o.basis[k / 3] * o.geff[k % 3];
    }

    // ---- optimiser: positions (FP32 state) ----
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float m = c.m_pos[3 * i + k], v = c.v_pos[3 * i + k];
        c.pos[3 * i + k] = opt_elem(sp, in.p[k], m, v, o.gp[k], sp.lr_pos);
        c.m_pos[3 * i + k] = m;
        c.v_pos[3 * i + k] = v;
    }
    // ---- attributes: 8 x 16-bit, moments BF16 ----
    {
        const float pa[8] = {in.rsc[0], in.rsc[1], in.rsc[2], in.rop, in.rq[0], in.rq[1], in.rq[2], in.rq[3]};
        const float ga[8] = {o.gs[0], o.gs[1], o.gs[2], o.gop, o.gq[0], o.gq[1], o.gq[2], o.gq[3]};
        const float lra[8] = {sp.lr_scale, sp.lr_scale, sp.lr_scale, sp.lr_opac, sp.lr_rot, sp.lr_rot, sp.lr_rot,
                              sp.lr_rot};
        uint4 mraw = reinterpret_cast<const uint4*>(c.m_attr)[i];
        uint4 vraw = reinterpret_cast<const uint4*>(c.v_attr)[i];
        __nv_bfloat16* mb = reinterpret_cast<__nv_bfloat16*>(&mraw);
        __nv_bfloat16* vb = reinterpret_cast<__nv_bfloat16*>(&vraw);
        uint4 praw;
        S* pb = reinterpret_cast<S*>(&praw);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            float m = __bfloat162float(mb[k]), v = __bfloat162float(vb[k]);
            const float pn = opt_elem(sp, pa[k], m, v, ga[k], lra[k]);
            const unsigned e = (unsigned)(8 * i + k);
            pb[k] = cvt_sr<S>(pn, mix32(e, seed));
            mb[k] = cvt_sr<__nv_bfloat16>(m, mix32(e, seed ^ 0x68E31DA4u));
            vb[k] = cvt_sr<__nv_bfloat16>(v, mix32(e, seed ^ 0xB5297A4Du));
        }
        reinterpret_cast<uint4*>(c.attr)[i] = praw;
        reinterpret_cast<uint4*>(c.m_attr)[i] = mraw;
        reinterpret_cast<uint4*>(c.v_attr)[i] = vraw;
    }
    // ---- SH: gradient basis[k] * geff[channel], moments BF16 ----
    {
        S* shw = static_cast<S*>(c.sh) + (size_t)mc3 * i;
        __nv_bfloat16* msh = static_cast<__nv_bfloat16*>(c.m_sh) + (size_t)mc3 * i;
        __nv_bfloat16* vsh = static_cast<__nv_bfloat16*>(c.v_sh) + (size_t)mc3 * i;
#pragma unroll
        for (int k = 0; k < 48; k++) {
            if (k < mc3) {
                const float g = o.basis[k / 3] * o.geff[k % 3];
                float m = __bfloat162float(msh[k]), v = __bfloat162float(vsh[k]);
                const float pn = opt_elem(sp, shf[k], m, v, g, sp.lr_sh);
                const unsigned e = (unsigned)((size_t)mc3 * i + k) ^ 0x5bd1e995u;
                shw[k] = cvt_sr<S>(pn, mix32(e, seed));
                msh[k] = cvt_sr<__nv_bfloat16>(m, mix32(e, seed ^ 0x68E31DA4u));
                vsh[k] = cvt_sr<__nv_bfloat16>(v, mix32(e, seed ^ 0xB5297A4Du));
            }
        }
    }
}

inline int grid_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_chosen_from_raw(cudaStream_t st, int N, int mc3, bool fp16, ModelPtrs raw, ChosenPtrs c) {
    if (N <= 0) return cudaSuccess;
    const int grid = grid_for((long long)N * mc3, 256) < 8 * 148 ? grid_for((long long)N * mc3, 256) : 8 * 148;
    if (fp16) k_chosen_from_raw<__half><<<grid, 256, 0, st>>>(N, mc3, raw, c);
    else k_chosen_from_raw<__nv_bfloat16><<<grid, 256, 0, st>>>(N, mc3, raw, c);
    return cudaGetLastError();
}

cudaError_t launch_chosen_to_raw(cudaStream_t st, int N, int mc3, bool fp16, ChosenPtrs c, ModelPtrs raw) {
    if (N <= 0) return cudaSuccess;
    const int grid = grid_for((long long)N * mc3, 256) < 8 * 148 ? grid_for((long long)N * mc3, 256) : 8 * 148;
    if (fp16) k_chosen_to_raw<__half><<<grid, 256, 0, st>>>(N, mc3, c, raw);
    else k_chosen_to_raw<__nv_bfloat16><<<grid, 256, 0, st>>>(N, mc3, c, raw);
    return cudaGetLastError();
}

cudaError_t launch_chosen_preprocess(cudaStream_t st, const StepParams* sp, int N, bool fp16, ChosenPtrs c,
                                     ScreenPtrs s, DepthKeys dk, uint2* rects, Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    if (fp16) k_chosen_preprocess<__half><<<grid_for(N, kBlock), kBlock, 0, st>>>(sp, N, c, s, dk, rects, ctrl);
    else k_chosen_preprocess<__nv_bfloat16><<<grid_for(N, kBlock), kBlock, 0, st>>>(sp, N, c, s, dk, rects, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_raster_fwd_fast(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                                   const unsigned* order, const unsigned* vals, ScreenPtrs s, PixelPtrs px,
                                   Control* ctrl) {
    if (num_tiles <= 0) return cudaSuccess;
    k_raster_fwd<true, FastBlend><<<num_tiles, kFwdThreads, 0, st>>>(sp, ranges, order, vals, s, px, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_chosen_backward_adam(cudaStream_t st, const StepParams* sp, int N, int mc3, bool fp16,
                                        ChosenPtrs c, RGradPtrs rg, GradPtrs gout, Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    if (mc3 > 48) return cudaErrorInvalidValue;
    const int grid = grid_for(N, kCBwdThreads);
    if (fp16) k_chosen_backward_adam<__half><<<grid, kCBwdThreads, 0, st>>>(sp, N, mc3, c, rg, gout, ctrl);
    else k_chosen_backward_adam<__nv_bfloat16><<<grid, kCBwdThreads, 0, st>>>(sp, N, mc3, c, rg, gout, ctrl);
    return cudaGetLastError();
}

}  // namespace gs3d
