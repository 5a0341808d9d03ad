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
#include <algorithm>
#include <type_traits>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"
#include "raster_common.cuh"
#include "ref_math.cuh"

namespace gs3d {
namespace {

// Blend decision of the reduced-storage forward on the base-2 exponent
// q = power * log2(e) (q_coeffs / q_at) once q has passed accept_threshold2:
// alpha = o * 2^q, no exact recheck.
struct FastBlend {
    static constexpr bool kBase2 = true;
    __device__ __forceinline__ static int decide(float q, float o, float T, float& alpha, float& e,
                                                 float& test_T) {
        e = ex2_approx(q);
        alpha = fmin_ref(0.99f, o * e);   // >= 1/255: q passed accept_threshold2
        test_T = fmaf(-alpha, T, T);   // T (1 - alpha)
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
    // BF16 is the top half of the FP32 pattern: add 16 random bits (r's upper half) below it, truncate
    unsigned u = __float_as_uint(x);
    if ((u & 0x7f800000u) == 0x7f800000u) return __float2bfloat16_rn(x);   // inf / nan
    u += r >> 16;
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

// One camera's screen record of a projected Gaussian (r from project_one) at
// entry o: the FP64 inverse of a near-degenerate 2D covariance, the reference's
// tile rectangle cut to the box of the alpha >= 1/255 ellipse, the record and
// the rectangle (whose area is the pair count).  The depth, radius and tile
// count arrays of the FP32 form have no reader in this form (its emission reads
// the rectangle, the sort the returned bits) and are not written.  Returns the
// depth bits for the depth sort, 0xFFFFFFFF for a Gaussian without pairs.
// olog, when given, holds (logf(255 o), accept_threshold2(o)) of the record's
// opacity o, computed once for all views of a Gaussian.
__device__ __forceinline__ unsigned chosen_record(const StepParams& sp, bool vis, Proj& r, long long o, ScreenPtrs s,
                                                  uint2* __restrict__ rects, const float* olog = nullptr) {
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
            const float tau = 2.0f * (olog ? olog[0] : logf(o255)) * 1.001f + 1e-3f;
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
        s.rec0[o] = make_float4(r.px, r.py, r.con[0], r.con[1]);
        s.rec1[o] = make_float4(r.con[2], r.opac, r.rgb[0], r.rgb[1]);
        s.cbt[o] = olog ? make_float2(r.rgb[2], olog[1]) : blue_thr(r.rgb[2], r.opac);
    } else {
        s.rec0[o] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.rec1[o] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.cbt[o] = blue_thr(0.f, 0.f);
    }
    rects[o] = rect;
    return cnt > 0 ? dbits : 0xFFFFFFFFu;
}

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
    const S* shrow = static_cast<const S*>(c.sh) + (size_t)mc3 * i;
    bool vis;
    if (mc3 == 48) {
        // degree-3 storage: the 96-byte row (16-byte aligned) as six 16-byte loads
        uint4 shv[6];
#pragma unroll
        for (int k = 0; k < 6; k++) shv[k] = reinterpret_cast<const uint4*>(shrow)[k];
        vis = project_one<S>(sp, p, sc, q, op, reinterpret_cast<const S*>(shv), r);
    } else {
        vis = project_one<S>(sp, p, sc, q, op, shrow, r);
    }
    dk.keys[i] = chosen_record(sp, vis, r, i, s, rects);
    dk.vals[i] = (unsigned)i;
}

// Several views: one thread per Gaussian loads, activates and forms the cov3D
// once and projects it into every view (entries view * N + i), writing the
// 32-bit (view, depth's upper 24 bits) keys of the depth sort.  The keys of
// view v sit at v * dk.seg_keys + i (a segment padded to whole sort tiles;
// threads N <= i < seg_keys write padding, whose key sorts last and whose value
// 0xFFFFFFFF marks no entry), so that the sort orders each view's segment apart
// on the depth digits (launch_radix_sort32_segmented).
template <typename S>
__global__ void __launch_bounds__(kBlock) k_chosen_preprocess_views(const StepParams* __restrict__ spp, int N,
                                                                    int n_views, ChosenPtrs c, ScreenPtrs s,
                                                                    DepthKeys dk, uint2* __restrict__ rects,
                                                                    Control* ctrl) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long seg = (long long)dk.seg_keys;
    if (i == 0) ctrl->gauss_keys = (unsigned long long)seg * n_views;
    if (i >= seg) return;
    if (i >= N) {
        for (int v = 0; v < n_views; v++) {
            dk.keys[v * seg + i] = 0xFFFFFFFFu;
            dk.vals[v * seg + i] = 0xFFFFFFFFu;
        }
        return;
    }
    const int mc3 = spp[0].max_coeffs * 3;
    const float p[3] = {c.pos[3 * i], c.pos[3 * i + 1], c.pos[3 * i + 2]};
    float rsc[3], rq[4], rop, sc[3], q[4], op, c3[6];
    load_attr<S>(c.attr, i, rsc, &rop, rq);
    activate_one(rsc, rq, rop, sc, q, &op);
    cov3d(sc, spp[0].cfg.scale_modifier, q, c3);
    const S* shrow = static_cast<const S*>(c.sh) + (size_t)mc3 * i;
    uint4 shv[6];
    if (mc3 == 48) {
#pragma unroll
        for (int k = 0; k < 6; k++) shv[k] = reinterpret_cast<const uint4*>(shrow)[k];
    }
    // without antialiasing the record's opacity is op in every view: its two logarithms once
    const float olog[2] = {logf(255.0f * op), accept_threshold2(op)};
    for (int v = 0; v < n_views; v++) {
        const StepParams& sp = spp[v];
        const long long o = (long long)v * N + i;
        Proj r;
        const bool vis = mc3 == 48 ? project_one<S>(sp, p, sc, q, op, reinterpret_cast<const S*>(shv), r, c3)
                                   : project_one<S>(sp, p, sc, q, op, shrow, r, c3);
        const float* const ol = sp.cfg.antialiasing ? nullptr : olog;
        dk.keys[v * seg + i] = ((unsigned)v << 24) | (chosen_record(sp, vis, r, o, s, rects, ol) >> 8);
        dk.vals[v * seg + i] = (unsigned)o;
    }
}

// ---- optimiser helpers ----

// Adam (optimizer.cpp:32-43 in FP32) or SGD on one element; the moments come
// in and go out as floats.
__device__ __forceinline__ float opt_elem(const StepParams& sp, float p, float& m, float& v, float g, float lr) {
    if (sp.use_adam) return adam_elem(p, m, v, g, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
    return p - lr * g;
}

// Random words of the roundings: the hash of (element, step) seeds a
// full-period LCG modulo 2^32 (odd increment, multiplier 1 mod 4) whose
// states follow; cvt_sr reads their upper bits.
__device__ __forceinline__ unsigned lcg_next(unsigned s) { return s * 0x2C1B3C6Du + 0x297A2D39u; }

// One element's three roundings.
__device__ __forceinline__ void sr_words(unsigned e, unsigned seed, unsigned& rp, unsigned& rm, unsigned& rv) {
    rp = mix32(e, seed);
    rm = lcg_next(rp);
    rv = lcg_next(rm);
}

// Eight consecutive 16-bit parameters (p) with their BF16 moments (m, v),
// updated in registers; e0 = the first element's global index.  One hash of
// (e0, step) seeds the LCG that gives all 24 roundings' random words.
template <typename S>
__device__ __forceinline__ void opt8(const StepParams& sp, uint4& p, uint4& m, uint4& v, const float g[8],
                                     const float lr[8], unsigned e0, unsigned salt) {
    S* pb = reinterpret_cast<S*>(&p);
    __nv_bfloat16* mb = reinterpret_cast<__nv_bfloat16*>(&m);
    __nv_bfloat16* vb = reinterpret_cast<__nv_bfloat16*>(&v);
    unsigned st = mix32(e0 ^ salt, sp.seed);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        float mm = __bfloat162float(mb[k]), vv = __bfloat162float(vb[k]);
        const float pn = opt_elem(sp, ldf(pb[k]), mm, vv, g[k], lr[k]);
        const unsigned rp = st = lcg_next(st), rm = st = lcg_next(st), rv = st = lcg_next(st);
        pb[k] = cvt_sr<S>(pn, rp);
        mb[k] = cvt_sr<__nv_bfloat16>(mm, rm);
        vb[k] = cvt_sr<__nv_bfloat16>(vv, rv);
    }
}

// The Adam constants of a step, read once per CTA.
struct AdamK {
    float b1, c1, b2, c2, bc1, bc2, eps;
    __device__ __forceinline__ explicit AdamK(const StepParams& sp)
        : b1(sp.beta1), c1(1.0f - sp.beta1), b2(sp.beta2), c2(1.0f - sp.beta2), bc1(sp.bc1), bc2(sp.bc2),
          eps(sp.eps) {}
};

// BF16 storage, Adam: opt8 on 32-bit words of two elements, with the same
// random words (p, m, v of each element in turn).  The stochastic rounding of
// a finite x is (bits(x) + (r >> 16)) >> 16, two of which one byte permute
// packs into a word.  A non-finite result would carry through the exponent
// there, so the caller redoes a chunk with one (false) element-wise (opt8).
__device__ __forceinline__ bool opt8_bf16_words(const AdamK& a, uint4& p, uint4& m, uint4& v, const float g[8],
                                                const float lr[8], unsigned st) {
    unsigned* pw = reinterpret_cast<unsigned*>(&p);
    unsigned* mw = reinterpret_cast<unsigned*>(&m);
    unsigned* vw = reinterpret_cast<unsigned*>(&v);
    bool finite = true;
#pragma unroll
    for (int w = 0; w < 4; w++) {
        unsigned pb[2], mb[2], vb[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int k = 2 * w + h;
            // element k is the low (h = 0) or high (h = 1) half of word w
            const float pk = __uint_as_float(h ? (pw[w] & 0xffff0000u) : (pw[w] << 16));
            float mk = __uint_as_float(h ? (mw[w] & 0xffff0000u) : (mw[w] << 16));
            float vk = __uint_as_float(h ? (vw[w] & 0xffff0000u) : (vw[w] << 16));
            mk = fmaf(a.b1, mk, a.c1 * g[k]);
            vk = fmaf(a.b2, vk, a.c2 * g[k] * g[k]);
            const float pn = pk - __fdividef(lr[k] * a.bc1 * mk, sqrtf(vk * a.bc2) + a.eps);
            const float kInf = __int_as_float(0x7f800000);
            finite &= (fabsf(pn) < kInf) & (fabsf(mk) < kInf) & (fabsf(vk) < kInf);
            const unsigned rp = st = lcg_next(st), rm = st = lcg_next(st), rv = st = lcg_next(st);
            pb[h] = __float_as_uint(pn) + (rp >> 16);
            mb[h] = __float_as_uint(mk) + (rm >> 16);
            vb[h] = __float_as_uint(vk) + (rv >> 16);
        }
        pw[w] = __byte_perm(pb[0], pb[1], 0x7632);
        mw[w] = __byte_perm(mb[0], mb[1], 0x7632);
        vw[w] = __byte_perm(vb[0], vb[1], 0x7632);
    }
    return finite;
}

// The Adam step of opt8 on words, for BF16 storage with Adam; false leaves the
// caller to redo the chunk element-wise from its stored inputs (another form,
// SGD, or a non-finite result).
template <typename S>
__device__ __forceinline__ bool opt8_words(const StepParams& sp, const AdamK& a, uint4& p, uint4& m, uint4& v,
                                           const float g[8], const float lr[8], unsigned e0, unsigned salt) {
    if constexpr (std::is_same<S, __nv_bfloat16>::value)
        return sp.use_adam && opt8_bf16_words(a, p, m, v, g, lr, mix32(e0 ^ salt, sp.seed));
    return false;
}

// ---- adjoint (staged, coalesced) ----

constexpr int kCB = 64;           // Gaussians (= threads) per CTA of the adjoint
// Row of one Gaussian's SH gradients in shared memory (several views): 52 floats, so that a thread
// updates its row with 16-byte accesses and the 8 threads of each 16-byte phase hit distinct banks
// (13 t mod 8 differs for t = 0..7).
constexpr int kShPitch = 52;

// One view: the SH gradient of coefficient k is basis[k / 3] * geff[k % 3], so the
// CTA keeps the 16 + 3 factors per Gaussian instead of the 48 products (18 KB per
// CTA of 64, 10 CTAs per SM).  Degree-3 storage (48 coefficients = six 8-wide
// optimiser chunks per Gaussian) keeps the bases chunk-major: chunk c of
// Gaussian t (coefficients 8c .. 8c + 7, bases b0 = 8c / 3 .. b0 + 3) reads
// the float4 bsh4[6 t + c], so that the 32 lanes of a warp, which take 32
// consecutive chunks, read 32 consecutive float4s.  Other storage keeps
// [basis][Gaussian].  The channel factors are [channel][Gaussian] with a
// pitch of 72: the lanes of a warp span at most six Gaussians, so the three
// rows of those six fall into distinct banks.  Several views sum the products: g_sh.
constexpr int kGeffPitch = 72;
__host__ __device__ constexpr int chunk_base0(int c) { return (8 * c) / 3; }   // first basis of chunk c

template <typename S, bool MULTI>
struct __align__(16) ChosenBwdShared {
    uint4 sh[kCB * 6];            // 16-bit SH, up to 48 per Gaussian (6 x 16 bytes)
    uint4 attr[kCB];              // 16-bit attributes, 8 per Gaussian
    float pos[3 * kCB];
    float dm2[2 * kCB], dcon[3 * kCB], drgb[3 * kCB], dop[kCB];
    float g_pos[3 * kCB], g_sc[3 * kCB], g_rot[4 * kCB], g_op[kCB];
    alignas(16) float g_sh[MULTI ? kShPitch * kCB : 4];
    alignas(16) float bsh[MULTI ? 4 : 24 * kCB];   // bases: 6 float4 chunks per Gaussian, or [basis][Gaussian]
    float geff[MULTI ? 1 : 3 * kGeffPitch];       // [channel][Gaussian]
    unsigned long long bar;       // completion of the bulk copies into the arrays above
    // SH gradient of coefficient kk of the CTA's Gaussian t
    __device__ __forceinline__ float gsh(int t, int kk, int mc3) const {
        if (MULTI) return g_sh[kShPitch * t + kk];
        const int b = kk / 3, ch = kk - 3 * b;
        float bv;
        if (mc3 == 48) {
            const int c = (3 * b) / 8;   // the chunk whose bases b0 .. b0 + 3 hold b
            bv = bsh[4 * (6 * t + c) + b - chunk_base0(c)];
        } else {
            bv = bsh[b * kCB + t];
        }
        return bv * geff[ch * kGeffPitch + t];
    }
};

// Thread 0: the bulk copies of slice g0's parameters (kCB Gaussians, all present) and, for one
// view, its screen gradients into sm, completing on sm.bar; the slice's optimiser moments travel
// to L2 meanwhile.
template <typename S, bool MULTI>
__device__ __forceinline__ void issue_slice_copies(ChosenBwdShared<S, MULTI>& sm, long long g0, int mc3, ChosenPtrs c,
                                                   RGradPtrs rg) {
    const S* shg = static_cast<const S*>(c.sh) + (size_t)mc3 * g0;
    const unsigned sh_bytes = (unsigned)(kCB * mc3 * (int)sizeof(S));
    const unsigned grad_bytes = MULTI ? 0u : (unsigned)kCB * (8u + 12u + 12u + 4u);
    mbar_arrive_expect_tx(&sm.bar, sh_bytes + (unsigned)kCB * (16u + 12u) + grad_bytes);
    tma_load_1d(sm.sh, shg, sh_bytes, &sm.bar);
    tma_load_1d(sm.attr, reinterpret_cast<const uint4*>(c.attr) + g0, 16u * kCB, &sm.bar);
    tma_load_1d(sm.pos, c.pos + 3 * g0, 12u * kCB, &sm.bar);
    if (!MULTI) {
        tma_load_1d(sm.dm2, rg.dm2 + 2 * g0, 8u * kCB, &sm.bar);
        tma_load_1d(sm.dcon, rg.dcon + 3 * g0, 12u * kCB, &sm.bar);
        tma_load_1d(sm.drgb, rg.drgb + 3 * g0, 12u * kCB, &sm.bar);
        tma_load_1d(sm.dop, rg.dop + g0, 4u * kCB, &sm.bar);
    }
    // the optimiser's moments of this slice travel to L2 while the adjoint computes
    const unsigned mv_sh = (unsigned)(kCB * mc3) * 2u;
    prefetch_l2(static_cast<const __nv_bfloat16*>(c.m_sh) + (size_t)mc3 * g0, mv_sh);
    prefetch_l2(static_cast<const __nv_bfloat16*>(c.v_sh) + (size_t)mc3 * g0, mv_sh);
    prefetch_l2(reinterpret_cast<const uint4*>(c.m_attr) + g0, 16u * kCB);
    prefetch_l2(reinterpret_cast<const uint4*>(c.v_attr) + g0, 16u * kCB);
    prefetch_l2(c.m_pos + 3 * g0, 12u * kCB);
    prefetch_l2(c.v_pos + 3 * g0, 12u * kCB);
}

// The same slice staged with plain loads (a partial last slice); the caller synchronises.
template <typename S, bool MULTI>
__device__ __forceinline__ void stage_slice_plain(ChosenBwdShared<S, MULTI>& sm, long long g0, int ng, int mc3,
                                                  ChosenPtrs c, RGradPtrs rg) {
    const int tid = threadIdx.x;
    const S* shg = static_cast<const S*>(c.sh) + (size_t)mc3 * g0;
    S* shs = reinterpret_cast<S*>(sm.sh);
    for (int e = tid; e < mc3 * ng; e += kCB) shs[e] = shg[e];
    for (int e = tid; e < ng; e += kCB) sm.attr[e] = reinterpret_cast<const uint4*>(c.attr)[g0 + e];
    for (int e = tid; e < 3 * ng; e += kCB) sm.pos[e] = c.pos[3 * g0 + e];
    if (!MULTI) {
        for (int e = tid; e < 2 * ng; e += kCB) sm.dm2[e] = rg.dm2[2 * g0 + e];
        for (int e = tid; e < 3 * ng; e += kCB) {
            sm.dcon[e] = rg.dcon[3 * g0 + e];
            sm.drgb[e] = rg.drgb[3 * g0 + e];
        }
        for (int e = tid; e < ng; e += kCB) sm.dop[e] = rg.dop[g0 + e];
    }
}

// One view: the adjoint of PreprocessorBackwardCPU::backward
// (preprocessor_backward_cpu.cpp:205-645) of each Gaussian of the staged slice
// into the shared-memory gradients; the slice's screen-gradient accumulators
// restart at zero for the next step.
template <typename S>
__device__ __forceinline__ void adjoint_slice(ChosenBwdShared<S, false>& sm, const StepParams& sp, long long g0,
                                              int ng, int mc3, RGradPtrs rg) {
    const int tid = threadIdx.x;
    const long long e0 = g0;
    // the screen-gradient accumulators restart at zero for the next step
    for (int e = tid; e < 2 * ng; e += kCB) rg.dm2[2 * e0 + e] = 0.f;
    for (int e = tid; e < 3 * ng; e += kCB) {
        rg.dcon[3 * e0 + e] = 0.f;
        rg.drgb[3 * e0 + e] = 0.f;
    }
    for (int e = tid; e < ng; e += kCB) rg.dop[e0 + e] = 0.f;
    if (tid >= ng) return;
    BwdIn in;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        in.dcn[k] = sm.dcon[3 * tid + k];
        in.drgb[k] = sm.drgb[3 * tid + k];
    }
    in.dm[0] = sm.dm2[2 * tid];
    in.dm[1] = sm.dm2[2 * tid + 1];
    in.dop = sm.dop[tid];
    BwdOut o;
#pragma unroll
    for (int k = 0; k < 3; k++) o.gp[k] = o.gs[k] = o.geff[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) o.gq[k] = 0.f;
    o.gop = 0.f;
#pragma unroll
    for (int k = 0; k < 16; k++) o.basis[k] = 0.f;
    // every gradient is linear in the screen gradients: a Gaussian without any adds none
    const bool any = in.dm[0] != 0.f || in.dm[1] != 0.f || in.dcn[0] != 0.f || in.dcn[1] != 0.f ||
                     in.dcn[2] != 0.f || in.drgb[0] != 0.f || in.drgb[1] != 0.f || in.drgb[2] != 0.f ||
                     in.dop != 0.f;
    if (any) {
#pragma unroll
        for (int k = 0; k < 3; k++) in.p[k] = sm.pos[3 * tid + k];
        in.act = nullptr;
        load_attr<S>(sm.attr, tid, in.rsc, &in.rop, in.rq);
        float shf[48];
        if (mc3 == 48) {
            // this Gaussian's 96 SH bytes as six 16-byte loads
            const uint4* row = sm.sh + 6 * tid;
#pragma unroll
            for (int qd = 0; qd < 6; qd++) {
                const uint4 vv = row[qd];
                const S* h = reinterpret_cast<const S*>(&vv);
#pragma unroll
                for (int k = 0; k < 8; k++) shf[8 * qd + k] = ldf(h[k]);
            }
        } else {
            const S* shs = reinterpret_cast<const S*>(sm.sh) + mc3 * tid;
#pragma unroll
            for (int k = 0; k < 48; k++) shf[k] = k < mc3 ? ldf(shs[k]) : 0.f;
        }
        in.sh = shf;
        backward_one(sp, in, o);
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        sm.g_pos[3 * tid + k] = o.gp[k];
        sm.g_sc[3 * tid + k] = o.gs[k];
        sm.geff[k * kGeffPitch + tid] = o.geff[k];
    }
#pragma unroll
    for (int k = 0; k < 4; k++) sm.g_rot[4 * tid + k] = o.gq[k];
    sm.g_op[tid] = o.gop;
    if (mc3 == 48) {
        float4* const b4 = reinterpret_cast<float4*>(sm.bsh) + 6 * tid;
#pragma unroll
        for (int c = 0; c < 6; c++) {
            constexpr int kLast = 15;
            const int b0 = chunk_base0(c);
            b4[c] = make_float4(o.basis[b0], o.basis[b0 + 1], o.basis[b0 + 2], o.basis[min(b0 + 3, kLast)]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) sm.bsh[k * kCB + tid] = o.basis[k];
    }
}

// Adam over the slice's contiguous parameters with 16-byte accesses and
// stochastic rounding (and, when asked, the FP32 gradients).
template <typename S, bool MULTI>
__device__ __forceinline__ void adam_slice(ChosenBwdShared<S, MULTI>& sm, const StepParams& sp, long long g0, int ng,
                                           int mc3, ChosenPtrs c, GradPtrs gout) {
    const int tid = threadIdx.x;
    if (gout.g_pos) {
        for (int e = tid; e < 3 * ng; e += kCB) {
            gout.g_pos[3 * g0 + e] = sm.g_pos[e];
            gout.g_sc[3 * g0 + e] = sm.g_sc[e];
        }
        for (int e = tid; e < 4 * ng; e += kCB) gout.g_rot[4 * g0 + e] = sm.g_rot[e];
        for (int e = tid; e < ng; e += kCB) gout.g_op[g0 + e] = sm.g_op[e];
        for (int e = tid; e < mc3 * ng; e += kCB) {
            const int t = e / mc3, k = e - t * mc3;
            gout.g_sh[(size_t)mc3 * g0 + e] = sm.gsh(t, k, mc3);
        }
    }
    const long long sh0 = (long long)mc3 * g0;
    // this thread's attribute moments (one Gaussian per thread: ng <= kCB) and position moments
    // (elements tid, tid + kCB, tid + 2 kCB of the slice) load during the SH updates
    uint4 am = make_uint4(0u, 0u, 0u, 0u), av = am;
    if (tid < ng) {
        am = reinterpret_cast<const uint4*>(c.m_attr)[g0 + tid];
        av = reinterpret_cast<const uint4*>(c.v_attr)[g0 + tid];
    }
    float pm[3] = {0.f, 0.f, 0.f}, pv[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int e = tid + j * kCB;
        if (e < 3 * ng) {
            pm[j] = c.m_pos[3 * g0 + e];
            pv[j] = c.v_pos[3 * g0 + e];
        }
    }
    S* shw = static_cast<S*>(c.sh);
    __nv_bfloat16* msh = static_cast<__nv_bfloat16*>(c.m_sh);
    __nv_bfloat16* vsh = static_cast<__nv_bfloat16*>(c.v_sh);
    const float lr_sh[8] = {sp.lr_sh, sp.lr_sh, sp.lr_sh, sp.lr_sh, sp.lr_sh, sp.lr_sh, sp.lr_sh, sp.lr_sh};
    if (ng == kCB) {
        // SH: 8 * mc3 chunks of 8 coefficients (16-byte aligned: the slice starts at 128 * mc3 * blockIdx
        // bytes); the parameters are already in shared memory
        const int nq = (kCB * mc3) / 8;
        uint4* m4 = reinterpret_cast<uint4*>(msh + sh0);
        uint4* v4 = reinterpret_cast<uint4*>(vsh + sh0);
        uint4* p4 = reinterpret_cast<uint4*>(shw + sh0);
        // each chunk's moments load one iteration ahead, so their latency overlaps the previous chunk
        uint4 mm_n = make_uint4(0u, 0u, 0u, 0u), vv_n = mm_n;
        if (tid < nq) {
            mm_n = m4[tid];
            vv_n = v4[tid];
        }
        const AdamK ak(sp);
        for (int q = tid; q < nq; q += kCB) {
            uint4 pp = sm.sh[q], mm = mm_n, vv = vv_n;
            if (q + kCB < nq) {
                mm_n = m4[q + kCB];
                vv_n = v4[q + kCB];
            }
            float gg[8];
            if (mc3 == 48) {
                // chunk c of Gaussian t: coefficients 8c .. 8c + 7
                const int t = q / 6, c = q - 6 * t;
                if (MULTI) {
                    const float4* gs = reinterpret_cast<const float4*>(&sm.g_sh[kShPitch * t + 8 * c]);
                    const float4 lo = gs[0], hi = gs[1];
                    gg[0] = lo.x, gg[1] = lo.y, gg[2] = lo.z, gg[3] = lo.w;
                    gg[4] = hi.x, gg[5] = hi.y, gg[6] = hi.z, gg[7] = hi.w;
                } else {
                    // coefficient 8c + k is basis b0 + (ch0 + k) / 3, channel (ch0 + k) % 3, with
                    // 8c = 3 b0 + ch0; bases b0 .. b0 + 3 are the chunk's float4
                    const float4 bb = reinterpret_cast<const float4*>(sm.bsh)[q];
                    const int ch0 = (2 * c) % 3;
                    const float* ge = sm.geff + t;
                    const float G0 = ge[ch0 * kGeffPitch];
                    const float G1 = ge[(ch0 == 2 ? 0 : ch0 + 1) * kGeffPitch];
                    const float G2 = ge[(ch0 == 0 ? 2 : ch0 - 1) * kGeffPitch];
                    // k % 3 == 1 moves to the next basis when ch0 = 2, k % 3 == 2 when ch0 >= 1
                    const bool up1 = ch0 == 2, up2 = ch0 != 0;
                    gg[0] = bb.x * G0;
                    gg[1] = (up1 ? bb.y : bb.x) * G1;
                    gg[2] = (up2 ? bb.y : bb.x) * G2;
                    gg[3] = bb.y * G0;
                    gg[4] = (up1 ? bb.z : bb.y) * G1;
                    gg[5] = (up2 ? bb.z : bb.y) * G2;
                    gg[6] = bb.z * G0;
                    gg[7] = (up1 ? bb.w : bb.z) * G1;
                }
            } else {
                // (Gaussian t, coefficient kk) of element 8q, then stepped by one
                int t = (8 * q) / mc3, kk = 8 * q - t * mc3;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    gg[k] = sm.gsh(t, kk, mc3);
                    if (++kk == mc3) {
                        kk = 0;
                        t++;
                    }
                }
            }
            if (!opt8_words<S>(sp, ak, pp, mm, vv, gg, lr_sh, (unsigned)(sh0 + 8 * q), 0x5bd1e995u)) {
                pp = sm.sh[q];
                mm = m4[q];
                vv = v4[q];
                opt8<S>(sp, pp, mm, vv, gg, lr_sh, (unsigned)(sh0 + 8 * q), 0x5bd1e995u);
            }
            p4[q] = pp;
            m4[q] = mm;
            v4[q] = vv;
        }
    } else {
        const S* shs = reinterpret_cast<const S*>(sm.sh);
        for (int e = tid; e < mc3 * ng; e += kCB) {
            const int t = e / mc3;
            float m = __bfloat162float(msh[sh0 + e]), v = __bfloat162float(vsh[sh0 + e]);
            const float pn = opt_elem(sp, ldf(shs[e]), m, v, sm.gsh(t, e - t * mc3, mc3), sp.lr_sh);
            unsigned rp, rm, rv;
            sr_words((unsigned)(sh0 + e) ^ 0x5bd1e995u, sp.seed, rp, rm, rv);
            shw[sh0 + e] = cvt_sr<S>(pn, rp);
            msh[sh0 + e] = cvt_sr<__nv_bfloat16>(m, rm);
            vsh[sh0 + e] = cvt_sr<__nv_bfloat16>(v, rv);
        }
    }
    // attributes: one 16-byte record per Gaussian
    const float lra[8] = {sp.lr_scale, sp.lr_scale, sp.lr_scale, sp.lr_opac, sp.lr_rot, sp.lr_rot, sp.lr_rot,
                          sp.lr_rot};
    if (tid < ng) {
        const int t = tid;
        const float gg[8] = {sm.g_sc[3 * t], sm.g_sc[3 * t + 1], sm.g_sc[3 * t + 2], sm.g_op[t],
                             sm.g_rot[4 * t], sm.g_rot[4 * t + 1], sm.g_rot[4 * t + 2], sm.g_rot[4 * t + 3]};
        uint4 pp = sm.attr[t];
        uint4 mm = am, vv = av;
        if (!opt8_words<S>(sp, AdamK(sp), pp, mm, vv, gg, lra, (unsigned)(8 * (g0 + t)), 0u)) {
            pp = sm.attr[t];
            mm = am;
            vv = av;
            opt8<S>(sp, pp, mm, vv, gg, lra, (unsigned)(8 * (g0 + t)), 0u);
        }
        reinterpret_cast<uint4*>(c.attr)[g0 + t] = pp;
        reinterpret_cast<uint4*>(c.m_attr)[g0 + t] = mm;
        reinterpret_cast<uint4*>(c.v_attr)[g0 + t] = vv;
    }
    // positions: FP32 parameters and moments
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int e = tid + j * kCB;
        if (e < 3 * ng) {
            const long long ge = 3 * g0 + e;
            float m = pm[j], v = pv[j];
            c.pos[ge] = opt_elem(sp, sm.pos[e], m, v, sm.g_pos[e], sp.lr_pos);
            c.m_pos[ge] = m;
            c.v_pos[ge] = v;
        }
    }
}

// One CTA per 64 consecutive Gaussians: bulk copies of their parameters and
// screen gradients into shared memory (the accumulators are zeroed for the
// next step), the per-Gaussian adjoint of PreprocessorBackwardCPU::backward
// (preprocessor_backward_cpu.cpp:205-645) from there into shared-memory
// gradients, then Adam over the CTA's contiguous parameter slice.
template <typename S, bool MULTI>
__global__ void __launch_bounds__(kCB, MULTI ? 8 : 10) k_chosen_backward(const StepParams* __restrict__ spp, int N, int mc3,
                                                         ChosenPtrs c, RGradPtrs rg, GradPtrs gout, Control* ctrl,
                                                         int n_views) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ChosenBwdShared<S, MULTI>& sm = *reinterpret_cast<ChosenBwdShared<S, MULTI>*>(smem_raw);
    const StepParams& sp = *spp;
    if ((ctrl->status & (kStatusOverflow | kStatusTimeout)) || sp.persist->sticky_overflow) return;
    const int tid = threadIdx.x;
    if (blockIdx.x == 0 && tid == 0 && sp.use_adam) atomicAdd(&sp.persist->applied_steps, 1ull);
    const long long g0 = (long long)blockIdx.x * kCB;
    const int ng = (int)min((long long)kCB, (long long)N - g0);
    // ---- phase 0: staging (several views: the screen gradients follow per view below) ----
    if (ng == kCB) {
        // a full CTA: every slice is a multiple of 16 bytes at a 16-byte aligned offset -> bulk copies
        if (tid == 0) {
            mbar_init(&sm.bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (tid == 0) issue_slice_copies(sm, g0, mc3, c, rg);
        mbar_wait(&sm.bar, 0, sp.spin_limit, &ctrl->status);
    } else {
        stage_slice_plain(sm, g0, ng, mc3, c, rg);
        __syncthreads();
    }
    // ---- phase 1: per-Gaussian adjoint (summed over the views) ----
    if constexpr (MULTI) {
        // Several views: the activation, cov3D, the cov3D -> scale / rotation chain and the sigmoid
        // do not depend on the camera and every gradient is linear in the screen gradients, so
        // one thread per Gaussian sums the views' camera-dependent parts (backward_view: SH,
        // conic -> cov3D, position) and applies the rest once.  Each view's screen gradients are
        // loaded one view ahead, straight into registers, and zeroed for the next step.
        if (tid < ng) {
            const long long gi = g0 + tid;
            float p[3], rsc[3], rq[4], rop, sc[3], q[4], op, c3[6];
#pragma unroll
            for (int k = 0; k < 3; k++) p[k] = sm.pos[3 * tid + k];
            load_attr<S>(sm.attr, tid, rsc, &rop, rq);
            activate_one(rsc, rq, rop, sc, q, &op);
            const float mod = sp.cfg.scale_modifier;
            cov3d(sc, mod, q, c3);
            float4* const shrow4 = reinterpret_cast<float4*>(&sm.g_sh[kShPitch * tid]);
#pragma unroll
            for (int q4 = 0; q4 < 12; q4++)
                if (4 * q4 < mc3) shrow4[q4] = make_float4(0.f, 0.f, 0.f, 0.f);
            float gp[3] = {0.f, 0.f, 0.f}, dcs[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, dops = 0.f;
            float nx[9];
            auto load_view = [&](long long e, float d[9]) {
                const float2 m = reinterpret_cast<const float2*>(rg.dm2)[e];
                d[0] = m.x;
                d[1] = m.y;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    d[2 + k] = rg.dcon[3 * e + k];
                    d[5 + k] = rg.drgb[3 * e + k];
                }
                d[8] = rg.dop[e];
            };
            load_view(gi, nx);
            for (int v = 0; v < n_views; v++) {
                const long long e = (long long)v * N + gi;   // this view's (view, Gaussian) entry
                float cur[9];
#pragma unroll
                for (int k = 0; k < 9; k++) cur[k] = nx[k];
                if (v + 1 < n_views) load_view(e + N, nx);
                // the screen-gradient accumulators restart at zero for the next step
                reinterpret_cast<float2*>(rg.dm2)[e] = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < 3; k++) rg.dcon[3 * e + k] = rg.drgb[3 * e + k] = 0.f;
                rg.dop[e] = 0.f;
                bool any = false;
#pragma unroll
                for (int k = 0; k < 9; k++) any |= cur[k] != 0.f;
                if (!any) continue;   // a view without screen gradients adds nothing
                BwdIn in;
                in.dm[0] = cur[0];
                in.dm[1] = cur[1];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    in.dcn[k] = cur[2 + k];
                    in.drgb[k] = cur[5 + k];
                }
                in.dop = cur[8];
                float shf[48];
                if (mc3 == 48) {
                    const uint4* row = sm.sh + 6 * tid;
#pragma unroll
                    for (int qd = 0; qd < 6; qd++) {
                        const uint4 vv = row[qd];
                        const S* h = reinterpret_cast<const S*>(&vv);
#pragma unroll
                        for (int k = 0; k < 8; k++) shf[8 * qd + k] = ldf(h[k]);
                    }
                } else {
                    const S* shs = reinterpret_cast<const S*>(sm.sh) + mc3 * tid;
#pragma unroll
                    for (int k = 0; k < 48; k++) shf[k] = k < mc3 ? ldf(shs[k]) : 0.f;
                }
                BwdOut o;
#pragma unroll
                for (int k = 0; k < 3; k++) o.gp[k] = o.geff[k] = 0.f;
#pragma unroll
                for (int k = 0; k < 16; k++) o.basis[k] = 0.f;
                float dcov[6];
                if (backward_view(spp[v], p, c3, shf, in, o, dcov)) {
#pragma unroll
                    for (int k = 0; k < 6; k++) dcs[k] += dcov[k];
                }
#pragma unroll
                for (int k = 0; k < 3; k++) gp[k] += o.gp[k];
                dops += cur[8];
                // SH gradient of coefficient k (basis k / 3, channel k % 3), four at a time
#pragma unroll
                for (int q4 = 0; q4 < 12; q4++) {
                    if (4 * q4 < mc3) {
                        float4 v4 = shrow4[q4];
                        v4.x += o.basis[(4 * q4) / 3] * o.geff[(4 * q4) % 3];
                        v4.y += o.basis[(4 * q4 + 1) / 3] * o.geff[(4 * q4 + 1) % 3];
                        v4.z += o.basis[(4 * q4 + 2) / 3] * o.geff[(4 * q4 + 2) % 3];
                        v4.w += o.basis[(4 * q4 + 3) / 3] * o.geff[(4 * q4 + 3) % 3];
                        shrow4[q4] = v4;
                    }
                }
            }
            BwdOut o;
            backward_cov3d(mod, sc, q, rq, dcs, o);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                sm.g_pos[3 * tid + k] = gp[k];
                sm.g_sc[3 * tid + k] = o.gs[k];
            }
#pragma unroll
            for (int k = 0; k < 4; k++) sm.g_rot[4 * tid + k] = o.gq[k];
            sm.g_op[tid] = dops * op * (1.0f - op);   // chain 3 (:231-232) on the summed opacity gradient
        }
    } else {
        adjoint_slice(sm, sp, g0, ng, mc3, rg);
    }
    __syncthreads();
    // ---- phase 2: optimiser over this CTA's slice (and the gradients, when kept) ----
    adam_slice(sm, sp, g0, ng, mc3, c, gout);
}

inline int grid_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_chosen_from_raw(cudaStream_t st, int N, int mc3, bool fp16, ModelPtrs raw, ChosenPtrs c) {
    if (N <= 0) return cudaSuccess;
    const int grid = std::min(grid_for((long long)N * mc3, 256), 8 * sm_count());
    if (fp16) k_chosen_from_raw<__half><<<grid, 256, 0, st>>>(N, mc3, raw, c);
    else k_chosen_from_raw<__nv_bfloat16><<<grid, 256, 0, st>>>(N, mc3, raw, c);
    return cudaGetLastError();
}

cudaError_t launch_chosen_to_raw(cudaStream_t st, int N, int mc3, bool fp16, ChosenPtrs c, ModelPtrs raw) {
    if (N <= 0) return cudaSuccess;
    const int grid = std::min(grid_for((long long)N * mc3, 256), 8 * sm_count());
    if (fp16) k_chosen_to_raw<__half><<<grid, 256, 0, st>>>(N, mc3, c, raw);
    else k_chosen_to_raw<__nv_bfloat16><<<grid, 256, 0, st>>>(N, mc3, c, raw);
    return cudaGetLastError();
}

cudaError_t launch_chosen_preprocess(cudaStream_t st, const StepParams* sp, int N, bool fp16, ChosenPtrs c,
                                     ScreenPtrs s, DepthKeys dk, uint2* rects, Control* ctrl, int n_views) {
    if (N <= 0 || n_views <= 0) return cudaSuccess;
    const int grid = grid_for(N, kBlock);
    if (n_views > 1 || dk.views24) {
        if (!dk.views24 || dk.seg_keys < (unsigned long long)N) return cudaErrorInvalidValue;
        const int grid_v = (int)((dk.seg_keys + kBlock - 1) / kBlock);
        if (fp16)
            k_chosen_preprocess_views<__half><<<grid_v, kBlock, 0, st>>>(sp, N, n_views, c, s, dk, rects, ctrl);
        else
            k_chosen_preprocess_views<__nv_bfloat16><<<grid_v, kBlock, 0, st>>>(sp, N, n_views, c, s, dk, rects,
                                                                                 ctrl);
    } else {
        if (fp16) k_chosen_preprocess<__half><<<grid, kBlock, 0, st>>>(sp, N, c, s, dk, rects, ctrl);
        else k_chosen_preprocess<__nv_bfloat16><<<grid, kBlock, 0, st>>>(sp, N, c, s, dk, rects, ctrl);
    }
    return cudaGetLastError();
}

cudaError_t launch_raster_fwd_fast_multi(cudaStream_t st, const StepParams* views, int n_views, unsigned n_tiles,
                                         const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                         ScreenPtrs s, PixelPtrs px, Control* ctrl, int ppt, int batch) {
    if (n_tiles == 0) return cudaSuccess;
    // persistent: as many CTAs as fit resident
    return with_ppt_batch(ppt, batch, [&](auto P, auto Bt) {
        constexpr int kP = decltype(P)::value, kB = decltype(Bt)::value;
        static int per_sm = 0;
        if (!per_sm) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_raster_fwd<kFusedL1, FastBlend, true, kP, kB>,
                                                              256 / kP, 0) != cudaSuccess ||
                per_sm < 1)
                per_sm = 1;
        }
        k_raster_fwd<kFusedL1, FastBlend, true, kP, kB><<<per_sm * sm_count(), 256 / kP, 0, st>>>(
            views, ranges, order, vals, s, px, ctrl, n_views, n_tiles);
        return cudaGetLastError();
    });
}

cudaError_t launch_raster_fwd_fast(cudaStream_t st, const StepParams* sp, int num_tiles, const unsigned* ranges,
                                   const unsigned* order, const unsigned* vals, ScreenPtrs s, PixelPtrs px,
                                   Control* ctrl, int ppt, int batch, bool loss_later) {
    if (num_tiles <= 0) return cudaSuccess;
    return with_ppt_batch(ppt, batch, [&](auto P, auto Bt) {
        constexpr int kP = decltype(P)::value, kB = decltype(Bt)::value;
        if (loss_later)
            k_raster_fwd<kLossLater, FastBlend, false, kP, kB><<<num_tiles, 256 / kP, 0, st>>>(sp, ranges, order, vals,
                                                                                              s, px, ctrl);
        else
            k_raster_fwd<kFusedL1, FastBlend, false, kP, kB><<<num_tiles, 256 / kP, 0, st>>>(sp, ranges, order, vals, s,
                                                                                            px, ctrl);
        return cudaGetLastError();
    });
}

cudaError_t launch_chosen_backward_adam(cudaStream_t st, const StepParams* sp, int N, int mc3, bool fp16,
                                        ChosenPtrs c, RGradPtrs rg, GradPtrs g, Control* ctrl, int n_views) {
    if (N <= 0) return cudaSuccess;
    if (mc3 > 48) return cudaErrorInvalidValue;
    const int grid = grid_for(N, kCB);
    // the same sizes for both 16-bit types
    const int smem1 = (int)sizeof(ChosenBwdShared<__half, false>), smemv = (int)sizeof(ChosenBwdShared<__half, true>);
    const int smem = n_views > 1 ? smemv : smem1;
    static std::atomic<unsigned long long> attr_done[4];
    cudaError_t e[4] = {set_smem_once(attr_done[0], k_chosen_backward<__half, false>, smem1),
                        set_smem_once(attr_done[1], k_chosen_backward<__nv_bfloat16, false>, smem1),
                        set_smem_once(attr_done[2], k_chosen_backward<__half, true>, smemv),
                        set_smem_once(attr_done[3], k_chosen_backward<__nv_bfloat16, true>, smemv)};
    for (cudaError_t x : e)
        if (x != cudaSuccess) return x;
    if (n_views > 1) {
        if (fp16) k_chosen_backward<__half, true><<<grid, kCB, smem, st>>>(sp, N, mc3, c, rg, g, ctrl, n_views);
        else k_chosen_backward<__nv_bfloat16, true><<<grid, kCB, smem, st>>>(sp, N, mc3, c, rg, g, ctrl, n_views);
    } else {
        if (fp16) k_chosen_backward<__half, false><<<grid, kCB, smem, st>>>(sp, N, mc3, c, rg, g, ctrl, 1);
        else k_chosen_backward<__nv_bfloat16, false><<<grid, kCB, smem, st>>>(sp, N, mc3, c, rg, g, ctrl, 1);
    }
    return cudaGetLastError();
}

}  // namespace gs3d
