// plain.cu -- plain-FP32 form of the 3DGS hot path for sm_100a.
//
// Compiled with -fmad=false and IEEE division / square root so that every
// float operation rounds like the reference's x86 build with
// -ffp-contract=off (harmonyos_3dgs CMakeLists.txt:19); the operation order
// below follows the reference's CPU stages line by line, which is what makes
// depths, radii, tile counts, keys, sorted order and tile ranges bit-exact.
//
// Kernels:
//   k_preprocess    one thread per Gaussian: (activation) -> projection ->
//                   EWA covariance -> conic / radius / tile rect -> SH colour,
//                   then a block scan + decoupled look-back over tiles_touched
//                   and a block-cooperative emission of (tile|depth, index)
//                   pairs.  Replaces preprocess + prefix sum + binning.
//   k_bin_arrays    the same scan + emission from host-provided screen arrays.
//   k_raster_fwd    one CTA per 16x16 tile, one thread per pixel; pairs are
//                   gathered in batches of 256 into shared memory; CTA-wide
//                   early exit once every pixel saturated.  Optional fused L1.
//   (k_raster_bwd lives in raster_bwd.cu, compiled with FMA contraction.)
//   k_preprocess_bwd  the full per-Gaussian adjoint chain, fused with Adam.
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "common.cuh"
#include "kernels.cuh"
#include "raster_common.cuh"

namespace gs3d {
namespace {

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
__device__ __forceinline__ float sh_channel(int deg, const float* __restrict__ sh, int c, float x, float y,
                                            float z) {
    float v = SH_C0 * sh[c];
    if (deg > 0) {
        v += -SH_C1 * y * sh[3 + c] + SH_C1 * z * sh[6 + c] + -SH_C1 * x * sh[9 + c];
        if (deg > 1) {
            const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            v += SH_C20 * xy * sh[12 + c] + SH_C21 * yz * sh[15 + c] +
                 SH_C22 * (2.0f * zz - xx - yy) * sh[18 + c] + SH_C23 * xz * sh[21 + c] +
                 SH_C24 * (xx - yy) * sh[24 + c];
            if (deg > 2) {
                v += SH_C30 * y * (3.0f * xx - yy) * sh[27 + c] + SH_C31 * xy * z * sh[30 + c] +
                     SH_C32 * y * (4.0f * zz - xx - yy) * sh[33 + c] +
                     SH_C33 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy) * sh[36 + c] +
                     SH_C34 * x * (4.0f * zz - xx - yy) * sh[39 + c] + SH_C35 * z * (xx - yy) * sh[42 + c] +
                     SH_C36 * x * (xx - 3.0f * yy) * sh[45 + c];
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

// Alpha / transmittance decisions of the front-to-back blend
// (rasterizer_cpu.cpp:149-166).  A Gaussian that is clearly below the alpha
// threshold is skipped on the fast exp alone; every other evaluation --
// near the threshold, or accepted -- recomputes exp correctly
// rounded, so alpha, the transmittance chain T and the stop decision follow
// the reference's glibc-based values (they differ only where glibc's expf is
// itself 1 ulp off, ~0.006% of inputs).
// Returns 0 = skip, 1 = blend, 2 = stop (transmittance would saturate).
__device__ __forceinline__ int blend_decision(float power, float o, float T, float& alpha, float& e,
                                              float& test_T) {
    // screening on the fast exp: for power in [skip_threshold, 0] (|power| < 6)
    // __expf is within 6e-7 relative of exp, far inside the 4e-6 band kept here
    if (o * __expf(power) < kAlphaMin * (1.0f - 4e-6f)) return 0;
    e = exp_ref(power);
    alpha = fmin_ref(0.99f, o * e);
    if (alpha < kAlphaMin) return 0;
    test_T = T * (1.0f - alpha);
    if (test_T < kTMin) return 2;
    return 1;
}

// ---------------- per-Gaussian forward (preprocessor_cpu.cpp:186-265) ----------------

struct Proj {
    float px, py, depth, con[3], opac, rgb[3];
    int radius, rmn[2], rmx[2];
    float cov3[6], pv[3], phw, cov2[3], det;
};

// Returns false when the Gaussian is culled.
__device__ __forceinline__ bool project_one(const StepParams& sp, const float p[3], const float sc[3],
                                            const float q[4], float op, const float* __restrict__ sh,
                                            Proj& r) {
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
    cov3d(sc, sp.cfg.scale_modifier, q, c3);
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

// ---------------- block scan + look-back + pair emission ----------------

struct EmitShared {
    int warp[8];
    int excl[kBlock];
    int rect[kBlock];      // xmin | ymin << 16
    int width[kBlock];
    int limit[kBlock];     // pairs actually emitted (rect area, <= count)
    unsigned depth[kBlock];
    unsigned gid[kBlock];  // Gaussian index written as the pair's value
    unsigned long long base;
};

// Scans cnt over the CTA, finds the CTA's global offset by decoupled
// look-back and writes the CTA's pairs with consecutive threads writing
// consecutive pairs (fully coalesced, balanced however uneven the rects).
// Pair order: Gaussian-major, then row-major inside the rect
// (tile_binner_cpu.cpp:90-97).
// With pr.tiles32 set, writes tile-only keys and counts the first nd 8-bit
// digits of every tile into thist[nd][256] (shared memory).
__device__ __forceinline__ void scan_and_emit(EmitShared& sm, int blk, unsigned gid, int cnt, int emit, int rx, int ry,
                                              int rw, unsigned dbits, int grid_x, PairPtrs pr,
                                              Control* ctrl, unsigned spin_limit, Persist* persist,
                                              unsigned* thist = nullptr, int nd = 0) {
    const int tid = threadIdx.x;
    int total;
    const int incl = block_inclusive_scan(cnt, sm.warp, &total);
    sm.excl[tid] = incl - cnt;
    sm.rect[tid] = rx | (ry << 16);
    sm.width[tid] = rw;
    sm.limit[tid] = emit;
    sm.depth[tid] = dbits;
    sm.gid[tid] = gid;
    if (tid == 0) {
        const unsigned long long ex =
            lookback_exclusive(pr.scan_desc, blk, (unsigned long long)total, &ctrl->status, spin_limit);
        sm.base = ex;
        if (blk == (int)gridDim.x - 1) ctrl->total_pairs = ex + (unsigned long long)total;
        if (ex + (unsigned long long)total > pr.capacity) {
            atomicOr(&ctrl->status, kStatusOverflow);
            if (persist) atomicOr(&persist->sticky_overflow, 1u);
        }
    }
    __syncthreads();
    const unsigned long long base = sm.base;
    for (int k = tid; k < total; k += kBlock) {
        int lo = 0, hi = kBlock;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (sm.excl[mid] <= k) lo = mid;
            else hi = mid;
        }
        const int local = k - sm.excl[lo];
        const unsigned long long dst = base + (unsigned long long)k;
        if (local >= sm.limit[lo] || dst >= pr.capacity) continue;
        const int w = sm.width[lo];
        const int r = sm.rect[lo];
        const int x = (r & 0xffff) + local % w;
        const int y = (r >> 16) + local / w;
        const unsigned tile = (unsigned)(y * grid_x + x);
        if (pr.tiles32) {
            pr.tiles32[dst] = tile;
            for (int d = 0; d < nd; d++) atomicAdd(&thist[d * 256 + ((tile >> (8 * d)) & 255u)], 1u);
        } else {
            pr.keys[dst] = ((unsigned long long)tile << 32) | sm.depth[lo];
        }
        pr.vals[dst] = sm.gid[lo];
    }
}

// ---------------- kernels ----------------

template <bool TRAIN, bool CACHE, bool EMIT>
__global__ void __launch_bounds__(kBlock) k_preprocess(const StepParams* __restrict__ spp, int N, ModelPtrs m,
                                                       ScreenPtrs s, PairPtrs pr, DepthKeys dk, Control* ctrl) {
    __shared__ EmitShared sm;
    __shared__ int s_blk;
    const StepParams& sp = *spp;
    if (EMIT) {
        if (threadIdx.x == 0) s_blk = (int)atomicAdd(&ctrl->tickets[0], 1u);
        __syncthreads();
    }
    const int blk = EMIT ? s_blk : (int)blockIdx.x;
    const int i = blk * kBlock + threadIdx.x;
    int cnt = 0, rx = 0, ry = 0, rw = 1;
    unsigned dbits = 0;
    if (i < N) {
        const int mc3 = sp.max_coeffs * 3;
        const float p[3] = {m.pos[3 * i], m.pos[3 * i + 1], m.pos[3 * i + 2]};
        float sc[3], q[4], op;
        if (TRAIN) {
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
        Proj r;
        const bool vis = project_one(sp, p, sc, q, op, m.sh + (size_t)mc3 * i, r);
        if (vis) {
            cnt = (r.rmx[1] - r.rmn[1]) * (r.rmx[0] - r.rmn[0]);
            rx = r.rmn[0];
            ry = r.rmn[1];
            rw = r.rmx[0] - r.rmn[0];
            dbits = __float_as_uint(r.depth);
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
        if (CACHE) {
#pragma unroll
            for (int k = 0; k < 6; k++) s.cov3D[6 * i + k] = vis ? r.cov3[k] : 0.f;
#pragma unroll
            for (int k = 0; k < 3; k++) s.p_view[3 * i + k] = vis ? r.pv[k] : 0.f;
            s.p_hom_w[i] = vis ? r.phw : 0.f;
#pragma unroll
            for (int k = 0; k < 3; k++) s.cov2D[3 * i + k] = vis ? r.cov2[k] : 0.f;
            s.det[i] = vis ? r.det : 0.f;
        }
    }
    if (EMIT) {
        scan_and_emit(sm, blk, (unsigned)i, cnt, cnt, rx, ry, rw, dbits, sp.grid_x, pr, ctrl, sp.spin_limit,
                      sp.persist);
    } else if (i < N) {
        // depth-sort input: Gaussians without pairs sort last (no finite depth has these bits)
        dk.keys[i] = cnt > 0 ? (unsigned long long)dbits : 0xFFFFFFFFull;
        dk.vals[i] = (unsigned)i;
        if (i == 0) ctrl->gauss_keys = (unsigned long long)N;
    }
}

// Pair emission in depth order: thread r takes the Gaussian of depth rank r,
// recomputes its tile rectangle from the stored mean and radius (the same
// tile_rect the preprocess used) and emits its pairs row-major.  With the
// Gaussians stably sorted by depth bits, a stable sort of these pairs by tile
// alone gives the (tile, depth bits, Gaussian index) order of the full-key sort.
__global__ void __launch_bounds__(kBlock) k_emit_ranked(const StepParams* __restrict__ spp, int N,
                                                        const unsigned* __restrict__ rank_gid, ScreenPtrs s,
                                                        PairPtrs pr, Control* ctrl) {
    __shared__ EmitShared sm;
    __shared__ int s_blk;
    __shared__ unsigned s_thist[kMaxPasses - kDepthDigits][256];
    const StepParams& sp = *spp;
    const int nd = sp.sort_passes - kDepthDigits;   // 8-bit digits of the tile ids
    for (int e = threadIdx.x; e < nd * 256; e += kBlock) (&s_thist[0][0])[e] = 0;
    if (threadIdx.x == 0) s_blk = (int)atomicAdd(&ctrl->tickets[0], 1u);
    __syncthreads();
    const int blk = s_blk;
    const int r = blk * kBlock + threadIdx.x;
    int cnt = 0, rx = 0, ry = 0, rw = 1;
    unsigned g = 0, dbits = 0;
    if (r < N) {
        g = rank_gid[r];
        cnt = s.tiles[g];
        if (cnt > 0) {
            const float4 r0 = s.rec0[g];
            int rmn[2], rmx[2];
            tile_rect(r0.x, r0.y, s.radius[g], sp.grid_x, sp.grid_y, sp.cfg.tile_w, sp.cfg.tile_h, rmn, rmx);
            rx = rmn[0];
            ry = rmn[1];
            rw = rmx[0] - rmn[0];
            dbits = __float_as_uint(s.depth[g]);
        }
    }
    scan_and_emit(sm, blk, g, cnt, cnt, rx, ry, rw, dbits, sp.grid_x, pr, ctrl, sp.spin_limit, sp.persist,
                  &s_thist[0][0], nd);
    __syncthreads();
    for (int e = threadIdx.x; e < nd * 256; e += kBlock) {
        const unsigned v = (&s_thist[0][0])[e];
        if (v) atomicAdd(&ctrl->hist[kDepthDigits + (e >> 8)][e & 255], v);
    }
}

// TileBinner::bin over host-provided screen arrays (tile_binner_cpu.cpp:33-99):
// offsets from tiles_touched, pairs from the rect recomputed from (mean, radius).
__global__ void __launch_bounds__(kBlock) k_bin_arrays(const StepParams* __restrict__ spp, int N,
                                                       ScreenArrays a, PairPtrs pr, Control* ctrl) {
    __shared__ EmitShared sm;
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
            tile_rect(a.means2D[2 * i], a.means2D[2 * i + 1], a.radii[i], sp.grid_x, sp.grid_y,
                      sp.cfg.tile_w, sp.cfg.tile_h, rmn, rmx);
            rx = rmn[0];
            ry = rmn[1];
            rw = max(1, rmx[0] - rmn[0]);
            emit = min(cnt, (rmx[0] - rmn[0]) * (rmx[1] - rmn[1]));
            dbits = __float_as_uint(a.depths[i]);
        }
    }
    scan_and_emit(sm, blk, (unsigned)i, cnt, emit, rx, ry, rw, dbits, sp.grid_x, pr, ctrl, sp.spin_limit, nullptr);
}

// Unpacks the screen records into PreprocessOutput's layout.
__global__ void k_export_screen(int N, ScreenPtrs s, ScreenArrays a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 r0 = s.rec0[i], r1 = s.rec1[i];
    a.means2D[2 * i] = r0.x;
    a.means2D[2 * i + 1] = r0.y;
    a.conics[3 * i] = r0.z;
    a.conics[3 * i + 1] = r0.w;
    a.conics[3 * i + 2] = r1.x;
    a.opac2d[i] = r1.y;
    a.rgb[3 * i] = r1.z;
    a.rgb[3 * i + 1] = r1.w;
    a.rgb[3 * i + 2] = s.col_b[i];
    a.depths[i] = s.depth[i];
    a.radii[i] = s.radius[i];
    a.tiles[i] = s.tiles[i];
}

// Rasterizer forward (rasterizer_cpu.cpp:38-53, 137-198).  One CTA of 128
// threads per 16x16 tile, two pixels per thread: warp w owns the 16x4 strip
// of rows 4w..4w+3, a thread the pixels (x, 4w + lane/16) and
// (x, 4w + 2 + lane/16).  Batches of 256 records are gathered into shared
// memory; a warp skips a Gaussian whose skip box misses its strip; the CTA
// stops once every pixel saturated.  Optional fused L1 (sign byte per pixel,
// double-precision loss sum).
constexpr int kFwdThreads = 128;
constexpr int kFwdBatch = 256;

template <bool FUSED_LOSS>
__global__ void __launch_bounds__(kFwdThreads) k_raster_fwd(const StepParams* __restrict__ spp,
                                                            const unsigned* __restrict__ ranges,
                                                            const unsigned* __restrict__ order,
                                                            const unsigned* __restrict__ vals, ScreenPtrs s,
                                                            PixelPtrs px, Control* ctrl) {
    __shared__ float4 s_r0[kFwdBatch];
    __shared__ float4 s_r1[kFwdBatch];
    __shared__ float s_b[kFwdBatch];
    __shared__ float s_thr[kFwdBatch];
    __shared__ float4 s_box[kFwdBatch];
    __shared__ double s_loss[kFwdThreads / 32];
    const StepParams& sp = *spp;
    const int W = sp.cam.width, H = sp.cam.height;
    const int tile = order ? (int)order[blockIdx.x] : (int)blockIdx.x;
    const int tx = tile % sp.grid_x, ty = tile / sp.grid_x;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x = tx * kTile + (int)(lane & 15);
    const int ybase = ty * kTile + 4 * (int)warp + (int)(lane >> 4);
    const unsigned rs = ranges[2 * tile], re = ranges[2 * tile + 1];
    const float fx = (float)x;
    const float wx0 = (float)(tx * kTile), wx1 = wx0 + (float)(kTile - 1);
    const float wy0 = (float)(ty * kTile + 4 * (int)warp), wy1 = wy0 + 3.0f;
    float fy[2], T[2], C[2][3];
    int cnt[2];
    unsigned last[2];
    bool done[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        const int y = ybase + 2 * p;
        fy[p] = (float)y;
        T[p] = 1.0f;
        C[p][0] = C[p][1] = C[p][2] = 0.0f;
        cnt[p] = 0;
        last[p] = 0;
        done[p] = !(x < W && y < H);
    }
    for (unsigned b = rs; b < re; b += kFwdBatch) {
        if (__syncthreads_count(done[0] && done[1]) == kFwdThreads) break;
#pragma unroll
        for (int e = threadIdx.x; e < kFwdBatch; e += kFwdThreads) {
            const unsigned j = b + (unsigned)e;
            if (j < re) {
                const unsigned g = vals[j];
                const float4 r0 = s.rec0[g];
                const float4 r1 = s.rec1[g];
                const float thr = skip_threshold(r1.y);
                s_r0[e] = r0;
                s_r1[e] = r1;
                s_b[e] = s.col_b[g];
                s_thr[e] = thr;
                s_box[e] = skip_box(r0, r1, thr);
            }
        }
        __syncthreads();
        const int nb = (int)min((unsigned)kFwdBatch, re - b);
        for (int k = 0; k < nb; k++) {
            if (done[0] && done[1]) break;
            if (box_misses(s_box[k], wx0, wx1, wy0, wy1)) continue;
            const float4 a = s_r0[k];
            const float4 c = s_r1[k];
            const float thr = s_thr[k];
            const float dx = a.x - fx;
#pragma unroll
            for (int p = 0; p < 2; p++) {
                if (done[p]) continue;
                const float dy = a.y - fy[p];
                const float power = power_rn(a, c, dx, dy);
                if (power < thr || power > 0.0f) continue;
                float alpha, e, test_T;
                const int dec = blend_decision(power, c.y, T[p], alpha, e, test_T);
                if (dec == 0) continue;
                if (dec == 2) {
                    done[p] = true;
                    continue;
                }
                C[p][0] += c.z * alpha * T[p];
                C[p][1] += c.w * alpha * T[p];
                C[p][2] += s_b[k] * alpha * T[p];
                T[p] = test_T;
                cnt[p]++;
                last[p] = b + (unsigned)k + 1u;
            }
        }
    }
    double lsum = 0.0;
#pragma unroll
    for (int p = 0; p < 2; p++) {
        const int y = ybase + 2 * p;
        if (x < W && y < H) {
            const int pix = y * W + x;
            const float o0 = C[p][0] + T[p] * sp.cfg.bg_color[0];
            const float o1 = C[p][1] + T[p] * sp.cfg.bg_color[1];
            const float o2 = C[p][2] + T[p] * sp.cfg.bg_color[2];
            px.image[3 * pix] = o0;
            px.image[3 * pix + 1] = o1;
            px.image[3 * pix + 2] = o2;
            if (px.T_final) px.T_final[pix] = T[p];
            if (px.n_contrib) px.n_contrib[pix] = cnt[p];
            if (px.last_j) px.last_j[pix] = last[p];
            if (FUSED_LOSS) {
                // loss.cpp:8-14: diff = rendered - gt, sign gradient +-1/n
                const float d0 = o0 - sp.gt[3 * pix], d1 = o1 - sp.gt[3 * pix + 1], d2 = o2 - sp.gt[3 * pix + 2];
                const unsigned sg = (d0 > 0.f ? 1u : (d0 < 0.f ? 2u : 0u)) | (d1 > 0.f ? 4u : (d1 < 0.f ? 8u : 0u)) |
                                    (d2 > 0.f ? 16u : (d2 < 0.f ? 32u : 0u));
                px.dsign[pix] = (unsigned char)sg;
                lsum += (double)fabsf(d0) + (double)fabsf(d1) + (double)fabsf(d2);
            }
        }
    }
    if (FUSED_LOSS) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0) s_loss[warp] = lsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < kFwdThreads / 32; w++) t += s_loss[w];
            atomicAdd(&ctrl->loss_sum, t);
        }
    }
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

// The whole per-Gaussian adjoint chain of PreprocessorBackwardCPU::backward
// (preprocessor_backward_cpu.cpp:205-645) for a visible Gaussian, with the
// forward quantities (activation, p_view, cov3D, cov2D, det, means2D)
// recomputed bit-identically instead of read from a cache.
__device__ __forceinline__ void backward_one(const StepParams& sp, const BwdIn& in, BwdOut& o) {
    const gs3d_camera& cam = sp.cam;
    const float* shp = in.sh;
    const float* p = in.p;
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
    // ---- chain 3: sigmoid (:231-232) ----
    o.gop = in.dop * op * (1.0f - op);
    // ---- forward recompute (the ForwardCache of preprocessor_cpu.cpp:254-264) ----
    float c3[6];
    cov3d(sc, sp.cfg.scale_modifier, q, c3);
    Ewa e;
    ewa_setup(p, cam.view_matrix, sp.focal_x, sp.focal_y, cam.tan_fovx, cam.tan_fovy, e);
    float c2[3];
    cov2d(e, c3, c2);
    c2[0] += 0.3f;
    c2[2] += 0.3f;
    const float det = c2[0] * c2[2] - c2[1] * c2[1];
    if (det == 0.0f) return;
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
    const float dcov[6] = {dV[0][0], dV[0][1] + dV[1][0], dV[0][2] + dV[2][0],
                           dV[1][1], dV[1][2] + dV[2][1], dV[2][2]};
    // ---- chain 1c: cov3D -> M -> scale, R (:395-442) ----
    const float mod = sp.cfg.scale_modifier;
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
    const float* rq = in.rq;
    float qlen = sqrtf(rq[0] * rq[0] + rq[1] * rq[1] + rq[2] * rq[2] + rq[3] * rq[3]);
    if (qlen < 1e-12f) qlen = 1e-12f;
    const float il = 1.0f / qlen;
    const float dot = dq0 * rr + dq1 * xq + dq2 * yq + dq3 * zq;
    o.gq[0] = (dq0 - rr * dot) * il;
    o.gq[1] = (dq1 - xq * dot) * il;
    o.gq[2] = (dq2 - yq * dot) * il;
    o.gq[3] = (dq3 - zq * dot) * il;
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
}

// ---- fused preprocess backward + optimiser, staged by TMA into shared memory ----
//
// One CTA owns kBwdG consecutive Gaussians.  A single thread issues TMA bulk
// copies (cp.async.bulk) of the CTA's slices of every parameter array, of the
// screen-space gradients and of the radii onto mbarrier A, and of the Adam
// moments onto mbarrier B.  The CTA waits on A, runs the per-Gaussian adjoint
// (one thread per Gaussian) while the moments are still arriving, then waits on
// B and applies the optimiser element by element out of shared memory with
// coalesced vector stores.  The partial slice at the end of the model (sizes
// not multiples of 16 bytes) is staged with ordinary loads instead.
constexpr int kBwdG = 128;        // Gaussians (= threads) per CTA
constexpr int kMaxMc3 = 48;       // SH floats per Gaussian at degree 3
constexpr int kBasisPitch = 17;   // padded row of the per-Gaussian SH basis values

// The Adam moments come last: modes without the fused optimiser launch with
// offsetof(BwdShared, m_sh) bytes of shared memory and fit more CTAs per SM.
struct __align__(16) BwdShared {
    unsigned long long bar_a, bar_b;
    float sh[kBwdG * kMaxMc3];
    float pos[kBwdG * 3], sc[kBwdG * 3], rot[kBwdG * 4], op[kBwdG];
    float dm2[kBwdG * 2], dcon[kBwdG * 3], drgb[kBwdG * 3], dop[kBwdG];
    int radius[kBwdG];
    float basis[kBwdG * kBasisPitch], geff[kBwdG * 3];
    float gpos[kBwdG * 3], gsc[kBwdG * 3], grot[kBwdG * 4], gop[kBwdG];
    float m_sh[kBwdG * kMaxMc3], v_sh[kBwdG * kMaxMc3];
    float m_pos[kBwdG * 3], v_pos[kBwdG * 3], m_sc[kBwdG * 3], v_sc[kBwdG * 3];
    float m_rot[kBwdG * 4], v_rot[kBwdG * 4], m_op[kBwdG], v_op[kBwdG];
};

// Ordinary (tail-slice) staging of n floats.
__device__ __forceinline__ void copy_in(float* dst, const float* src, int n) {
    for (int e = threadIdx.x; e < n; e += kBwdG) dst[e] = src[e];
}

// Zeroes n floats of a gradient accumulator (coalesced, vectorised when aligned).
__device__ __forceinline__ void zero_out(float* dst, int n) {
    const int n4 = (((size_t)dst & 15) == 0) ? (n >> 2) : 0;
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (int q = threadIdx.x; q < n4; q += kBwdG) d4[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int e = 4 * n4 + threadIdx.x; e < n; e += kBwdG) dst[e] = 0.f;
}

// Optimiser over one parameter-group slice of n elements: parameters, moments
// and gradients read from shared memory, results stored to global memory.
template <class GradFn>
__device__ __forceinline__ void update_slice(const StepParams& sp, float* p_g, float* m_g, float* v_g,
                                             const float* p_s, const float* m_s, const float* v_s, int n,
                                             float lr, GradFn grad) {
    const bool vec = (((size_t)p_g | (size_t)m_g | (size_t)v_g) & 15) == 0;
    const int n4 = vec ? (n >> 2) : 0;
    for (int q = threadIdx.x; q < n4; q += kBwdG) {
        float pp[4], mm[4], vv[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = 4 * q + u;
            pp[u] = p_s[e];
            if (sp.use_adam) {
                mm[u] = m_s[e];
                vv[u] = v_s[e];
                pp[u] = adam_elem(pp[u], mm[u], vv[u], grad(e), lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            } else {
                pp[u] = pp[u] - lr * grad(e);
            }
        }
        reinterpret_cast<float4*>(p_g)[q] = make_float4(pp[0], pp[1], pp[2], pp[3]);
        if (sp.use_adam) {
            reinterpret_cast<float4*>(m_g)[q] = make_float4(mm[0], mm[1], mm[2], mm[3]);
            reinterpret_cast<float4*>(v_g)[q] = make_float4(vv[0], vv[1], vv[2], vv[3]);
        }
    }
    for (int e = 4 * n4 + threadIdx.x; e < n; e += kBwdG) {
        float pe = p_s[e];
        if (sp.use_adam) {
            float mm = m_s[e], vv = v_s[e];
            pe = adam_elem(pe, mm, vv, grad(e), lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            m_g[e] = mm;
            v_g[e] = vv;
        } else {
            pe = pe - lr * grad(e);
        }
        p_g[e] = pe;
    }
}

// Modes of k_preprocess_bwd.
constexpr int kBwdGrads = 0;   // stage API: write GradientOutput
constexpr int kBwdFused = 1;   // train step: apply the optimiser in the same kernel
constexpr int kBwdSplit = 2;   // train step: write GradientOutput for k_optimizer, zero the accumulators

// Preprocess backward (preprocessor_backward_cpu.cpp:8-645) for models whose
// SH arrays hold MC3 floats per Gaussian, fused with the optimiser update of all
// parameters or writing GradientOutput (see the modes above).
template <int MODE, int MC3>
__global__ void __launch_bounds__(kBwdG, MODE == 1 ? 2 : 4) k_preprocess_bwd(const StepParams* __restrict__ spp, int N,
                                                             ModelPtrs raw, AdamPtrs adam, ScreenPtrs s,
                                                             RGradPtrs rg, GradPtrs gout, Control* ctrl) {
    constexpr bool FUSED = MODE == kBwdFused;
    constexpr bool TRAIN = MODE != kBwdGrads;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    BwdShared& sm = *reinterpret_cast<BwdShared*>(smem_raw);
    const StepParams& sp = *spp;
    // an overflowed (or timed-out) step, or any step after one the host has not
    // acknowledged yet, updates nothing
    if (TRAIN && ((ctrl->status & (kStatusOverflow | kStatusTimeout)) || sp.persist->sticky_overflow)) return;
    if (FUSED && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&sp.persist->applied_steps, 1ull);
    const int tid = threadIdx.x;
    const size_t g0 = (size_t)blockIdx.x * kBwdG;
    const int ng = min(kBwdG, N - (int)g0);
    constexpr int mc3 = MC3;
    const bool want_mv = FUSED && sp.use_adam;
    const bool bulk = ng == kBwdG;   // every slice of a full CTA is a multiple of 512 bytes

    // ---- phase 0: staging ----
    if (bulk) {
        if (tid == 0) {
            mbar_init(&sm.bar_a, 1);
            mbar_init(&sm.bar_b, 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (tid == 0) {
            const unsigned B = 4u * kBwdG;   // bytes of one float per Gaussian
            mbar_arrive_expect_tx(&sm.bar_a, B * (11u + (unsigned)mc3 + 9u + 1u));
            tma_load_1d(sm.pos, raw.pos + 3 * g0, 3 * B, &sm.bar_a);
            tma_load_1d(sm.sc, raw.sc + 3 * g0, 3 * B, &sm.bar_a);
            tma_load_1d(sm.rot, raw.rot + 4 * g0, 4 * B, &sm.bar_a);
            tma_load_1d(sm.op, raw.op + g0, B, &sm.bar_a);
            tma_load_1d(sm.sh, raw.sh + (size_t)mc3 * g0, (unsigned)mc3 * B, &sm.bar_a);
            tma_load_1d(sm.dm2, rg.dm2 + 2 * g0, 2 * B, &sm.bar_a);
            tma_load_1d(sm.dcon, rg.dcon + 3 * g0, 3 * B, &sm.bar_a);
            tma_load_1d(sm.drgb, rg.drgb + 3 * g0, 3 * B, &sm.bar_a);
            tma_load_1d(sm.dop, rg.dop + g0, B, &sm.bar_a);
            tma_load_1d(sm.radius, s.radius + g0, B, &sm.bar_a);
            if (want_mv) {
                mbar_arrive_expect_tx(&sm.bar_b, 2u * B * (11u + (unsigned)mc3));
                tma_load_1d(sm.m_pos, adam.m_pos + 3 * g0, 3 * B, &sm.bar_b);
                tma_load_1d(sm.v_pos, adam.v_pos + 3 * g0, 3 * B, &sm.bar_b);
                tma_load_1d(sm.m_sc, adam.m_sc + 3 * g0, 3 * B, &sm.bar_b);
                tma_load_1d(sm.v_sc, adam.v_sc + 3 * g0, 3 * B, &sm.bar_b);
                tma_load_1d(sm.m_rot, adam.m_rot + 4 * g0, 4 * B, &sm.bar_b);
                tma_load_1d(sm.v_rot, adam.v_rot + 4 * g0, 4 * B, &sm.bar_b);
                tma_load_1d(sm.m_op, adam.m_op + g0, B, &sm.bar_b);
                tma_load_1d(sm.v_op, adam.v_op + g0, B, &sm.bar_b);
                tma_load_1d(sm.m_sh, adam.m_sh + (size_t)mc3 * g0, (unsigned)mc3 * B, &sm.bar_b);
                tma_load_1d(sm.v_sh, adam.v_sh + (size_t)mc3 * g0, (unsigned)mc3 * B, &sm.bar_b);
            }
        }
        mbar_wait(&sm.bar_a, 0, sp.spin_limit, &ctrl->status);
    } else {
        copy_in(sm.pos, raw.pos + 3 * g0, 3 * ng);
        copy_in(sm.sc, raw.sc + 3 * g0, 3 * ng);
        copy_in(sm.rot, raw.rot + 4 * g0, 4 * ng);
        copy_in(sm.op, raw.op + g0, ng);
        copy_in(sm.sh, raw.sh + (size_t)mc3 * g0, mc3 * ng);
        copy_in(sm.dm2, rg.dm2 + 2 * g0, 2 * ng);
        copy_in(sm.dcon, rg.dcon + 3 * g0, 3 * ng);
        copy_in(sm.drgb, rg.drgb + 3 * g0, 3 * ng);
        copy_in(sm.dop, rg.dop + g0, ng);
        for (int e = tid; e < ng; e += kBwdG) sm.radius[e] = s.radius[g0 + e];
        if (want_mv) {
            copy_in(sm.m_pos, adam.m_pos + 3 * g0, 3 * ng);
            copy_in(sm.v_pos, adam.v_pos + 3 * g0, 3 * ng);
            copy_in(sm.m_sc, adam.m_sc + 3 * g0, 3 * ng);
            copy_in(sm.v_sc, adam.v_sc + 3 * g0, 3 * ng);
            copy_in(sm.m_rot, adam.m_rot + 4 * g0, 4 * ng);
            copy_in(sm.v_rot, adam.v_rot + 4 * g0, 4 * ng);
            copy_in(sm.m_op, adam.m_op + g0, ng);
            copy_in(sm.v_op, adam.v_op + g0, ng);
            copy_in(sm.m_sh, adam.m_sh + (size_t)mc3 * g0, mc3 * ng);
            copy_in(sm.v_sh, adam.v_sh + (size_t)mc3 * g0, mc3 * ng);
        }
        __syncthreads();
    }
    if (TRAIN) {
        // the screen-gradient accumulators start at zero for the next step's raster backward
        zero_out(rg.dm2 + 2 * g0, 2 * ng);
        zero_out(rg.dcon + 3 * g0, 3 * ng);
        zero_out(rg.drgb + 3 * g0, 3 * ng);
        zero_out(rg.dop + g0, ng);
    }

    // ---- phase 1: per-Gaussian adjoint ----
    BwdOut o;
#pragma unroll
    for (int k = 0; k < 3; k++) { o.gp[k] = 0.f; o.gs[k] = 0.f; o.geff[k] = 0.f; }
#pragma unroll
    for (int k = 0; k < 4; k++) o.gq[k] = 0.f;
    o.gop = 0.f;
#pragma unroll
    for (int k = 0; k < 16; k++) o.basis[k] = 0.f;
    if (tid < ng && sm.radius[tid] > 0) {
        float shr[kMaxMc3];
        if (mc3 == kMaxMc3) {
            const float4* s4 = reinterpret_cast<const float4*>(sm.sh + tid * kMaxMc3);
#pragma unroll
            for (int q = 0; q < kMaxMc3 / 4; q++) {
                const float4 v = s4[q];
                shr[4 * q] = v.x; shr[4 * q + 1] = v.y; shr[4 * q + 2] = v.z; shr[4 * q + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kMaxMc3; k++) shr[k] = k < mc3 ? sm.sh[tid * mc3 + k] : 0.0f;
        }
        BwdIn in;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            in.p[k] = sm.pos[3 * tid + k];
            in.rsc[k] = sm.sc[3 * tid + k];
            in.dcn[k] = sm.dcon[3 * tid + k];
            in.drgb[k] = sm.drgb[3 * tid + k];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) in.rq[k] = sm.rot[4 * tid + k];
        in.rop = sm.op[tid];
        in.act = nullptr;
        float act[8];
        if (MODE == kBwdGrads && sp.raw_rot) {
            // activated device model (stage API): its values are the activation, raw_rot the raw quaternion
#pragma unroll
            for (int k = 0; k < 3; k++) act[k] = sm.sc[3 * tid + k];
#pragma unroll
            for (int k = 0; k < 4; k++) act[3 + k] = sm.rot[4 * tid + k];
            act[7] = sm.op[tid];
#pragma unroll
            for (int k = 0; k < 4; k++) in.rq[k] = sp.raw_rot[4 * (g0 + tid) + k];
            in.act = act;
        }
        in.dm[0] = sm.dm2[2 * tid];
        in.dm[1] = sm.dm2[2 * tid + 1];
        in.dop = sm.dop[tid];
        in.sh = shr;
        backward_one(sp, in, o);
    }
    if (tid < ng) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            sm.gpos[3 * tid + k] = o.gp[k];
            sm.gsc[3 * tid + k] = o.gs[k];
            sm.geff[3 * tid + k] = o.geff[k];
        }
#pragma unroll
        for (int k = 0; k < 4; k++) sm.grot[4 * tid + k] = o.gq[k];
        sm.gop[tid] = o.gop;
#pragma unroll
        for (int k = 0; k < 16; k++) sm.basis[tid * kBasisPitch + k] = o.basis[k];
    }
    __syncthreads();

    // ---- phase 2: element-wise optimiser (or GradientOutput) ----
    auto sh_grad = [&](int e) {
        const int gg = e / mc3, j = e - gg * mc3;
        const int k = j / 3, c = j - 3 * k;
        return sm.basis[gg * kBasisPitch + k] * sm.geff[3 * gg + c];
    };
    if (FUSED) {
        if (bulk && want_mv) mbar_wait(&sm.bar_b, 0, sp.spin_limit, &ctrl->status);
        update_slice(sp, raw.pos + 3 * g0, adam.m_pos + 3 * g0, adam.v_pos + 3 * g0, sm.pos, sm.m_pos, sm.v_pos,
                     3 * ng, sp.lr_pos, [&](int e) { return sm.gpos[e]; });
        update_slice(sp, raw.sc + 3 * g0, adam.m_sc + 3 * g0, adam.v_sc + 3 * g0, sm.sc, sm.m_sc, sm.v_sc, 3 * ng,
                     sp.lr_scale, [&](int e) { return sm.gsc[e]; });
        update_slice(sp, raw.rot + 4 * g0, adam.m_rot + 4 * g0, adam.v_rot + 4 * g0, sm.rot, sm.m_rot, sm.v_rot,
                     4 * ng, sp.lr_rot, [&](int e) { return sm.grot[e]; });
        update_slice(sp, raw.op + g0, adam.m_op + g0, adam.v_op + g0, sm.op, sm.m_op, sm.v_op, ng, sp.lr_opac,
                     [&](int e) { return sm.gop[e]; });
        update_slice(sp, raw.sh + (size_t)mc3 * g0, adam.m_sh + (size_t)mc3 * g0, adam.v_sh + (size_t)mc3 * g0,
                     sm.sh, sm.m_sh, sm.v_sh, mc3 * ng, sp.lr_sh, sh_grad);
    } else {
        for (int e = tid; e < 3 * ng; e += kBwdG) {
            gout.g_pos[3 * g0 + e] = sm.gpos[e];
            gout.g_sc[3 * g0 + e] = sm.gsc[e];
        }
        for (int e = tid; e < 4 * ng; e += kBwdG) gout.g_rot[4 * g0 + e] = sm.grot[e];
        for (int e = tid; e < ng; e += kBwdG) gout.g_op[g0 + e] = sm.gop[e];
        for (int e = tid; e < mc3 * ng; e += kBwdG) gout.g_sh[(size_t)mc3 * g0 + e] = sh_grad(e);
    }
}

// Optimiser over one parameter array: element-wise Adam / SGD (optimizer.cpp:9-43)
// with float4 loads and stores.
__device__ __forceinline__ void update_array(const StepParams& sp, float* __restrict__ p, float* __restrict__ m,
                                             float* __restrict__ v, const float* __restrict__ g, long long n,
                                             float lr) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long n4 = n >> 2;
    float4* p4 = reinterpret_cast<float4*>(p);
    float4* m4 = reinterpret_cast<float4*>(m);
    float4* v4 = reinterpret_cast<float4*>(v);
    const float4* g4 = reinterpret_cast<const float4*>(g);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
        float4 pp = p4[q];
        const float4 gg = g4[q];
        if (sp.use_adam) {
            float4 mm = m4[q], vv = v4[q];
            pp.x = adam_elem(pp.x, mm.x, vv.x, gg.x, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            pp.y = adam_elem(pp.y, mm.y, vv.y, gg.y, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            pp.z = adam_elem(pp.z, mm.z, vv.z, gg.z, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            pp.w = adam_elem(pp.w, mm.w, vv.w, gg.w, lr, sp.beta1, sp.beta2, sp.eps, sp.bc1, sp.bc2);
            m4[q] = mm;
            v4[q] = vv;
        } else {
            pp.x = pp.x - lr * gg.x;
            pp.y = pp.y - lr * gg.y;
            pp.z = pp.z - lr * gg.z;
            pp.w = pp.w - lr * gg.w;
        }
        p4[q] = pp;
    }
    for (long long i = 4 * n4 + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        apply_update(sp, &p[i], &m[i], &v[i], g[i], lr);
}

// Stand-alone optimiser step over the gradient arrays (optimizer.cpp:9-101).
// With ctrl (the split train step) an overflowed or unacknowledged step updates nothing.
__global__ void __launch_bounds__(256) k_optimizer(const StepParams* __restrict__ spp, long long n, int mc3,
                                                   ModelPtrs raw, AdamPtrs adam, GradPtrs g, const Control* ctrl) {
    const StepParams& sp = *spp;
    if (ctrl && ((ctrl->status & (kStatusOverflow | kStatusTimeout)) || sp.persist->sticky_overflow)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0 && sp.use_adam) atomicAdd(&sp.persist->applied_steps, 1ull);
    update_array(sp, raw.sh, adam.m_sh, adam.v_sh, g.g_sh, n * mc3, sp.lr_sh);
    update_array(sp, raw.pos, adam.m_pos, adam.v_pos, g.g_pos, 3 * n, sp.lr_pos);
    update_array(sp, raw.sc, adam.m_sc, adam.v_sc, g.g_sc, 3 * n, sp.lr_scale);
    update_array(sp, raw.rot, adam.m_rot, adam.v_rot, g.g_rot, 4 * n, sp.lr_rot);
    update_array(sp, raw.op, adam.m_op, adam.v_op, g.g_op, n, sp.lr_opac);
}

inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_preprocess_plain(cudaStream_t st, const StepParams* sp, int N, bool train, bool cache,
                                    ModelPtrs m, ScreenPtrs s, PairPtrs pr, Control* ctrl, DepthKeys dk) {
    if (N <= 0) return cudaSuccess;
    const int grid = blocks_for(N, kBlock);
    if (dk.keys) {
        if (train) {
            if (cache) k_preprocess<true, true, false><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
            else k_preprocess<true, false, false><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
        } else {
            if (cache) k_preprocess<false, true, false><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
            else k_preprocess<false, false, false><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
        }
    } else if (train) {
        if (cache) k_preprocess<true, true, true><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
        else k_preprocess<true, false, true><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
    } else {
        if (cache) k_preprocess<false, true, true><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
        else k_preprocess<false, false, true><<<grid, kBlock, 0, st>>>(sp, N, m, s, pr, dk, ctrl);
    }
    return cudaGetLastError();
}

cudaError_t launch_emit_ranked(cudaStream_t st, const StepParams* sp, int N, const unsigned* rank_gid,
                               ScreenPtrs s, PairPtrs pr, Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    k_emit_ranked<<<blocks_for(N, kBlock), kBlock, 0, st>>>(sp, N, rank_gid, s, pr, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_bin_arrays(cudaStream_t st, const StepParams* sp, int N, ScreenArrays a, PairPtrs pr,
                              Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    k_bin_arrays<<<blocks_for(N, kBlock), kBlock, 0, st>>>(sp, N, a, pr, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_export_screen(cudaStream_t st, int N, ScreenPtrs s, ScreenArrays a) {
    if (N <= 0) return cudaSuccess;
    k_export_screen<<<blocks_for(N, 256), 256, 0, st>>>(N, s, a);
    return cudaGetLastError();
}

cudaError_t launch_raster_fwd_plain(cudaStream_t st, const StepParams* sp, int num_tiles, bool fused_loss,
                                    const unsigned* ranges, const unsigned* order, const unsigned* vals,
                                    ScreenPtrs s, PixelPtrs px, Control* ctrl) {
    if (num_tiles <= 0) return cudaSuccess;
    if (fused_loss) k_raster_fwd<true><<<num_tiles, kFwdThreads, 0, st>>>(sp, ranges, order, vals, s, px, ctrl);
    else k_raster_fwd<false><<<num_tiles, kFwdThreads, 0, st>>>(sp, ranges, order, vals, s, px, ctrl);
    return cudaGetLastError();
}

namespace {
template <int MODE, int MC3>
cudaError_t launch_bwd_mc(cudaStream_t st, const StepParams* sp, int N, ModelPtrs raw, AdamPtrs adam, ScreenPtrs s,
                          RGradPtrs rg, GradPtrs gout, Control* ctrl) {
    const int smem = MODE == kBwdFused ? (int)sizeof(BwdShared) : (int)offsetof(BwdShared, m_sh);
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e =
            cudaFuncSetAttribute(k_preprocess_bwd<MODE, MC3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    k_preprocess_bwd<MODE, MC3><<<blocks_for(N, kBwdG), kBwdG, smem, st>>>(sp, N, raw, adam, s, rg, gout, ctrl);
    return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_bwd_mode(cudaStream_t st, const StepParams* sp, int N, int mc3, ModelPtrs raw, AdamPtrs adam,
                            ScreenPtrs s, RGradPtrs rg, GradPtrs gout, Control* ctrl) {
    switch (mc3) {
        case 3: return launch_bwd_mc<MODE, 3>(st, sp, N, raw, adam, s, rg, gout, ctrl);
        case 12: return launch_bwd_mc<MODE, 12>(st, sp, N, raw, adam, s, rg, gout, ctrl);
        case 27: return launch_bwd_mc<MODE, 27>(st, sp, N, raw, adam, s, rg, gout, ctrl);
        case 48: return launch_bwd_mc<MODE, 48>(st, sp, N, raw, adam, s, rg, gout, ctrl);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace

cudaError_t launch_preprocess_bwd_plain(cudaStream_t st, const StepParams* sp, int N, int mc3, int mode,
                                        ModelPtrs raw, AdamPtrs adam, ScreenPtrs s, RGradPtrs rg, GradPtrs gout,
                                        Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    switch (mode) {
        case kBwdGrads: return launch_bwd_mode<kBwdGrads>(st, sp, N, mc3, raw, adam, s, rg, gout, ctrl);
        case kBwdFused: return launch_bwd_mode<kBwdFused>(st, sp, N, mc3, raw, adam, s, rg, gout, ctrl);
        case kBwdSplit: return launch_bwd_mode<kBwdSplit>(st, sp, N, mc3, raw, adam, s, rg, gout, ctrl);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_optimizer_plain(cudaStream_t st, const StepParams* sp, int N, int mc3, ModelPtrs raw,
                                   AdamPtrs adam, GradPtrs g, const Control* ctrl) {
    if (N <= 0) return cudaSuccess;
    k_optimizer<<<8 * 148, 256, 0, st>>>(sp, (long long)N, mc3, raw, adam, g, ctrl);
    return cudaGetLastError();
}

}  // namespace gs3d
