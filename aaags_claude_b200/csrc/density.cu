// density.cu -- adaptive density control on the device: the reference's
// DensityController (harmonyos_3dgs src/density_controller.cpp:9-204) and the
// OwnedRawParams append / compact it works through (include/train_types.h:108-140),
// for sm_100a.  Compiled with the plain form's flags (-fmad=false, IEEE
// division and square root): the float operations below round like the
// reference's x86 build, in its order.
//
// densify_and_prune as a sequence of data-parallel passes over the model:
//   k_dc_classify    clone / split flags per Gaussian (average gradient, the
//                    largest activated scale against 1 % of the extent);
//   scan             exclusive prefix sums of the flags (k_scan_blocks,
//                    k_scan_totals, k_scan_add): each Gaussian's rank among
//                    the clones and among the splits;
//   k_dc_expand_map  the source Gaussian of every entry of the post-split
//                    array: kept originals, then the clones, then two
//                    children per split (the reference's append order);
//   k_gather_rows    row gathers of the five parameter arrays;
//   k_dc_children    the children's positions and log-scales: Box-Muller
//                    samples from the controller's LCG advanced to the
//                    split's rank (12 steps per split, by jump-ahead);
//   k_dc_keep        prune flags (opacity, screen size at the post-split
//                    index, world size), scanned again and gathered into the
//                    new model.
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"
#include "kernels.cuh"

namespace gs3d {
namespace {

constexpr int kScanBlock = 1024;

// std::max(a, b) of the reference (a < b ? b : a)
__device__ __forceinline__ float max_ref(float a, float b) { return (a < b) ? b : a; }

// max_j exp(raw_scale_j) starting from 0 (density_controller.cpp:55-57)
__device__ __forceinline__ float max_scale(const float* s) {
    float m = 0.0f;
#pragma unroll
    for (int j = 0; j < 3; j++) m = max_ref(m, exp_ref(s[j]));
    return m;
}

// The controller's LCG (density_controller.cpp:10) and its n-fold composition.
constexpr unsigned long long kLcgA = 6364136223846793005ULL;
constexpr unsigned long long kLcgC = 1442695040888963407ULL;

__device__ __forceinline__ unsigned long long lcg_jump(unsigned long long s, unsigned long long n) {
    unsigned long long a = kLcgA, c = kLcgC;          // the map s -> a s + c
    unsigned long long ja = 1ULL, jc = 0ULL;          // accumulated map
    while (n) {
        if (n & 1ULL) {
            ja = a * ja;
            jc = a * jc + c;
        }
        c = a * c + c;
        a = a * a;
        n >>= 1;
    }
    return ja * s + jc;
}

// DensityController::randn (density_controller.cpp:9-16) with correctly
// rounded log and cos (the reference's glibc logf / cosf may differ by one ulp)
__device__ __forceinline__ float randn(unsigned long long& st) {
    st = st * kLcgA + kLcgC;
    float u1 = (float)((st >> 33) & 0xFFFFFFULL) / (float)0xFFFFFF;
    if (u1 < 1e-7f) u1 = 1e-7f;
    st = st * kLcgA + kLcgC;
    const float u2 = (float)((st >> 33) & 0xFFFFFFULL) / (float)0xFFFFFF;
    return sqrtf(-2.0f * (float)log((double)u1)) * (float)cos((double)(6.28318530718f * u2));
}

// accumulate_stats (density_controller.cpp:28-40); the raster-gradient entries
// it read are zeroed for the next step when `clear` is set.
__global__ void k_dc_accumulate(int N, float2* __restrict__ dm2, const int* __restrict__ radii, float* accum,
                                float* denom, int* max_radii, bool clear) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float2 d = dm2[i];
    accum[i] += sqrtf(d.x * d.x + d.y * d.y);
    denom[i] += 1.0f;
    if (radii && radii[i] > max_radii[i]) max_radii[i] = radii[i];
    if (clear) dm2[i] = make_float2(0.0f, 0.0f);
}

// clone = average gradient >= threshold and small; split = ... and large
// (density_controller.cpp:50-58, 77-84, 136-140)
__global__ void k_dc_classify(int N, const float* __restrict__ sc, const float* __restrict__ accum,
                              const float* __restrict__ denom, float threshold, float size_thr, int* clone,
                              int* split) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float avg = denom[i] > 0.0f ? accum[i] / denom[i] : 0.0f;
    const bool hot = !(avg < threshold);
    const bool small = !(max_scale(sc + 3 * (size_t)i) > size_thr);
    clone[i] = hot && small ? 1 : 0;
    split[i] = hot && !small ? 1 : 0;
}

// ---- exclusive scan of int flags (three passes) ----

__device__ __forceinline__ int block_excl_scan(int v, int* s_warp, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_warp[lane] = w;   // inclusive warp totals
    }
    __syncthreads();
    const int base = warp > 0 ? s_warp[warp - 1] : 0;
    *total = s_warp[(blockDim.x >> 5) - 1];
    return base + x - v;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_blocks(const int* __restrict__ in, int* __restrict__ out,
                                                            int* __restrict__ sums, int n) {
    __shared__ int s_warp[32];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    int total;
    const int e = block_excl_scan(v, s_warp, &total);
    if (i < n) out[i] = e;
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One block: exclusive scan of the block sums in place; sums[nb] = grand total.
__global__ void __launch_bounds__(kScanBlock) k_scan_totals(int* sums, int nb) {
    __shared__ int s_warp[32];
    __shared__ int s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nb; b0 += kScanBlock) {
        const int i = b0 + threadIdx.x;
        const int v = i < nb ? sums[i] : 0;
        int total;
        const int e = block_excl_scan(v, s_warp, &total);
        const int carry = s_carry;
        if (i < nb) sums[i] = carry + e;
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = s_carry;
}

__global__ void k_scan_add(int* out, const int* __restrict__ sums, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / kScanBlock];
}

// Source Gaussian of every post-split entry (-1 - rank for the second child
// marker is not needed: children are told apart by their position).
__global__ void k_dc_expand_map(int N, const int* __restrict__ clone, const int* __restrict__ split,
                                const int* __restrict__ crank, const int* __restrict__ srank, int n_c, int n_s,
                                int* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int kept = N - n_s;
    if (!split[i]) src[i - srank[i]] = i;
    if (clone[i]) src[kept + crank[i]] = i;
    if (split[i]) {
        const int c0 = kept + n_c + 2 * srank[i];
        src[c0] = i;
        src[c0 + 1] = i;
    }
}

// dst[r][c] = src[idx[r]][c] for rows r < rows of `width` floats
__global__ void k_gather_rows(float* __restrict__ dst, const float* __restrict__ srcp, const int* __restrict__ idx,
                              long long rows, int width) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= rows * width) return;
    const long long r = t / width;
    const int c = (int)(t - r * width);
    dst[t] = srcp[(long long)idx[r] * width + c];
}

// The two children of every split (density_controller.cpp:86-121): the
// original's scale and normalised rotation, log-scales reduced by
// log(1.6), positions offset by R (randn * scale), with the LCG advanced to
// 12 steps per earlier split.
__global__ void k_dc_children(int N, const float* __restrict__ pos, const float* __restrict__ sc,
                              const float* __restrict__ rot, const int* __restrict__ split,
                              const int* __restrict__ srank, int kept_plus_clones, unsigned long long rng0,
                              float log_factor, float* __restrict__ t_pos, float* __restrict__ t_sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || !split[i]) return;
    float scale[3], q[4];
#pragma unroll
    for (int j = 0; j < 3; j++) scale[j] = exp_ref(sc[3 * (size_t)i + j]);
#pragma unroll
    for (int j = 0; j < 4; j++) q[j] = rot[4 * (size_t)i + j];
    const float ql = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if (ql > 1e-8f)
#pragma unroll
        for (int j = 0; j < 4; j++) q[j] /= ql;
    const float r = q[0], x = q[1], y = q[2], z = q[3];
    const float R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y + r * z),     2 * (x * z - r * y),
                        2 * (x * y - r * z),     1 - 2 * (x * x + z * z), 2 * (y * z + r * x),
                        2 * (x * z + r * y),     2 * (y * z - r * x),     1 - 2 * (x * x + y * y)};
    float nsl[3];
#pragma unroll
    for (int j = 0; j < 3; j++) nsl[j] = sc[3 * (size_t)i + j] - log_factor;
    unsigned long long st = lcg_jump(rng0, 12ULL * (unsigned long long)srank[i]);
    const int c0 = kept_plus_clones + 2 * srank[i];
    for (int k = 0; k < 2; k++) {
        float smp[3];
        smp[0] = randn(st) * scale[0];
        smp[1] = randn(st) * scale[1];
        smp[2] = randn(st) * scale[2];
        float off[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int row = 0; row < 3; row++)
#pragma unroll
            for (int col = 0; col < 3; col++) off[row] += R[row * 3 + col] * smp[col];
        const size_t e = (size_t)(c0 + k);
#pragma unroll
        for (int j = 0; j < 3; j++) {
            t_pos[3 * e + j] = pos[3 * (size_t)i + j] + off[j];
            t_sc[3 * e + j] = nsl[j];
        }
    }
}

// Prune flags over the post-split array (density_controller.cpp:144-170):
// keep[e] = 0 when sigmoid(opacity) < min_opacity, when e < min(N, M) and
// the statistics entry e (indexed like the reference, by the post-split
// position) saw a radius above max_screen_size, or when the largest scale
// exceeds 10 % of the extent.
__global__ void k_dc_keep(int M, int N, const float* __restrict__ t_sc, const float* __restrict__ t_op,
                          const int* __restrict__ max_radii, float min_opacity, int max_screen_size, float world_thr,
                          int* __restrict__ keep) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M) return;
    bool prune = 1.0f / (1.0f + exp_ref(-t_op[e])) < min_opacity;
    if (e < min(N, M) && max_radii[e] > max_screen_size) prune = true;
    if (max_scale(t_sc + 3 * (size_t)e) > world_thr) prune = true;
    keep[e] = prune ? 0 : 1;
}

// inv[out[e]] = e for kept entries
__global__ void k_dc_invert(int M, const int* __restrict__ keep, const int* __restrict__ out, int* __restrict__ inv) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < M && keep[e]) inv[out[e]] = e;
}

__global__ void k_fill(float* p, long long n, float v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_dc_accumulate(cudaStream_t st, int N, float* dm2, const int* radii, DensityPtrs d, bool clear) {
    if (N <= 0) return cudaSuccess;
    k_dc_accumulate<<<blocks(N, 256), 256, 0, st>>>(N, reinterpret_cast<float2*>(dm2), radii, d.accum, d.denom,
                                                    d.max_radii, clear);
    return cudaGetLastError();
}

cudaError_t launch_scan_int(cudaStream_t st, const int* in, int* out, int* sums, int n) {
    if (n <= 0) return cudaSuccess;
    const int nb = blocks(n, kScanBlock);
    k_scan_blocks<<<nb, kScanBlock, 0, st>>>(in, out, sums, n);
    k_scan_totals<<<1, kScanBlock, 0, st>>>(sums, nb);
    k_scan_add<<<blocks(n, 256), 256, 0, st>>>(out, sums, n);
    return cudaGetLastError();
}

cudaError_t launch_dc_classify(cudaStream_t st, int N, const float* sc, DensityPtrs d, float threshold,
                               float size_thr) {
    if (N <= 0) return cudaSuccess;
    k_dc_classify<<<blocks(N, 256), 256, 0, st>>>(N, sc, d.accum, d.denom, threshold, size_thr, d.clone, d.split);
    return cudaGetLastError();
}

cudaError_t launch_dc_expand(cudaStream_t st, int N, int n_c, int n_s, ModelPtrs m, int mc3, DensityPtrs d,
                             ModelPtrs t, unsigned long long rng0, float log_factor) {
    if (N <= 0) return cudaSuccess;
    const long long M = (long long)N + n_c + n_s;
    k_dc_expand_map<<<blocks(N, 256), 256, 0, st>>>(N, d.clone, d.split, d.crank, d.srank, n_c, n_s, d.src);
    k_gather_rows<<<blocks(M * 3, 256), 256, 0, st>>>(t.pos, m.pos, d.src, M, 3);
    k_gather_rows<<<blocks(M * 3, 256), 256, 0, st>>>(t.sc, m.sc, d.src, M, 3);
    k_gather_rows<<<blocks(M * 4, 256), 256, 0, st>>>(t.rot, m.rot, d.src, M, 4);
    k_gather_rows<<<blocks(M * mc3, 256), 256, 0, st>>>(t.sh, m.sh, d.src, M, mc3);
    k_gather_rows<<<blocks(M, 256), 256, 0, st>>>(t.op, m.op, d.src, M, 1);
    if (n_s > 0)
        k_dc_children<<<blocks(N, 128), 128, 0, st>>>(N, m.pos, m.sc, m.rot, d.split, d.srank, N - n_s + n_c, rng0,
                                                      log_factor, t.pos, t.sc);
    return cudaGetLastError();
}

cudaError_t launch_dc_keep(cudaStream_t st, int M, int N, ModelPtrs t, DensityPtrs d, float min_opacity,
                           int max_screen_size, float world_thr) {
    if (M <= 0) return cudaSuccess;
    k_dc_keep<<<blocks(M, 256), 256, 0, st>>>(M, N, t.sc, t.op, d.max_radii, min_opacity, max_screen_size, world_thr,
                                              d.keep);
    return cudaGetLastError();
}

cudaError_t launch_dc_compact(cudaStream_t st, int M, int new_n, ModelPtrs t, int mc3, DensityPtrs d, ModelPtrs out) {
    if (M <= 0 || new_n <= 0) return cudaSuccess;
    k_dc_invert<<<blocks(M, 256), 256, 0, st>>>(M, d.keep, d.out, d.src);
    k_gather_rows<<<blocks((long long)new_n * 3, 256), 256, 0, st>>>(out.pos, t.pos, d.src, new_n, 3);
    k_gather_rows<<<blocks((long long)new_n * 3, 256), 256, 0, st>>>(out.sc, t.sc, d.src, new_n, 3);
    k_gather_rows<<<blocks((long long)new_n * 4, 256), 256, 0, st>>>(out.rot, t.rot, d.src, new_n, 4);
    k_gather_rows<<<blocks((long long)new_n * mc3, 256), 256, 0, st>>>(out.sh, t.sh, d.src, new_n, mc3);
    k_gather_rows<<<blocks(new_n, 256), 256, 0, st>>>(out.op, t.op, d.src, new_n, 1);
    return cudaGetLastError();
}

cudaError_t launch_fill(cudaStream_t st, float* p, long long n, float v) {
    if (n <= 0) return cudaSuccess;
    k_fill<<<blocks(n, 256), 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

}  // namespace gs3d
