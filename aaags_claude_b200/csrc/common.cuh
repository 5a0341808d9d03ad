// common.cuh -- device-side shared definitions of the 3DGS hot path.
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gs3d_types.h"

namespace gs3d {

constexpr int kTile = 16;            // 16x16 pixel tiles (RenderConfig default, include/types.h:64-65)
constexpr int kBlock = 256;          // threads per CTA of the per-Gaussian and per-tile kernels
constexpr int kMaxPasses = 8;         // radix passes (8-bit digits over <= 64 key bits)
constexpr int kHistParts = 128;      // copies of the multi-view emission's tile-digit counts (atomic spread)
constexpr int kDepthDigits = 4;       // depth-first ordering: digits of the Gaussian depth sort (control slots
                                      // 0..3); the pair sort on the tile bits uses slots kDepthDigits..
constexpr int kChosenDepthSkip = 1;   // reduced-storage form: low depth digits left out of the depth sort
                                      // (ordering by the upper 24 bits: sign, exponent, 15 mantissa bits)

// Device-status bits (Control::status).
constexpr unsigned kStatusOverflow = 1u;  // more tile pairs than capacity
constexpr unsigned kStatusTimeout = 2u;   // a bounded device-side wait gave up

// Device state that survives across steps (zeroed when a model is uploaded).
struct Persist {
    unsigned long long applied_steps;  // optimiser updates actually applied
    unsigned sticky_overflow;          // set by any overflowed step until the host acknowledges it
    unsigned pad_;
};

// Per-step parameters, resident in device memory so that a captured graph
// reads fresh camera / learning-rate values on every replay.
struct StepParams {
    gs3d_camera cam;
    gs3d_render_config cfg;
    float focal_x, focal_y;
    int grid_x, grid_y, num_tiles;
    int sh_deg_fwd;       // min(cfg.sh_degree, model degree): forward SH degree
    int sh_deg_model;     // model degree: the backward's SH degree (preprocessor_backward_cpu.cpp:213)
    int max_coeffs;
    int num_gaussians;
    int num_pixels;
    float inv_n;          // 1.0f / (H*W*3)  (loss.cpp:6)
    // optimiser
    int use_adam;
    float lr_pos, lr_scale, lr_rot, lr_sh, lr_opac;
    float beta1, beta2, eps, bc1, bc2;
    // radix sort
    int sort_bits;        // significant key bits (32 + tile bits)
    int sort_passes;
    unsigned spin_limit;  // bounded waits
    const float* gt;      // [H*W*3] device target of the fused L1 (read per replay)
    Persist* persist;
    const float* raw_rot; // [N*4] raw quaternions when the device model is an activated one (backward only)
    unsigned seed;        // per-step seed of the reduced-storage form's stochastic rounding
    // multi-view steps (one StepParams per view; zero for a single view): the view's
    // first global tile id and first pixel in the concatenated per-view buffers
    unsigned tile_base;
    unsigned pix_base;
};

// Small device control block, zeroed by one memset at the start of a step.
// The first kControlReadback bytes are what the host reads back per step.
struct Control {
    unsigned long long total_pairs;   // written by the last preprocess / bin block
    unsigned status;                  // kStatus* bits
    unsigned pad_;
    double loss_sum;                  // sum |image - gt| of the fused L1
    unsigned tickets[16];             // dynamic CTA tickets (0: preprocess/bin, 1..8: sort passes)
    unsigned hist[kMaxPasses][256];   // radix digit histograms of all passes
    unsigned long long gauss_keys;    // depth-first pipeline: keys of the Gaussian depth sort
    unsigned work[2];                 // persistent multi-view rasterisers: next tile of the forward / backward
    unsigned tile_bucket[2][33];      // heavy-first tile order over many tiles: bucket sizes, then cursors
};
constexpr size_t kControlReadback = 24;

// Raises `kernel`'s dynamic shared-memory limit to `bytes` on the current
// device, once per device: the attribute belongs to the device's context, so a
// process with contexts on several GPUs sets it on each.  `done` keeps one bit
// per device ordinal.
template <class K>
inline cudaError_t set_smem_once(std::atomic<unsigned long long>& done, K* kernel, int bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// The largest shared-memory carveout for `kernel` (kernels built for several
// CTAs per SM that need most of the 228 KB), once per device.
template <typename K>
inline cudaError_t set_carveout_max_once(std::atomic<unsigned long long>& done, K* kernel) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// Streaming multiprocessors of the current device, queried once per device
// ordinal (grid sizes of the grid-stride and persistent launches; results never
// depend on it).  1 if the query fails, which keeps every launch valid.
inline int sm_count() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    std::atomic<int>& slot = cache[dev & 63];
    int n = slot.load(std::memory_order_relaxed);
    if (n > 0) return n;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) return 1;
    slot.store(n, std::memory_order_relaxed);
    return n;
}

// ---- relaxed 64-bit accesses for decoupled look-back descriptors ----
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Look-back descriptor: flag in bits 62-63, value in bits 0-61.
constexpr unsigned long long kDescAgg = 1ull << 62;     // this block's aggregate only
constexpr unsigned long long kDescPrefix = 2ull << 62;  // inclusive prefix through this block
constexpr unsigned long long kDescValue = (1ull << 62) - 1;

// Decoupled look-back (Merrill & Garland, "Single-pass Parallel Prefix Scan
// with Decoupled Look-back", 2016), run by one thread for one counter.
// Descriptor of block b lives at desc[b * stride + lane_off].  Returns the
// exclusive prefix of block `blk`.  Waits are bounded: after spin_limit polls
// of a descriptor that is still empty the status word gets kStatusTimeout and
// the partial prefix is used (the result is then invalid and the host reports
// GS3DC_ERR_DEVICE_TIMEOUT).  Block indices are tickets taken in launch order,
// so every predecessor is resident or finished and publishes without waiting.
// first_blk > 0: the scan restarts there (segments of blocks scanned apart).
__device__ __forceinline__ unsigned long long lookback_exclusive_strided(
    unsigned long long* desc, int blk, int stride, int lane_off, unsigned long long aggregate,
    unsigned* status, unsigned spin_limit, int first_blk = 0) {
    unsigned long long* mine = desc + (size_t)blk * stride + lane_off;
    if (blk == first_blk) {
        st_relaxed(mine, kDescPrefix | aggregate);
        return 0ull;
    }
    st_relaxed(mine, kDescAgg | aggregate);
    unsigned long long excl = 0;
    int j = blk - 1;
    unsigned spins = 0;
    while (j >= first_blk) {
        const unsigned long long d = ld_relaxed(desc + (size_t)j * stride + lane_off);
        const unsigned long long flag = d & ~kDescValue;
        if (flag == 0ull) {
            if (++spins > spin_limit) {
                atomicOr(status, kStatusTimeout);
                break;
            }
            __nanosleep(32);
            continue;
        }
        excl += d & kDescValue;
        if (flag == kDescPrefix) break;
        --j;
    }
    st_relaxed(mine, kDescPrefix | (excl + aggregate));
    return excl;
}

// The same look-back for one counter, run by a whole warp: lane l examines
// block base - l, so one round covers 32 predecessors.  The prefix ends at the
// nearest block that published an inclusive prefix; every block after it must
// have published at least its aggregate, else the round is polled again
// (bounded as above).  Blocks before block 0 count as a zero prefix.  Every
// lane returns the exclusive prefix.
//
// Split in two for callers with work to do between publishing and walking:
// lookback_publish (one thread) and warp_lookback_walk (the whole warp, after
// the publish).
__device__ __forceinline__ void lookback_publish(unsigned long long* desc, int blk, unsigned long long aggregate) {
    st_relaxed(desc + blk, (blk == 0 ? kDescPrefix : kDescAgg) | aggregate);
}

__device__ __forceinline__ unsigned long long warp_lookback_walk(unsigned long long* desc, int blk,
                                                                 unsigned long long aggregate, unsigned* status,
                                                                 unsigned spin_limit) {
    const int lane = (int)(threadIdx.x & 31);
    unsigned long long* mine = desc + blk;
    if (blk == 0) return 0ull;
    unsigned long long excl = 0;
    int base = blk - 1;
    unsigned spins = 0;
    for (;;) {
        const int j = base - lane;
        const unsigned long long d = j >= 0 ? ld_relaxed(desc + j) : kDescPrefix;
        const unsigned long long flag = d & ~kDescValue;
        const unsigned empty = __ballot_sync(0xffffffffu, flag == 0ull);
        const unsigned pre = __ballot_sync(0xffffffffu, flag == kDescPrefix);
        const int first = pre ? __ffs(pre) - 1 : 31;   // lanes 0..first hold the blocks to add
        const unsigned need = first == 31 ? 0xffffffffu : ((2u << first) - 1u);
        if (empty & need) {
            if (++spins > spin_limit) {
                if (lane == 0) atomicOr(status, kStatusTimeout);
                break;
            }
            __nanosleep(32);
            continue;
        }
        unsigned long long v = lane <= first ? (d & kDescValue) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if (pre) break;
        base -= 32;
    }
    if (lane == 0) st_relaxed(mine, kDescPrefix | (excl + aggregate));
    return excl;
}

__device__ __forceinline__ unsigned long long warp_lookback_exclusive(unsigned long long* desc, int blk,
                                                                      unsigned long long aggregate,
                                                                      unsigned* status, unsigned spin_limit) {
    if ((threadIdx.x & 31) == 0) lookback_publish(desc, blk, aggregate);
    return warp_lookback_walk(desc, blk, aggregate, status, spin_limit);
}


// ---- TMA bulk copies (cp.async.bulk) completing on an mbarrier ----
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the async (TMA) proxy.
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces `bytes` of transactions to wait for.
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned phase) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return done != 0;
}

// Bounded wait for `phase` of the barrier: false (and kStatusTimeout) if the
// copies have not landed after spin_limit polls.
// Bulk prefetch of [src, src + bytes) into L2 (no shared memory, no completion
// to wait for); src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void prefetch_l2(const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned phase, unsigned spin_limit,
                                          unsigned* status) {
    for (unsigned i = 0; i < spin_limit; i++)
        if (mbar_try_wait(bar, phase)) return true;
    atomicOr(status, kStatusTimeout);
    return false;
}

// Correctly rounded float exp (double evaluation, one rounding).  glibc's
// expf, which the reference calls through std::exp(float), agrees with it on
// all but ~0.006% of inputs (by 1 ulp there).
__device__ __forceinline__ float exp_ref(float x) { return (float)exp((double)x); }

// Block-wide inclusive scan of one int per thread (256 threads); returns the
// inclusive value, *total gets the block sum.  s_warp needs 8 ints.
template <int NW = kBlock / 32>   // warps of the CTA, <= 32
__device__ __forceinline__ int block_inclusive_scan(int v, int* s_warp, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    if (lane == 31) s_warp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int w = lane < NW ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < NW; o <<= 1) {
            int n = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += n;
        }
        if (lane < NW) s_warp[lane] = w;
    }
    __syncthreads();
    int add = warp > 0 ? s_warp[warp - 1] : 0;
    *total = s_warp[NW - 1];
    return v + add;
}

}  // namespace gs3d
