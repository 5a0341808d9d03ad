// sort_static.cu -- gs3dc_sort_pairs_static: the pair sort of gs3dc_sort_pairs
// on caller-owned device buffers, with its scratch (control block, look-back
// descriptors, the second key/value buffer of the LSD ping-pong) in one
// file-scope __device__ array instead of memory allocated at run time.
//
// It is for callers that must not allocate device memory on their path: code
// without a gs3dc context (creating one allocates), frame loops that run under
// a fixed device-memory budget, and callers that cannot take the implicit
// device-wide synchronisation of cudaMalloc / cudaFree.  It calls no
// cudaMalloc, cudaFree or allocating library routine.
//
// Limits and sharing rules:
//   * at most GS3DC_STATIC_SORT_MAX_PAIRS pairs per call (the scratch is sized
//     for that many: about 16 MiB of device memory per device, reserved when
//     this library's device code is loaded);
//   * every call on a device uses the same scratch, which keeps the last call's
//     contents; each call clears the parts that must start at zero.  Calls
//     that overlap on the GPU (on different streams or host threads) race on
//     it and give wrong results;
//   * every call looks up the scratch's device address on the current device
//     (cudaGetSymbolAddress), so a device reset that reloads the module at a
//     new address leaves no stale pointer behind;
//   * a call is synchronous (it reads the status back and waits for the
//     stream), so it cannot be captured into a CUDA graph: on a capturing
//     stream it returns GS3DC_ERR_INVALID_ARG before doing anything.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "common.cuh"
#include "gs3d_cuda.h"
#include "kernels.cuh"

namespace gs3d {
namespace {

constexpr unsigned long long kStaticMaxPairs = GS3DC_STATIC_SORT_MAX_PAIRS;
constexpr unsigned long long kStaticMaxSortTiles = (kStaticMaxPairs + kSortTile - 1) / kSortTile;

constexpr size_t round256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets inside the scratch array.
constexpr size_t kOffControl = 0;
constexpr size_t kOffParams = round256(kOffControl + sizeof(Control));
constexpr size_t kOffFlags = round256(kOffParams + sizeof(StepParams));
constexpr size_t kOffDesc = round256(kOffFlags + sizeof(unsigned));
constexpr size_t kDescWords = (size_t)kMaxPasses * kStaticMaxSortTiles * 256;
constexpr size_t kOffKeys = round256(kOffDesc + kDescWords * sizeof(unsigned long long));
constexpr size_t kOffVals = round256(kOffKeys + kStaticMaxPairs * sizeof(unsigned long long));
constexpr size_t kScratchBytes = round256(kOffVals + kStaticMaxPairs * sizeof(unsigned));

static_assert(kScratchBytes < (size_t(17) << 20), "static sort scratch stays near 16 MiB");

}  // namespace
}  // namespace gs3d

// The scratch of every gs3dc_sort_pairs_static call on a device.
static __device__ __align__(256) unsigned char g_sort_scratch[gs3d::kScratchBytes];

namespace gs3d {
namespace {

// Flags a key whose tile field is >= num_tiles (k_ranges would index past the
// caller's tile_ranges with it).
__global__ void k_static_check(const unsigned long long* __restrict__ keys, unsigned long long n,
                               unsigned num_tiles, unsigned* bad) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    bool any = false;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        any |= (unsigned)(keys[i] >> 32) >= num_tiles;
    if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(bad, 1u);
}

// Publishes the pair count the sort kernels read (zero when a key was bad, so
// that they do nothing) and the bound of their look-back waits.
__global__ void k_static_commit(Control* ctrl, StepParams* sp, const unsigned* bad, unsigned long long n,
                                unsigned spin_limit) {
    if (threadIdx.x == 0) {
        ctrl->total_pairs = *bad ? 0ull : n;
        sp->spin_limit = spin_limit;
    }
}

int report(char* err, size_t err_len, int status, const char* fmt, ...) {
    if (err && err_len) {
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(err, err_len, fmt, ap);
        va_end(ap);
    }
    return status;
}

// The current device's scratch address.  In host code g_sort_scratch names a
// host-side stand-in, not device memory; the device address comes from the
// runtime, looked up on every call (a cheap table lookup once the module is
// loaded) so that it always belongs to the device's current context.
cudaError_t scratch_for_current_device(unsigned char** out, int* device) {
    cudaError_t e = cudaGetDevice(device);
    if (e != cudaSuccess) return e;
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

// True when the byte ranges [a, a + na) and [b, b + nb) share a byte.
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return na && nb && x < y + nb && y < x + na;
}

// True when p is device (or managed) memory of `device`.
bool is_device_pointer(const void* p, int device) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

int bit_length_u32(unsigned x) { return x ? 32 - __builtin_clz(x) : 0; }

}  // namespace
}  // namespace gs3d

using namespace gs3d;

#define CKS(call)                                                                                      \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return report(err, err_len, GS3DC_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));      \
    } while (0)

extern "C" int gs3dc_sort_pairs_static(int64_t total_pairs, const uint64_t* keys, const uint32_t* values,
                                       int num_tiles, uint64_t* keys_sorted, uint32_t* values_sorted,
                                       uint32_t* tile_ranges, void* stream, char* err, size_t err_len) {
    if (err && err_len) err[0] = '\0';
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CKS(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone)
            return report(err, err_len, GS3DC_ERR_INVALID_ARG,
                          "the stream is being captured: this call waits for the stream and reads its status "
                          "back, so it cannot be part of a CUDA graph");
    }
    if (total_pairs < 0 || num_tiles <= 0)
        return report(err, err_len, GS3DC_ERR_INVALID_ARG, "bad pair input (P=%lld, tiles=%d)",
                      (long long)total_pairs, num_tiles);
    if ((unsigned long long)total_pairs > kStaticMaxPairs)
        return report(err, err_len, GS3DC_ERR_INVALID_ARG,
                      "%lld pairs exceed the static sort scratch (at most %llu pairs per call); "
                      "use gs3dc_sort_pairs for larger sorts",
                      (long long)total_pairs, kStaticMaxPairs);
    unsigned char* scratch = nullptr;
    int device = -1;
    CKS(scratch_for_current_device(&scratch, &device));
    const unsigned long long P = (unsigned long long)total_pairs;
    if (!tile_ranges || !is_device_pointer(tile_ranges, device) ||
        (P && (!keys || !values || !keys_sorted || !values_sorted || !is_device_pointer(keys, device) ||
               !is_device_pointer(values, device) || !is_device_pointer(keys_sorted, device) ||
               !is_device_pointer(values_sorted, device))))
        return report(err, err_len, GS3DC_ERR_INVALID_ARG,
                      "keys, values, keys_sorted, values_sorted and tile_ranges must be device memory of "
                      "the current device (%d)", device);
    if ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(keys_sorted)) & 7u ||
        (reinterpret_cast<uintptr_t>(values) | reinterpret_cast<uintptr_t>(values_sorted) |
         reinterpret_cast<uintptr_t>(tile_ranges)) & 3u)
        return report(err, err_len, GS3DC_ERR_INVALID_ARG, "misaligned key / value / range pointer");
    {
        // outputs may coincide exactly with their own input (in place) but overlap nothing else
        const size_t kb = P * sizeof(uint64_t), vb = P * sizeof(uint32_t), rb = 2 * (size_t)num_tiles * 4;
        const struct {
            const void* p;
            size_t n;
        } in_k{keys, kb}, in_v{values, vb}, out_k{keys_sorted, kb}, out_v{values_sorted, vb}, out_r{tile_ranges, rb};
        const bool bad_overlap =
            (overlaps(out_k.p, out_k.n, in_k.p, in_k.n) && out_k.p != in_k.p) ||
            (overlaps(out_v.p, out_v.n, in_v.p, in_v.n) && out_v.p != in_v.p) ||
            overlaps(out_k.p, out_k.n, in_v.p, in_v.n) || overlaps(out_v.p, out_v.n, in_k.p, in_k.n) ||
            overlaps(out_k.p, out_k.n, out_v.p, out_v.n) || overlaps(out_r.p, out_r.n, in_k.p, in_k.n) ||
            overlaps(out_r.p, out_r.n, in_v.p, in_v.n) || overlaps(out_r.p, out_r.n, out_k.p, out_k.n) ||
            overlaps(out_r.p, out_r.n, out_v.p, out_v.n);
        if (bad_overlap)
            return report(err, err_len, GS3DC_ERR_INVALID_ARG,
                          "output buffers overlap an input or each other (only keys == keys_sorted and "
                          "values == values_sorted, exactly, may share memory)");
    }

    Control* ctrl = reinterpret_cast<Control*>(scratch + kOffControl);
    StepParams* sp = reinterpret_cast<StepParams*>(scratch + kOffParams);
    unsigned* bad = reinterpret_cast<unsigned*>(scratch + kOffFlags);
    unsigned long long* desc = reinterpret_cast<unsigned long long*>(scratch + kOffDesc);
    unsigned long long* alt_keys = reinterpret_cast<unsigned long long*>(scratch + kOffKeys);
    unsigned* alt_vals = reinterpret_cast<unsigned*>(scratch + kOffVals);

    CKS(cudaMemsetAsync(tile_ranges, 0, 2 * (size_t)num_tiles * sizeof(uint32_t), st));
    if (P == 0) {
        CKS(cudaStreamSynchronize(st));
        return GS3DC_OK;
    }
    const int bits = 32 + bit_length_u32(num_tiles > 1 ? (unsigned)(num_tiles - 1) : 0u);
    const int passes = (bits + 7) / 8;
    const unsigned long long desc_stride = ((P + kSortTile - 1) / kSortTile) * 256ull;

    // The LSD passes alternate between two buffers; start in the one that makes
    // the last pass land in the caller's output.
    unsigned long long* k0 = (passes & 1) ? alt_keys : reinterpret_cast<unsigned long long*>(keys_sorted);
    unsigned* v0 = (passes & 1) ? alt_vals : values_sorted;
    unsigned long long* k1 = (passes & 1) ? reinterpret_cast<unsigned long long*>(keys_sorted) : alt_keys;
    unsigned* v1 = (passes & 1) ? values_sorted : alt_vals;
    if (static_cast<const void*>(k0) != static_cast<const void*>(keys))
        CKS(cudaMemcpyAsync(k0, keys, P * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    if (static_cast<const void*>(v0) != static_cast<const void*>(values))
        CKS(cudaMemcpyAsync(v0, values, P * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));

    // what must start at zero: control block (histograms, tickets, status),
    // the bad-key flag and this call's look-back descriptors
    CKS(cudaMemsetAsync(ctrl, 0, sizeof(Control), st));
    CKS(cudaMemsetAsync(bad, 0, sizeof(unsigned), st));
    CKS(cudaMemsetAsync(desc, 0, (size_t)passes * desc_stride * sizeof(unsigned long long), st));
    k_static_check<<<2 * sm_count(), 256, 0, st>>>(k0, P, (unsigned)num_tiles, bad);
    CKS(cudaGetLastError());
    k_static_commit<<<1, 32, 0, st>>>(ctrl, sp, bad, P, 1u << 22);
    CKS(cudaGetLastError());
    int which = 0;
    CKS(launch_radix_sort(st, sp, passes, P, k0, v0, k1, v1, desc, desc_stride, ctrl, &which));
    CKS(launch_tile_ranges(st, P, reinterpret_cast<unsigned long long*>(keys_sorted), tile_ranges, ctrl));

    struct {
        unsigned status;
        unsigned bad;
    } h{};
    CKS(cudaMemcpyAsync(&h.status, &ctrl->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CKS(cudaMemcpyAsync(&h.bad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CKS(cudaStreamSynchronize(st));
    if (h.bad)
        return report(err, err_len, GS3DC_ERR_INVALID_ARG, "a key's tile field is >= num_tiles (%d)", num_tiles);
    if (h.status & kStatusTimeout)
        return report(err, err_len, GS3DC_ERR_DEVICE_TIMEOUT, "a sort look-back wait exceeded its poll limit");
    return GS3DC_OK;
}
