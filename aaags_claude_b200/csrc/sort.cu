// sort.cu -- stable LSD radix sort of (tile|depth key, Gaussian index) pairs
// and tile-range identification, replacing SorterCPU::sort
// (harmonyos_3dgs src/cpu/sorter_cpu.cpp:6-44).
//
// Design (one-sweep, after Adinets & Merrill, "Onesweep: A Faster Least
// Significant Digit Radix Sort for GPUs", 2022):
//   k_radix_hist  one read of the keys counts the 8-bit digits of every pass
//                 (hist_add: one shared add for a digit the warp shares).
//   k_onesweep    one launch per pass.  A CTA takes the next 4096-key tile by
//                 ticket, ranks its keys per warp with peer_mask8 /
//                 popc, publishes its per-digit counts and finds its global
//                 per-digit offsets by decoupled look-back (bounded waits),
//                 reorders the tile in shared memory and writes it out in
//                 digit-contiguous runs.  Ranks follow input order, so the sort
//                 is stable: equal keys keep the Gaussian order of the binning,
//                 i.e. the result is the (key, value)-sorted order.
//   k_ranges      (start, end) per tile from the sorted keys
//                 (sorter_cpu.cpp:28-43).
// Only the significant key bits are sorted: 32 depth bits plus
// ceil(log2(num_tiles)) tile bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "kernels.cuh"

namespace gs3d {
namespace {

constexpr int kHistThreads = 512;

// The lanes of `mask` whose 8-bit digit equals this lane's (this lane
// included), from eight ballots over the digit's bits: the same set
// __match_any_sync returns, at a fraction of its cost when the digits of a
// warp are mostly distinct.  Called by every lane of `mask`.
__device__ __forceinline__ unsigned peer_mask8(unsigned mask, unsigned d) {
    unsigned peers = mask;
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const bool bit = (d >> b) & 1u;
        const unsigned bal = __ballot_sync(mask, bit);
        peers &= bit ? bal : ~bal;
    }
    return peers;
}

// Adds one to bin d of the shared histogram h for each lane of mask (which
// all call it).  A digit the whole warp shares (the upper digits of depth keys,
// a segment's padding) takes one add; other digits take one add per lane.
// (Measured against one add per distinct value, found with 8 ballots or
// match_any: 64-view step 33.71 / 34.03 -> 33.26 ms.)
__device__ __forceinline__ void hist_add(unsigned* h, unsigned mask, unsigned d) {
    const int leader = __ffs(mask) - 1;
    const unsigned d0 = __shfl_sync(mask, d, leader);
    if (__all_sync(mask, d == d0)) {
        if ((int)(threadIdx.x & 31) == leader) atomicAdd(&h[d0], (unsigned)__popc(mask));
    } else {
        atomicAdd(&h[d], 1u);
    }
}

// Digit histograms of digits [first, passes) (digit d = key bits 8d..8d+7)
// into ctrl->hist[slot_base + d - first].
template <typename K>
__global__ void __launch_bounds__(kHistThreads) k_radix_hist(const K* __restrict__ keys,
                                                             unsigned long long capacity, int first, int passes,
                                                             int slot_base, const unsigned long long* count,
                                                             Control* ctrl) {
    __shared__ unsigned s_h[kMaxPasses * 256];
    for (int e = first * 256 + threadIdx.x; e < passes * 256; e += blockDim.x) s_h[e] = 0;
    __syncthreads();
    const unsigned long long P = min(*count, capacity);
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < P; base += stride) {
        const unsigned long long i = base + threadIdx.x;
        const bool valid = i < P;
        const unsigned mask = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const K key = keys[i];
            for (int p = first; p < passes; p++) hist_add(&s_h[p * 256], mask, (unsigned)(key >> (8 * p)) & 255u);
        }
    }
    __syncthreads();
    for (int e = first * 256 + threadIdx.x; e < passes * 256; e += blockDim.x)
        if (s_h[e]) atomicAdd(&ctrl->hist[slot_base + (e >> 8) - first][e & 255], s_h[e]);
}

// Digit histograms per segment: the keys are segments of seg_keys keys (a
// multiple of kSegTile), sorted apart; CTA b counts digits [first, first +
// digits) of keys [b kSegTile, (b + 1) kSegTile), which lie in one segment,
// into seg_hist[(segment * digits + digit - first) * 256 + value].
constexpr unsigned long long kSegTile = 8192;
__global__ void __launch_bounds__(kHistThreads) k_seg_hist(const unsigned* __restrict__ keys,
                                                           unsigned long long seg_keys, int first, int digits,
                                                           unsigned* __restrict__ seg_hist) {
    __shared__ unsigned s_h[kMaxPasses * 256];
    for (int e = threadIdx.x; e < digits * 256; e += blockDim.x) s_h[e] = 0;
    __syncthreads();
    const unsigned long long base = (unsigned long long)blockIdx.x * kSegTile;
    // 16-byte loads, all issued before the counting (kSegTile / 4 / kHistThreads = 4 per thread)
    constexpr int kVec = (int)(kSegTile / 4 / kHistThreads);
    static_assert(kSegTile % (4 * kHistThreads) == 0, "whole 16-byte loads per thread");
    uint4 kv[kVec];
    const uint4* k4 = reinterpret_cast<const uint4*>(keys + base);
#pragma unroll
    for (int j = 0; j < kVec; j++) kv[j] = k4[j * kHistThreads + threadIdx.x];
#pragma unroll
    for (int j = 0; j < kVec; j++) {
        const unsigned kk[4] = {kv[j].x, kv[j].y, kv[j].z, kv[j].w};
#pragma unroll
        for (int e = 0; e < 4; e++)
            for (int p = 0; p < digits; p++)
                hist_add(&s_h[p * 256], 0xffffffffu, (kk[e] >> (8 * (first + p))) & 255u);
    }
    __syncthreads();
    const unsigned long long seg = base / seg_keys;
    for (int e = threadIdx.x; e < digits * 256; e += blockDim.x)
        if (s_h[e]) atomicAdd(&seg_hist[seg * (unsigned long long)digits * 256ull + (unsigned long long)e], s_h[e]);
}

// Segments of a segmented onesweep (SEG): seg_keys keys each (a multiple of
// the CTA's keys), their digit histograms from k_seg_hist.
struct SegSort {
    const unsigned* hist;
    unsigned long long seg_keys;
    int first, digits;
};

// Keys per thread of a onesweep CTA: 16, or 32 for large sorts of 32-bit keys
// (8192 keys per CTA: half the CTAs, so half the per-digit look-backs; measured
// faster from tens of millions of keys on, slower at a few million).
constexpr unsigned long long kWideSweepKeys = 1ull << 25;

// Shared memory of one onesweep CTA (dynamic; ~58 KB for 64-bit keys at 16 per
// thread, ~42 / ~74 KB for 32-bit keys at 16 / 32).
template <typename K, int ITEMS>
struct SweepShared {
    K keys[kSortThreads * ITEMS];
    unsigned vals[kSortThreads * ITEMS];
    unsigned whist[kSortThreads / 32][256];   // per-warp digit counts, then the warp's first tile slot of digit d
    unsigned long long gdelta[256];           // output index of tile slot j holding digit d: gdelta[d] + j
    unsigned long long scan[8];
    int tile;
};

// CTAs per SM a onesweep launch is built for: with the values loaded only for
// the scatter, a thread holds its keys and 16-bit ranks, and shared memory
// allows 3 CTAs at 8192 32-bit keys or 4096 64-bit keys, 5 at 4096 32-bit keys.
template <typename K, int ITEMS>
constexpr int sweep_ctas_per_sm() { return ITEMS > 16 || sizeof(K) > 4 ? 3 : 5; }

// Exclusive scan over the 256 threads of one 64-bit value each.
__device__ __forceinline__ unsigned long long block_exclusive_scan64(unsigned long long v, unsigned long long* s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long n = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += n;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    unsigned long long add = 0;
    for (int w = 0; w < warp; w++) add += s_w[w];
    __syncthreads();
    return x - v + add;
}

// One pass over digit `pass` (key bits 8*pass..); `slot` selects the digit
// histogram and CTA ticket in the control block.  The values are not held in
// registers: the CTA asks for its slice to be brought into L2 when it starts
// and loads each value where it scatters it.  SEG: the keys are segments
// sorted apart (SegSort): a CTA's digit offsets start at its segment and its
// look-back stops at the segment's first CTA.
template <typename K, int ITEMS, bool SEG = false>
__global__ void __launch_bounds__(kSortThreads, sweep_ctas_per_sm<K, ITEMS>()) k_onesweep(const StepParams* __restrict__ sp,
                                                              const K* __restrict__ kin,
                                                              const unsigned* __restrict__ vin,
                                                              K* __restrict__ kout,
                                                              unsigned* __restrict__ vout,
                                                              unsigned long long capacity, int pass, int slot,
                                                              unsigned long long* desc,
                                                              const unsigned long long* count,
                                                              Control* ctrl, SegSort sg = SegSort{}) {
    constexpr int kItems = ITEMS;
    constexpr int kTileKeys = kSortThreads * kItems;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SweepShared<K, ITEMS>& sm = *reinterpret_cast<SweepShared<K, ITEMS>*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int shift = 8 * pass;
    const unsigned long long P = min(*count, capacity);
    if (tid == 0) sm.tile = (int)atomicAdd(&ctrl->tickets[1 + slot], 1u);
    for (int e = tid; e < (kSortThreads / 32) * 256; e += kSortThreads) (&sm.whist[0][0])[e] = 0;
    __syncthreads();
    const int t = sm.tile;
    const unsigned long long base = (unsigned long long)t * kTileKeys;
    if (base >= P) return;

    if (tid == 0) {
        // the tile's values (whole 16-byte units inside [base, P), from a 16-byte aligned start: a
        // caller's buffer may be only 4-byte aligned) into L2 for the scatter
        const unsigned long long nv = min((unsigned long long)kTileKeys, P - base) & ~3ull;
        if (nv && (reinterpret_cast<uintptr_t>(vin + base) & 15u) == 0)
            prefetch_l2(vin + base, (unsigned)(nv * sizeof(unsigned)));
    }
    K key[kItems];
    unsigned rank2[(kItems + 1) / 2];   // two 16-bit ranks per register (a rank is < 32 * kItems)
#pragma unroll
    for (int it = 0; it < kItems; it++) {
        const unsigned long long idx = base + (unsigned long long)(warp * 32 * kItems + it * 32 + lane);
        key[it] = idx < P ? kin[idx] : (K)~(K)0;   // sentinel: digit 255, ranks after every real key
    }
    const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int it = 0; it < kItems; it++) {
        const unsigned d = (unsigned)(key[it] >> shift) & 255u;
        const unsigned peers = peer_mask8(0xffffffffu, d);
        // one leader per digit adds the group's size to the warp's count and
        // shuffles the old value to its group.  The atomic has returned before
        // the shuffle that every lane passes, so it precedes every atomic of
        // the warp's later items: the value counts this digit in earlier items.
        const int leader = __ffs(peers) - 1;
        unsigned prior = 0;
        if (lane == leader) prior = atomicAdd(&sm.whist[warp][d], (unsigned)__popc(peers));
        prior = __shfl_sync(0xffffffffu, prior, leader);
        const unsigned rank = prior + (unsigned)__popc(peers & lt_mask);
        if (it & 1) rank2[it >> 1] |= rank << 16;
        else rank2[it >> 1] = rank;
    }
    __syncthreads();
    // thread d owns digit d: per-warp exclusive prefixes and the tile count
    const unsigned d = (unsigned)tid;
    unsigned run = 0;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; w++) {
        const unsigned c = sm.whist[w][d];
        sm.whist[w][d] = run;
        run += c;
    }
    // global offset of digit d for this tile: all smaller digits everywhere,
    // plus digit d in the tiles before this one (decoupled look-back)
    unsigned long long seg_base = 0;
    int first_t = 0;
    unsigned long long hist_d;
    if (SEG) {
        const unsigned long long seg = base / sg.seg_keys;
        seg_base = seg * sg.seg_keys;
        first_t = (int)(seg_base / kTileKeys);
        hist_d = sg.hist[(seg * (unsigned long long)sg.digits + (unsigned long long)(pass - sg.first)) * 256ull + d];
    } else {
        hist_d = ctrl->hist[slot][d];
    }
    const unsigned long long digit_start = seg_base + block_exclusive_scan64(hist_d, sm.scan);
    const unsigned long long tile_excl = lookback_exclusive_strided(
        desc, t, 256, (int)d, (unsigned long long)run, &ctrl->status, sp->spin_limit, first_t);
    // tile-local start of digit d, folded into the warps' prefixes and the output offset
    const unsigned dp = (unsigned)block_exclusive_scan64((unsigned long long)run, sm.scan);
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; w++) sm.whist[w][d] += dp;
    sm.gdelta[d] = digit_start + tile_excl - dp;
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kItems; it++) {
        const unsigned long long idx = base + (unsigned long long)(warp * 32 * kItems + it * 32 + lane);
        const unsigned dd = (unsigned)(key[it] >> shift) & 255u;
        const unsigned pos = sm.whist[warp][dd] + ((rank2[it >> 1] >> (16 * (it & 1))) & 0xffffu);
        sm.keys[pos] = key[it];
        sm.vals[pos] = idx < P ? vin[idx] : 0u;
    }
    __syncthreads();
    const int n_valid = (int)min((unsigned long long)kTileKeys, P - base);
    for (int j = tid; j < n_valid; j += kSortThreads) {
        const K k = sm.keys[j];
        const unsigned dd = (unsigned)(k >> shift) & 255u;
        const unsigned long long out = sm.gdelta[dd] + (unsigned long long)j;
        kout[out] = k;
        vout[out] = sm.vals[j];
    }
}

__device__ __forceinline__ unsigned tile_of(unsigned long long key) { return (unsigned)(key >> 32); }

// Ranges of (view, tile) runs: a run starts / ends where the global id changes.
// A key is the view's local tile id in its low 8 * tile digits bits and the
// view above them (the emission puts it there; the sort leaves it alone).
// Four pairs per thread from one 16-byte load; each id is compared with its
// successor's (as k_ranges32).
__global__ void k_ranges_views4(const unsigned* __restrict__ keys, const StepParams* __restrict__ views,
                                unsigned long long capacity, unsigned* __restrict__ ranges, Control* ctrl) {
    const unsigned long long P = min(ctrl->total_pairs, capacity);
    const int tile_bits = 8 * (views[0].sort_passes - kDepthDigits);
    const unsigned local_mask = (1u << tile_bits) - 1u;   // tile_bits <= 24
    // grid-stride over the pairs present (the grid is sized for the SMs, not the capacity)
    const unsigned long long step = 4ull * gridDim.x * blockDim.x;
    for (unsigned long long i0 = 4ull * ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x); i0 < P;
         i0 += step) {
        unsigned k[5];
        if (i0 + 4 <= capacity) {
            const uint4 kk = *reinterpret_cast<const uint4*>(keys + i0);
            k[0] = kk.x, k[1] = kk.y, k[2] = kk.z, k[3] = kk.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) k[j] = i0 + j < P ? keys[i0 + j] : 0u;
        }
        k[4] = i0 + 4 < P ? keys[i0 + 4] : 0u;
        unsigned t[5];
#pragma unroll
        for (int j = 0; j < 5; j++) t[j] = views[k[j] >> tile_bits].tile_base + (k[j] & local_mask);
        if (i0 == 0) ranges[2 * t[0]] = 0u;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const unsigned long long i = i0 + (unsigned long long)j;
            if (i >= P) break;
            const bool last = i + 1 == P;
            if (last || t[j + 1] != t[j]) {
                ranges[2 * t[j] + 1] = (unsigned)(i + 1);
                if (!last) ranges[2 * t[j + 1]] = (unsigned)(i + 1);
            }
        }
    }
}


// One thread per key (the grid covers the capacity): a tile's range starts
// where its key differs from the previous one and ends where it differs
// from the next.
template <typename K>
__global__ void k_ranges(const K* __restrict__ keys, unsigned long long capacity, unsigned* __restrict__ ranges,
                         Control* ctrl) {
    const unsigned long long P = min(ctrl->total_pairs, capacity);
    const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const unsigned t = tile_of(keys[i]);
    if (i == 0 || tile_of(keys[i - 1]) != t) ranges[2 * t] = (unsigned)i;
    if (i == P - 1 || tile_of(keys[i + 1]) != t) ranges[2 * t + 1] = (unsigned)(i + 1);
}

// Tile ranges over sorted 32-bit tile ids, four ids per thread from one
// 16-byte load: a run ends at i + 1 where id i differs from id i + 1 (or i is
// the last pair), and the next run starts there.
__global__ void k_ranges32(const unsigned* __restrict__ tiles, unsigned long long capacity,
                           unsigned* __restrict__ ranges, Control* ctrl) {
    const unsigned long long P = min(ctrl->total_pairs, capacity);
    // grid-stride over the pairs present (the grid is sized for the SMs, not the capacity)
    const unsigned long long step = 4ull * gridDim.x * blockDim.x;
    for (unsigned long long i0 = 4ull * ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x); i0 < P;
         i0 += step) {
        unsigned t[5];
        if (i0 + 4 <= capacity) {
            const uint4 v = *reinterpret_cast<const uint4*>(tiles + i0);
            t[0] = v.x;
            t[1] = v.y;
            t[2] = v.z;
            t[3] = v.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) t[j] = i0 + j < P ? tiles[i0 + j] : 0u;
        }
        t[4] = i0 + 4 < P ? tiles[i0 + 4] : 0u;
        if (i0 == 0) ranges[2 * t[0]] = 0u;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const unsigned long long i = i0 + (unsigned long long)j;
            if (i >= P) break;
            const bool last = i + 1 == P;
            if (last || t[j + 1] != t[j]) {
                ranges[2 * t[j] + 1] = (unsigned)(i + 1);
                if (!last) ranges[2 * t[j + 1]] = (unsigned)(i + 1);
            }
        }
    }
}

// Heavy-first tile order: one CTA buckets the tiles by floor(log2(pairs))
// and writes them heaviest bucket first, so the rasterisers (one CTA per
// tile) start the long central tiles before the many short ones instead of
// finishing on them.  The order inside a bucket does not matter (tiles are
// independent).
__global__ void __launch_bounds__(1024) k_tile_order(const unsigned* __restrict__ ranges, int num_tiles,
                                                     unsigned* __restrict__ order) {
    __shared__ unsigned s_cnt[33];
    __shared__ unsigned s_off[33];
    if (threadIdx.x < 33) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) {
        const unsigned n = ranges[2 * t + 1] - ranges[2 * t];
        atomicAdd(&s_cnt[n ? 32 - __clz(n) : 0], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned acc = 0;
        for (int b = 32; b >= 0; b--) {   // heaviest bucket first
            s_off[b] = acc;
            acc += s_cnt[b];
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < num_tiles; t += blockDim.x) {
        const unsigned n = ranges[2 * t + 1] - ranges[2 * t];
        order[atomicAdd(&s_off[n ? 32 - __clz(n) : 0], 1u)] = (unsigned)t;
    }
}

// The same order over many tiles (several views' tiles): per-CTA bucket counts
// into ctrl->tile_bucket[0], then every CTA reserves its bucket ranges with one
// global atomic per bucket (cursors in ctrl->tile_bucket[1], starting at the
// heavy-first bucket offsets) and writes its tiles there.
__device__ __forceinline__ int tile_bucket_of(const unsigned* __restrict__ ranges, int t) {
    const unsigned n = ranges[2 * t + 1] - ranges[2 * t];
    return n ? 32 - __clz(n) : 0;
}

__global__ void __launch_bounds__(256) k_tile_bucket_count(const unsigned* __restrict__ ranges, int num_tiles,
                                                          Control* ctrl) {
    __shared__ unsigned s_cnt[33];
    if (threadIdx.x < 33) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < num_tiles; t += gridDim.x * blockDim.x)
        atomicAdd(&s_cnt[tile_bucket_of(ranges, t)], 1u);
    __syncthreads();
    if (threadIdx.x < 33 && s_cnt[threadIdx.x]) atomicAdd(&ctrl->tile_bucket[0][threadIdx.x], s_cnt[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_tile_bucket_scatter(const unsigned* __restrict__ ranges, int num_tiles,
                                                            Control* ctrl, unsigned* __restrict__ order) {
    __shared__ unsigned s_cnt[33], s_base[33], s_off[33];
    if (threadIdx.x < 33) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    const int t0 = blockIdx.x * blockDim.x * 4;
    int bk[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int t = t0 + r * blockDim.x + threadIdx.x;
        bk[r] = t < num_tiles ? tile_bucket_of(ranges, t) : -1;
        if (bk[r] >= 0) atomicAdd(&s_cnt[bk[r]], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 33) {
        // heavy-first offset of bucket b: the sizes of the heavier buckets
        unsigned off = 0;
        for (int h = 32; h > (int)threadIdx.x; h--) off += ctrl->tile_bucket[0][h];
        const unsigned n = s_cnt[threadIdx.x];
        s_base[threadIdx.x] = off + (n ? atomicAdd(&ctrl->tile_bucket[1][threadIdx.x], n) : 0u);
        s_off[threadIdx.x] = 0;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int t = t0 + r * blockDim.x + threadIdx.x;
        if (bk[r] >= 0) order[s_base[bk[r]] + atomicAdd(&s_off[bk[r]], 1u)] = (unsigned)t;
    }
}

// One warp plays block 1 of a look-back whose block 0 never publishes, first
// with the warp-wide look-back, then with the one-thread look-back: each wait
// must run out after spin_limit polls; kStatusTimeout is raised when both did.
__global__ void k_wait_selftest(unsigned long long* desc, unsigned* status, unsigned spin_limit) {
    __shared__ unsigned s_warp, s_thread;
    if (threadIdx.x == 0) s_warp = s_thread = 0u;
    __syncwarp();
    warp_lookback_exclusive(desc, 1, 5ull, &s_warp, spin_limit);
    __syncwarp();
    if (threadIdx.x == 0) {
        lookback_exclusive_strided(desc, 1, 1, 0, 5ull, &s_thread, spin_limit);
        if ((s_warp & kStatusTimeout) && (s_thread & kStatusTimeout)) atomicOr(status, kStatusTimeout);
    }
}

}  // namespace

namespace {
__global__ void __launch_bounds__(256) k_clear_regions(ClearRegions r) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        unsigned long long* p = r.p[k];
        if (!p) continue;
        for (unsigned long long i = t; i < r.words[k]; i += stride) p[i] = 0ull;
    }
}
}  // namespace

cudaError_t launch_clear_regions(cudaStream_t st, const ClearRegions& r) {
    unsigned long long most = 0;
    for (int k = 0; k < 4; k++)
        if (r.p[k] && r.words[k] > most) most = r.words[k];
    if (most == 0) return cudaSuccess;
    const unsigned long long want = (most + 255) / 256;
    const unsigned long long cap = 8ull * (unsigned long long)sm_count();
    const unsigned blocks = (unsigned)(want < cap ? want : cap);
    k_clear_regions<<<blocks, 256, 0, st>>>(r);
    return cudaGetLastError();
}

cudaError_t launch_wait_selftest(cudaStream_t st, unsigned long long* desc2, unsigned* status, unsigned spin_limit) {
    k_wait_selftest<<<1, 32, 0, st>>>(desc2, status, spin_limit);
    return cudaGetLastError();
}

namespace {

// Digits [first, passes) of the keys, slots slot_base..; desc holds
// (passes - first) * desc_stride zeroed descriptors (strides sized for kSortTile
// keys per CTA are an upper bound for either CTA size).
template <typename K, int ITEMS>
cudaError_t radix_sort_impl(cudaStream_t st, const StepParams* sp, int first, int passes, int slot_base,
                            bool hist_done, unsigned long long capacity, K* keys0, unsigned* vals0, K* keys1,
                            unsigned* vals1, unsigned long long* desc, unsigned long long desc_stride,
                            Control* ctrl, int* which, cudaEvent_t after_hist, const unsigned long long* count) {
    *which = 0;
    if (capacity == 0 || passes <= first) return cudaSuccess;
    if (!count) count = &ctrl->total_pairs;
    static std::atomic<unsigned long long> attr_done{0};
    const int smem = (int)sizeof(SweepShared<K, ITEMS>);
    cudaError_t e = set_smem_once(attr_done, k_onesweep<K, ITEMS>, smem);
    if (e != cudaSuccess) return e;
    static std::atomic<unsigned long long> carve_done{0};
    if ((e = set_carveout_max_once(carve_done, k_onesweep<K, ITEMS>)) != cudaSuccess) return e;
    if (!hist_done) {
        k_radix_hist<K><<<2 * sm_count(), kHistThreads, 0, st>>>(keys0, capacity, first, passes, slot_base, count, ctrl);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (after_hist && (e = cudaEventRecord(after_hist, st)) != cudaSuccess) return e;
    const unsigned long long tile_keys = (unsigned long long)kSortThreads * ITEMS;
    const unsigned long long tiles = (capacity + tile_keys - 1) / tile_keys;
    K* kin = keys0;
    unsigned* vin = vals0;
    K* kout = keys1;
    unsigned* vout = vals1;
    for (int p = first; p < passes; p++) {
        const int slot = slot_base + p - first;
        k_onesweep<K, ITEMS><<<(unsigned)tiles, kSortThreads, smem, st>>>(
            sp, kin, vin, kout, vout, capacity, p, slot, desc + (unsigned long long)(p - first) * desc_stride, count,
            ctrl);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        K* tk = kin;
        kin = kout;
        kout = tk;
        unsigned* tv = vin;
        vin = vout;
        vout = tv;
    }
    *which = (passes - first) & 1;
    return cudaSuccess;
}

template <int ITEMS>
cudaError_t radix_sort_seg_impl(cudaStream_t st, const StepParams* sp, int first, int digits,
                                unsigned long long capacity, unsigned long long seg_keys, unsigned* keys0,
                                unsigned* vals0, unsigned* keys1, unsigned* vals1, unsigned long long* desc,
                                unsigned long long desc_stride, unsigned* seg_hist, Control* ctrl, int* which) {
    *which = 0;
    if (capacity == 0 || digits <= 0) return cudaSuccess;
    static std::atomic<unsigned long long> attr_done{0}, carve_done{0};
    const int smem = (int)sizeof(SweepShared<unsigned, ITEMS>);
    cudaError_t e = set_smem_once(attr_done, k_onesweep<unsigned, ITEMS, true>, smem);
    if (e != cudaSuccess) return e;
    if ((e = set_carveout_max_once(carve_done, k_onesweep<unsigned, ITEMS, true>)) != cudaSuccess) return e;
    k_seg_hist<<<(unsigned)(capacity / kSegTile), kHistThreads, 0, st>>>(keys0, seg_keys, first, digits, seg_hist);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const unsigned long long tiles = capacity / ((unsigned long long)kSortThreads * ITEMS);
    const SegSort sg{seg_hist, seg_keys, first, digits};
    unsigned *kin = keys0, *vin = vals0, *kout = keys1, *vout = vals1;
    for (int p = first; p < first + digits; p++) {
        k_onesweep<unsigned, ITEMS, true><<<(unsigned)tiles, kSortThreads, smem, st>>>(
            sp, kin, vin, kout, vout, capacity, p, p - first, desc + (unsigned long long)(p - first) * desc_stride,
            &ctrl->gauss_keys, ctrl, sg);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    *which = digits & 1;
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_radix_sort32_segmented(cudaStream_t st, const StepParams* sp, int first_digit, int digits,
                                          unsigned long long capacity, unsigned long long seg_keys, unsigned* keys0,
                                          unsigned* vals0, unsigned* keys1, unsigned* vals1,
                                          unsigned long long* desc, unsigned long long desc_stride,
                                          unsigned* seg_hist, Control* ctrl, int* which) {
    if (seg_keys == 0 || seg_keys % kSegTile != 0 || capacity % seg_keys != 0) return cudaErrorInvalidValue;
    if (capacity >= kWideSweepKeys)
        return radix_sort_seg_impl<32>(st, sp, first_digit, digits, capacity, seg_keys, keys0, vals0, keys1, vals1,
                                       desc, desc_stride, seg_hist, ctrl, which);
    return radix_sort_seg_impl<kSortItems>(st, sp, first_digit, digits, capacity, seg_keys, keys0, vals0, keys1,
                                           vals1, desc, desc_stride, seg_hist, ctrl, which);
}

cudaError_t launch_radix_sort(cudaStream_t st, const StepParams* sp, int passes, unsigned long long capacity,
                              unsigned long long* keys0, unsigned* vals0, unsigned long long* keys1,
                              unsigned* vals1, unsigned long long* desc, unsigned long long desc_stride,
                              Control* ctrl, int* which, cudaEvent_t after_hist, int first_pass,
                              const unsigned long long* count) {
    // 64-bit keys: digit p uses slot p, descriptors from desc + p * desc_stride
    return radix_sort_impl<unsigned long long, kSortItems>(st, sp, first_pass, passes, first_pass, false, capacity, keys0,
                                               vals0, keys1, vals1, desc + (unsigned long long)first_pass * desc_stride,
                                               desc_stride, ctrl, which, after_hist, count);
}

cudaError_t launch_radix_sort32(cudaStream_t st, const StepParams* sp, int digits, int slot_base, bool hist_done,
                                unsigned long long capacity, unsigned* keys0, unsigned* vals0, unsigned* keys1,
                                unsigned* vals1, unsigned long long* desc, unsigned long long desc_stride,
                                Control* ctrl, int* which, cudaEvent_t after_hist, const unsigned long long* count,
                                int first_digit) {
    if (capacity >= kWideSweepKeys)
        return radix_sort_impl<unsigned, 32>(st, sp, first_digit, digits, slot_base, hist_done, capacity, keys0, vals0, keys1,
                                     vals1, desc, desc_stride, ctrl, which, after_hist, count);
    return radix_sort_impl<unsigned, kSortItems>(st, sp, first_digit, digits, slot_base, hist_done, capacity, keys0, vals0, keys1,
                                     vals1, desc, desc_stride, ctrl, which, after_hist, count);
}

cudaError_t launch_tile_ranges(cudaStream_t st, unsigned long long capacity, const unsigned long long* keys_sorted,
                               unsigned* ranges, Control* ctrl) {
    if (capacity == 0) return cudaSuccess;
    k_ranges<<<(unsigned)((capacity + 255) / 256), 256, 0, st>>>(keys_sorted, capacity, ranges, ctrl);
    return cudaGetLastError();
}

// CTAs of 256 threads for the four-keys-per-thread range kernels: enough for the
// capacity, at most 8 per SM (the kernels stride over the pairs present, which
// a step finds on the device; a grid over the whole capacity spent its time
// starting CTAs with nothing to do).
static unsigned ranges_grid(unsigned long long capacity) {
    const unsigned long long need = (capacity + 1023) / 1024, cap = 8ull * (unsigned long long)sm_count();
    return (unsigned)(need < cap ? need : cap);
}

cudaError_t launch_tile_ranges_views(cudaStream_t st, unsigned long long capacity, const unsigned* tiles_sorted,
                                     const StepParams* views, unsigned* ranges, Control* ctrl) {
    if (capacity == 0) return cudaSuccess;
    k_ranges_views4<<<ranges_grid(capacity), 256, 0, st>>>(tiles_sorted, views, capacity, ranges, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_tile_ranges32(cudaStream_t st, unsigned long long capacity, const unsigned* tiles_sorted,
                                 unsigned* ranges, Control* ctrl) {
    if (capacity == 0) return cudaSuccess;
    k_ranges32<<<ranges_grid(capacity), 256, 0, st>>>(tiles_sorted, capacity, ranges, ctrl);
    return cudaGetLastError();
}

cudaError_t launch_tile_order(cudaStream_t st, const unsigned* ranges, int num_tiles, unsigned* order,
                              Control* ctrl) {
    if (num_tiles <= 0) return cudaSuccess;
    if (num_tiles <= 65536 || !ctrl) {   // one view: a single CTA
        k_tile_order<<<1, 1024, 0, st>>>(ranges, num_tiles, order);
        return cudaGetLastError();
    }
    const int grid = (num_tiles + 1023) / 1024;
    k_tile_bucket_count<<<std::min(grid, 4 * sm_count()), 256, 0, st>>>(ranges, num_tiles, ctrl);
    k_tile_bucket_scatter<<<grid, 256, 0, st>>>(ranges, num_tiles, ctrl, order);
    return cudaGetLastError();
}

}  // namespace gs3d
