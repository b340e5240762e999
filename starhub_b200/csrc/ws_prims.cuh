// Deterministic scan and stable LSD radix sort with device-resident counts.
//
// Every launch is sized from a host-known capacity and reads the live element
// count from device memory, so the index build needs no host synchronisation
// and can be captured in a CUDA graph.  The sort is stable (equal keys keep
// their input order), which is what the reference's cub::DeviceRadixSort
// calls rely on (libs/star/common/algorithm_types.cuh:37-83).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace ws {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;   // 4096 keys per tile
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;    // 2048 elements per tile

__device__ __forceinline__ uint32_t warp_incl_scan_u32(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024, multiple of 32).
__device__ __forceinline__ uint32_t block_excl_scan_u32(uint32_t v, uint32_t *total, uint32_t *smem32) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t inc = warp_incl_scan_u32(v);
    __syncthreads();
    if (lane == 31) smem32[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? smem32[lane] : 0u;
        w = warp_incl_scan_u32(w);
        if (lane < nw) smem32[lane] = w;
    }
    __syncthreads();
    const uint32_t warp_off = warp > 0 ? smem32[warp - 1] : 0u;
    if (total) *total = smem32[nw - 1];
    return warp_off + inc - v;
}

// ---------------------------------------------------------------------------
// Exclusive scan: out[i] = sum_{j<i} in[i]; out[n] = total.  n read from n_dev
// (or n_static when n_dev is null).  Three launches: tile sums, scan of tile
// sums (one block), tile scans.
// ---------------------------------------------------------------------------
static __global__ void k_scan_tile_sums(const uint32_t *in, const uint32_t *n_dev, uint32_t n_static, uint32_t *tile_sums) {
    __shared__ uint32_t sm[32];
    const uint32_t n = n_dev ? *n_dev : n_static;
    const uint32_t base = blockIdx.x * kScanTile;
    uint32_t s = 0;
    if (base < n) {
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            const uint32_t idx = base + threadIdx.x * kScanItems + i;
            if (idx < n) s += in[idx];
        }
    }
    uint32_t total;
    block_excl_scan_u32(s, &total, sm);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Tiles past the live count hold zero sums; only the used ones are scanned, and the total
// goes to tile_sums[num_tiles].
static __global__ void k_scan_tile_offsets(uint32_t *tile_sums, int num_tiles, const uint32_t *n_dev,
                                           uint32_t n_static) {
    __shared__ uint32_t sm[32];
    __shared__ uint32_t carry;
    const uint32_t n = n_dev ? *n_dev : n_static;
    const int used = min(num_tiles, (int)(n / kScanTile) + 1);
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < used; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const uint32_t v = i < used ? tile_sums[i] : 0u;
        uint32_t total;
        const uint32_t ex = block_excl_scan_u32(v, &total, sm);
        if (i < used) tile_sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) tile_sums[num_tiles] = carry;
}

static __global__ void k_scan_apply(const uint32_t *in, const uint32_t *n_dev, uint32_t n_static,
                             const uint32_t *tile_offsets, int num_tiles, uint32_t *out) {
    __shared__ uint32_t sm[32];
    const uint32_t n = n_dev ? *n_dev : n_static;
    const uint32_t base = blockIdx.x * kScanTile;
    if (base > n) return;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t idx = base + threadIdx.x * kScanItems + i;
        v[i] = idx < n ? in[idx] : 0u;
        s += v[i];
    }
    uint32_t ex = block_excl_scan_u32(s, nullptr, sm) + tile_offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t idx = base + threadIdx.x * kScanItems + i;
        if (idx < n) out[idx] = ex;
        ex += v[i];
    }
    if (base <= n && n < base + kScanTile && threadIdx.x == 0) out[n] = tile_offsets[num_tiles];
}

// Host driver.  `in` and `out` may alias.  tile_sums needs cap/2048 + 2 entries.
inline void exclusive_scan(const uint32_t *in, uint32_t *out, const uint32_t *n_dev, uint32_t n_static,
                           uint32_t cap, uint32_t *tile_sums, cudaStream_t st) {
    const int tiles = (int)((cap + kScanTile) / kScanTile);
    k_scan_tile_sums<<<tiles, kScanThreads, 0, st>>>(in, n_dev, n_static, tile_sums);
    k_scan_tile_offsets<<<1, 1024, 0, st>>>(tile_sums, tiles, n_dev, n_static);
    k_scan_apply<<<tiles, kScanThreads, 0, st>>>(in, n_dev, n_static, tile_sums, tiles, out);
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (key, u32 value), D = 8 or 9 bits per pass (256 or 512 digits; each
// thread of a 256-thread block looks after one or two of them).
// hist layout: hist[digit * max_tiles + tile].
// ---------------------------------------------------------------------------
template <class K, int D>
__global__ void k_radix_upsweep(const K *keys, const uint32_t *n_dev, uint32_t n_static, int shift,
                                uint32_t *hist, int max_tiles) {
    constexpr uint32_t kDigits = 1u << D;
    __shared__ uint32_t h[kDigits];
    const uint32_t n = n_dev ? *n_dev : n_static;
    for (uint32_t d = threadIdx.x; d < kDigits; d += kSortThreads) h[d] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * (uint32_t)kSortTile;
    if (base < n) {
#pragma unroll 4
        for (int r = 0; r < kSortRounds; ++r) {
            const uint32_t idx = base + r * kSortThreads + threadIdx.x;
            if (idx < n) atomicAdd(&h[(uint32_t)(keys[idx] >> shift) & (kDigits - 1u)], 1u);
        }
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < kDigits; d += kSortThreads) hist[(size_t)d * max_tiles + blockIdx.x] = h[d];
}

// Exclusive scan of one digit's tile counts (one block per digit) over the tiles in use,
// 1024 consecutive counts per pass (4 per thread), with the running total carried along.
static __global__ void k_radix_scan(uint32_t *hist, int max_tiles, const uint32_t *n_dev, uint32_t n_static,
                                    uint32_t *digit_total) {
    __shared__ uint32_t sm[32];
    const uint32_t n = n_dev ? *n_dev : n_static;
    const int used = min(max_tiles, (int)((n + kSortTile - 1) / kSortTile));
    uint32_t *row = hist + (size_t)blockIdx.x * max_tiles;
    uint32_t carry = 0;
    for (int base = 0; base < used; base += 4 * (int)blockDim.x) {
        const int i0 = base + 4 * (int)threadIdx.x;
        uint32_t v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = (i0 + k < used) ? row[i0 + k] : 0u;
        const uint32_t local = v[0] + v[1] + v[2] + v[3];
        uint32_t total;
        uint32_t run = block_excl_scan_u32(local, &total, sm) + carry;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (i0 + k < used) row[i0 + k] = run;
            run += v[k];
        }
        carry += total;
        __syncthreads();   // sm is reused by the next pass's scan
    }
    if (threadIdx.x == 0) digit_total[blockIdx.x] = carry;
}

template <class K, int D>
__global__ void __launch_bounds__(kSortThreads)
k_radix_scatter(const K *keys_in, const uint32_t *vals_in, K *keys_out, uint32_t *vals_out,
                const uint32_t *n_dev, uint32_t n_static, int shift,
                const uint32_t *hist, int max_tiles, const uint32_t *digit_total) {
    constexpr uint32_t kDigits = 1u << D;
    constexpr int kPer = (int)kDigits / kSortThreads;   // digits per thread
    static_assert(kPer == 1 || kPer == 2, "8- or 9-bit digits");
    __shared__ uint32_t digit_base[kDigits];
    __shared__ uint32_t run[kDigits];
    __shared__ uint16_t wcount[kSortThreads / 32][kDigits];
    __shared__ uint32_t sm[32];
    const uint32_t n = n_dev ? *n_dev : n_static;
    const uint32_t base = blockIdx.x * (uint32_t)kSortTile;
    if (base >= n) return;                      // uniform for the whole block
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    {
        // thread t owns digits kPer t .. kPer t + kPer - 1
        uint32_t tot[kPer], sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            tot[k] = digit_total[kPer * t + k];
            sum += tot[k];
        }
        uint32_t ex = block_excl_scan_u32(sum, nullptr, sm);
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            const uint32_t d = (uint32_t)(kPer * t + k);
            digit_base[d] = ex + hist[(size_t)d * max_tiles + blockIdx.x];
            run[d] = 0;
            ex += tot[k];
        }
    }
    for (int r = 0; r < kSortRounds; ++r) {
        const uint32_t idx = base + r * kSortThreads + t;
        const bool valid = idx < n;
        K key = 0;
        uint32_t val = 0;
        uint32_t d = kDigits;
        if (valid) {
            key = keys_in[idx];
            val = vals_in[idx];
            d = (uint32_t)(key >> shift) & (kDigits - 1u);
        }
        __syncthreads();
#pragma unroll
        for (int w = 0; w < kSortThreads / 32; ++w)
#pragma unroll
            for (int k = 0; k < kPer; ++k) wcount[w][kPer * t + k] = 0;
        __syncthreads();
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank_w = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank_w == 0) wcount[warp][d] = (uint16_t)__popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t pre = 0;
            for (int w = 0; w < warp; ++w) pre += wcount[w][d];
            const uint32_t pos = digit_base[d] + run[d] + pre + (uint32_t)rank_w;
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            uint32_t tot = 0;
#pragma unroll
            for (int w = 0; w < kSortThreads / 32; ++w) tot += wcount[w][kPer * t + k];
            run[kPer * t + k] += tot;
        }
        if (base + (uint32_t)(r + 1) * kSortThreads >= n) break;   // uniform
    }
}

inline int sort_max_tiles(uint32_t cap) { return (int)((cap + kSortTile - 1) / kSortTile) + 1; }
constexpr int kSortMaxDigits = 512;

// Sorts `bits` low bits of the keys, 9 bits per pass when that saves a pass over 8 bits.
// Buffers a/b ping-pong; returns true when the result ended in the `alt` buffers.  hist needs
// kSortMaxDigits * sort_max_tiles(cap) entries, digit_total kSortMaxDigits.
template <class K>
inline bool radix_sort(K *keys, uint32_t *vals, K *keys_alt, uint32_t *vals_alt,
                       const uint32_t *n_dev, uint32_t n_static, uint32_t cap, int bits,
                       uint32_t *hist, uint32_t *digit_total, cudaStream_t st) {
    const int max_tiles = sort_max_tiles(cap);
    const int step = ((bits + 8) / 9 < (bits + 7) / 8) ? 9 : 8;
    bool in_alt = false;
    for (int shift = 0; shift < bits; shift += step) {
        K *ki = in_alt ? keys_alt : keys;
        uint32_t *vi = in_alt ? vals_alt : vals;
        K *ko = in_alt ? keys : keys_alt;
        uint32_t *vo = in_alt ? vals : vals_alt;
        if (step == 9) {
            k_radix_upsweep<K, 9><<<max_tiles, kSortThreads, 0, st>>>(ki, n_dev, n_static, shift, hist, max_tiles);
            k_radix_scan<<<512, 256, 0, st>>>(hist, max_tiles, n_dev, n_static, digit_total);
            k_radix_scatter<K, 9><<<max_tiles, kSortThreads, 0, st>>>(ki, vi, ko, vo, n_dev, n_static, shift, hist,
                                                                       max_tiles, digit_total);
        } else {
            k_radix_upsweep<K, 8><<<max_tiles, kSortThreads, 0, st>>>(ki, n_dev, n_static, shift, hist, max_tiles);
            k_radix_scan<<<256, 256, 0, st>>>(hist, max_tiles, n_dev, n_static, digit_total);
            k_radix_scatter<K, 8><<<max_tiles, kSortThreads, 0, st>>>(ki, vi, ko, vo, n_dev, n_static, shift, hist,
                                                                       max_tiles, digit_total);
        }
        in_alt = !in_alt;
    }
    return in_alt;
}

// Radix passes of radix_sort for `bits` key bits.
inline int radix_passes(int bits) { return std::min((bits + 8) / 9, (bits + 7) / 8); }

inline int bits_for(uint64_t max_value) {
    int b = 1;
    while (b < 64 && (max_value >> b) != 0) ++b;
    return b;
}

}  // namespace ws
