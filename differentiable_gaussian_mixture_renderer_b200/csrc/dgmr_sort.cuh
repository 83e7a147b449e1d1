// Device-wide building blocks of the binning stage: an inclusive scan of u32
// counts and a stable LSD radix sort of (u32 key, u32 value) pairs.  Both
// read the element count from device memory (so a frame needs no host
// round trip between its preprocess and its sort) and bound it by the
// capacity the buffers were sized for.
//
// They replace the reference's cub::DeviceScan::InclusiveSum and
// cub::DeviceRadixSort::SortPairs (splat_forward.cu:187-202, :256-274).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dgmr_launch_count.h"

namespace dgmr {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItemsPerThread = 8;
constexpr int kSortTile = kSortThreads * kSortItemsPerThread; // 2048 items per tile
constexpr int kSortBins = 256; // 8-bit digits

// Guards on data-dependent indices: a violated guard skips the access, sets
// bit 2 of the frame flags and records the first site's code in stats[3].
constexpr uint32_t kFlagBounds = 4u;
__device__ __forceinline__ void flag_bounds(uint32_t* stats, uint32_t site)
{
    if (stats) {
        atomicOr(&stats[1], kFlagBounds);
        atomicCAS(&stats[3], 0u, site);
    }
}

__device__ __forceinline__ uint32_t dev_count(const uint32_t* n_dev, uint32_t n_static, uint32_t capacity)
{
    const uint32_t n = n_dev ? *n_dev : n_static;
    return n < capacity ? n : capacity;
}

// ---------------------------------------------------------------- scan
// per-tile sums of `in` (tile = kSortTile items)
static __global__ void k_scan_tile_sums(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ tile_sums)
{
    __shared__ uint32_t warp_sums[kSortWarps];
    const uint32_t tile = blockIdx.x;
    const uint32_t base = tile * kSortTile;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kSortItemsPerThread; ++i) {
        const uint32_t idx = base + i * kSortThreads + threadIdx.x;
        if (idx < n)
            s += in[idx];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        warp_sums[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kSortWarps; ++w)
            t += warp_sums[w];
        tile_sums[tile] = t;
    }
}

// exclusive scan of the tile sums in one block (tile counts are small)
static __global__ void k_scan_tile_offsets(uint32_t* __restrict__ tile_sums, uint32_t n_tiles)
{
    __shared__ uint32_t carry;
    __shared__ uint32_t warp_tot[32];
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n_tiles; base += blockDim.x) {
        const uint32_t idx = base + threadIdx.x;
        const uint32_t v = idx < n_tiles ? tile_sums[idx] : 0;
        uint32_t x = v;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o)
                x += y;
        }
        if (lane == 31)
            warp_tot[warp] = x;
        __syncthreads();
        if (warp == 0) {
            const int nw = blockDim.x / 32;
            uint32_t t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o)
                    t += y;
            }
            if (lane < nw)
                warp_tot[lane] = t; // inclusive over warps
        }
        __syncthreads();
        const uint32_t warp_excl = warp == 0 ? 0 : warp_tot[warp - 1];
        const uint32_t excl = carry + warp_excl + x - v;
        if (idx < n_tiles)
            tile_sums[idx] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1)
            carry = excl + v;
        __syncthreads();
    }
}

// inclusive scan within each tile plus the tile's offset
static __global__ void k_scan_apply(const uint32_t* __restrict__ in, uint32_t n, const uint32_t* __restrict__ tile_offsets, uint32_t* __restrict__ out)
{
    __shared__ uint32_t warp_tot[kSortWarps];
    __shared__ uint32_t carry;
    const uint32_t tile = blockIdx.x;
    const uint32_t base = tile * kSortTile;
    if (threadIdx.x == 0)
        carry = tile_offsets[tile];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = 0; i < kSortItemsPerThread; ++i) {
        const uint32_t idx = base + i * kSortThreads + threadIdx.x;
        const uint32_t v = idx < n ? in[idx] : 0;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o)
                x += y;
        }
        if (lane == 31)
            warp_tot[warp] = x;
        __syncthreads();
        uint32_t wex = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t t = warp_tot[w];
            wex += (w < warp) ? t : 0;
            tot += t;
        }
        if (idx < n)
            out[idx] = carry + wex + x;
        __syncthreads();
        if (threadIdx.x == 0)
            carry += tot;
        __syncthreads();
    }
}

// ---------------------------------------------------------------- radix sort
// Histogram of one digit per tile: hist[d * tile_stride + tile].
// Key rebasing for a sort whose keys span a narrow range: range = {min, max}
// over the keys that matter (live[i] != 0), or min > max when none does.  The
// first pass replaces every key by key - min (a dead key by max - min) before
// counting it; any pass whose digit is then zero for every key only copies.
// The order of the live keys is unchanged (equal keys stay equal, the stable
// passes keep their input order), so the sorted positions of the live items
// are those of the full 32-bit sort.
__device__ __forceinline__ bool range_rebases(const uint32_t* range) { return range && range[0] <= range[1]; }
__device__ __forceinline__ bool pass_is_copy(const uint32_t* range, int shift)
{
    return range_rebases(range) && ((range[1] - range[0]) >> shift) == 0u;
}

// min / max of the live keys into range (initialised to {~0, 0})
static __global__ void k_key_range(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ live, uint32_t n, uint32_t* __restrict__ range)
{
    uint32_t lo = 0xffffffffu, hi = 0u;
    // four items per thread and step, every load issued before the first is used
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 4u * stride) {
        uint32_t kv[4], lv[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t i = i0 + uint32_t(r) * stride;
            kv[r] = i < n ? keys[i] : 0u;
            lv[r] = i < n ? live[i] : 0u;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (lv[r]) {
                lo = kv[r] < lo ? kv[r] : lo;
                hi = kv[r] > hi ? kv[r] : hi;
            }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    // one pair of atomics per block (per warp, they serialised on two addresses)
    __shared__ uint32_t s_lo[32], s_hi[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = int(blockDim.x >> 5);
    if (lane == 0) {
        s_lo[warp] = lo;
        s_hi[warp] = hi;
    }
    __syncthreads();
    if (warp == 0) {
        lo = lane < n_warps ? s_lo[lane] : 0xffffffffu;
        hi = lane < n_warps ? s_hi[lane] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0 && lo <= hi) {
            atomicMin(&range[0], lo);
            atomicMax(&range[1], hi);
        }
    }
}

static __global__ void k_radix_hist(uint32_t* __restrict__ keys, const uint32_t* n_dev, uint32_t n_static, uint32_t capacity, int shift, uint32_t mask,
    uint32_t* __restrict__ hist, uint32_t tile_stride, const uint32_t* __restrict__ range, const uint32_t* __restrict__ live, bool rebase)
{
    __shared__ uint32_t h[kSortWarps][kSortBins];
    if (pass_is_copy(range, shift))
        return;
    const bool rb = rebase && range_rebases(range);
    const uint32_t kmin = rb ? range[0] : 0u, kspan = rb ? range[1] - range[0] : 0u;
    const uint32_t n = dev_count(n_dev, n_static, capacity);
    const uint32_t n_tiles = (n + kSortTile - 1) / kSortTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        for (int i = threadIdx.x; i < kSortWarps * kSortBins; i += kSortThreads)
            (&h[0][0])[i] = 0;
        __syncthreads();
        const uint32_t base = tile * kSortTile + warp * (kSortTile / kSortWarps);
        // the tile's keys (and live flags) are all requested before the first
        // is used, so their latencies overlap; per-warp histograms keep
        // shared-memory atomic contention inside one warp
        uint32_t kv[kSortItemsPerThread], lv[kSortItemsPerThread];
#pragma unroll
        for (int r = 0; r < kSortItemsPerThread; ++r) {
            const uint32_t idx = base + r * 32 + lane;
            kv[r] = idx < n ? keys[idx] : 0u;
            lv[r] = (rb && idx < n) ? live[idx] : 0u;
        }
#pragma unroll
        for (int r = 0; r < kSortItemsPerThread; ++r) {
            const uint32_t idx = base + r * 32 + lane;
            if (idx < n) {
                uint32_t k = kv[r];
                if (rb) {
                    k = lv[r] ? k - kmin : kspan;
                    keys[idx] = k;
                }
                atomicAdd(&h[warp][(k >> shift) & mask], 1u);
            }
        }
        __syncthreads();
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w)
            t += h[w][threadIdx.x];
        hist[threadIdx.x * tile_stride + tile] = t;
        __syncthreads();
    }
}

// Exclusive scan of each digit's row over tiles; row totals to digit_total.
static __global__ void k_radix_scan_rows(uint32_t* __restrict__ hist, const uint32_t* n_dev, uint32_t n_static, uint32_t capacity, uint32_t tile_stride,
    uint32_t* __restrict__ digit_total, const uint32_t* __restrict__ range, int shift)
{
    __shared__ uint32_t warp_tot[kSortWarps];
    __shared__ uint32_t carry;
    if (pass_is_copy(range, shift))
        return;
    const uint32_t n = dev_count(n_dev, n_static, capacity);
    const uint32_t n_tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* row = hist + size_t(blockIdx.x) * tile_stride;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t b = 0; b < n_tiles; b += kSortThreads) {
        const uint32_t idx = b + threadIdx.x;
        const uint32_t v = idx < n_tiles ? row[idx] : 0;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o)
                x += y;
        }
        if (lane == 31)
            warp_tot[warp] = x;
        __syncthreads();
        uint32_t wex = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t t = warp_tot[w];
            wex += (w < warp) ? t : 0;
            tot += t;
        }
        if (idx < n_tiles)
            row[idx] = carry + wex + x - v;
        __syncthreads();
        if (threadIdx.x == 0)
            carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        digit_total[blockIdx.x] = carry;
}

// Lanes of the warp holding the same digit as this lane (a digit of at most
// 8 bits; lanes without an item match each other only): one ballot per digit
// bit, on the ALU pipe, instead of __match_any_sync.
__device__ __forceinline__ uint32_t warp_same_digit(uint32_t d, bool valid, uint32_t mask)
{
    const uint32_t v = __ballot_sync(0xffffffffu, valid);
    uint32_t peers = valid ? v : ~v;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        if (!((mask >> b) & 1u))
            break; // mask is 2^bits - 1, the same on every lane
        const bool one = valid && ((d >> b) & 1u);
        const uint32_t ones = __ballot_sync(0xffffffffu, one);
        peers &= one ? ones : ~ones;
    }
    return peers;
}

// Stable scatter: warp w of a tile owns a contiguous 256-item slice and ranks
// its items in order (warp_same_digit's ballots), so equal digits keep input order.
// The tile is first rearranged in shared memory into digit order, then written
// out so that consecutive threads store consecutive addresses of each digit's
// run (coalesced), instead of every lane storing into a different bucket.
static __global__ void __launch_bounds__(256) k_radix_scatter(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, const uint32_t* n_dev, uint32_t n_static, uint32_t capacity, int shift, uint32_t mask,
    const uint32_t* __restrict__ hist, uint32_t tile_stride, const uint32_t* __restrict__ digit_total, uint32_t* __restrict__ stats,
    const uint32_t* __restrict__ range)
{
    __shared__ uint32_t wcount[kSortWarps][kSortBins];
    __shared__ uint32_t gbase[kSortBins]; // global start of this tile's run of each digit
    __shared__ uint32_t lbase[kSortBins]; // start of each digit's run inside the tile
    __shared__ uint32_t dbase[kSortBins];
    __shared__ uint32_t warp_tot[kSortWarps];
    __shared__ uint32_t s_key[kSortTile];
    __shared__ uint32_t s_val[kSortTile];
    const uint32_t n = dev_count(n_dev, n_static, capacity);
    if (pass_is_copy(range, shift)) {
        // every key has digit 0 here and in every later pass: the order stays and
        // no later pass reads the keys, so only the values move (eight loads in
        // flight per thread before the stores)
        const uint32_t stride = gridDim.x * blockDim.x;
        for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 8u * stride) {
            uint32_t v[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const uint32_t i = i0 + uint32_t(r) * stride;
                v[r] = i < n ? vals_in[i] : 0u;
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const uint32_t i = i0 + uint32_t(r) * stride;
                if (i < n)
                    vals_out[i] = v[r];
            }
        }
        return;
    }
    const uint32_t n_tiles = (n + kSortTile - 1) / kSortTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;

    // block-wide exclusive scan of one value per thread (256 threads)
    const auto block_excl_scan = [&](uint32_t v) -> uint32_t {
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o)
                x += y;
        }
        if (lane == 31)
            warp_tot[warp] = x;
        __syncthreads();
        uint32_t wex = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w)
            wex += (w < warp) ? warp_tot[w] : 0;
        __syncthreads();
        return wex + x - v;
    };

    dbase[threadIdx.x] = block_excl_scan(digit_total[threadIdx.x]);
    __syncthreads();

    for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        // every global load of the tile is issued before the first is used:
        // this tile's start of digit threadIdx.x, then the keys and values
        const uint32_t hrow = hist[threadIdx.x * tile_stride + tile];
        const uint32_t tile_base = tile * kSortTile;
        const uint32_t base = tile_base + warp * (kSortTile / kSortWarps);
        uint32_t k[kSortItemsPerThread], v[kSortItemsPerThread], rank[kSortItemsPerThread];
#pragma unroll
        for (int r = 0; r < kSortItemsPerThread; ++r) {
            const uint32_t idx = base + r * 32 + lane;
            k[r] = idx < n ? keys_in[idx] : 0u;
            v[r] = idx < n ? vals_in[idx] : 0u;
        }
        for (int i = threadIdx.x; i < kSortWarps * kSortBins; i += kSortThreads)
            (&wcount[0][0])[i] = 0;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kSortItemsPerThread; ++r) {
            const uint32_t idx = base + r * 32 + lane;
            const bool valid = idx < n;
            const uint32_t d = valid ? ((k[r] >> shift) & mask) : 0xffffffffu;
            const uint32_t peers = warp_same_digit(d, valid, mask);
            rank[r] = (valid ? wcount[warp][d] : 0u) + __popc(peers & lt_mask);
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1)
                wcount[warp][d] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // per digit: prefix over warps (in place) and the tile's count of that digit
        uint32_t count = 0;
        {
            const uint32_t d = threadIdx.x;
#pragma unroll
            for (int w = 0; w < kSortWarps; ++w) {
                const uint32_t t = wcount[w][d];
                wcount[w][d] = count;
                count += t;
            }
            gbase[d] = dbase[d] + hrow;
        }
        lbase[threadIdx.x] = block_excl_scan(count);
        __syncthreads();
        // digit-ordered staging in shared memory
#pragma unroll
        for (int r = 0; r < kSortItemsPerThread; ++r) {
            const uint32_t idx = base + r * 32 + lane;
            if (idx < n) {
                const uint32_t d = (k[r] >> shift) & mask;
                const uint32_t lpos = lbase[d] + wcount[warp][d] + rank[r];
                s_key[lpos] = k[r];
                s_val[lpos] = v[r];
            }
        }
        __syncthreads();
        const uint32_t in_tile = (n - tile_base) < uint32_t(kSortTile) ? (n - tile_base) : uint32_t(kSortTile);
        for (uint32_t i = threadIdx.x; i < in_tile; i += kSortThreads) {
            const uint32_t key = s_key[i];
            const uint32_t d = (key >> shift) & mask;
            const uint32_t pos = gbase[d] + (i - lbase[d]);
            if (pos < n) {
                keys_out[pos] = key;
                vals_out[pos] = s_val[i];
            } else {
                flag_bounds(stats, 0x11u);
            }
        }
        __syncthreads();
    }
}

// Temporary storage for sort_pairs over at most `capacity` items.
inline size_t radix_temp_bytes(uint32_t capacity)
{
    const size_t tiles = (size_t(capacity) + kSortTile - 1) / kSortTile;
    return (size_t(kSortBins) * (tiles + 1) + kSortBins) * sizeof(uint32_t);
}

// Stable sort of (keys, vals) by key bits [begin_bit, end_bit).  The data
// ping-pongs between (k0, v0) and (k1, v1); returns 0 if the result is in
// k0/v0, 1 if in k1/v1.  n comes from *n_dev (device) when non-null, else
// n_static.  With range / live (see k_key_range) the keys are rebased in place
// by the first pass and passes over all-zero digits copy the values only; the
// sorted keys are then not produced (only the values' order is).
inline int radix_sort_pairs(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, const uint32_t* n_dev, uint32_t n_static, uint32_t capacity, int end_bit,
    void* temp, int n_sms, cudaStream_t stream, uint32_t* stats = nullptr, int begin_bit = 0, const uint32_t* range = nullptr,
    const uint32_t* live = nullptr)
{
    const uint32_t tiles = (capacity + kSortTile - 1) / kSortTile;
    if (tiles == 0)
        return 0;
    const uint32_t stride = tiles + 1;
    uint32_t* hist = static_cast<uint32_t*>(temp);
    uint32_t* dtotal = hist + size_t(kSortBins) * stride;
    const uint32_t grid = tiles < uint32_t(n_sms * 8) ? tiles : uint32_t(n_sms * 8);
    int cur = 0;
    // fewest 8-bit-or-narrower passes, with the bits spread evenly over them
    // (e.g. 13 tile bits -> 7 + 6): fewer buckets per pass keep the runs each
    // tile writes per digit longer
    const int n_pass = (end_bit - begin_bit + 7) / 8;
    const int width = n_pass ? (end_bit - begin_bit + n_pass - 1) / n_pass : 8;
    for (int shift = begin_bit; shift < end_bit; shift += width) {
        const int bits = (end_bit - shift) < width ? (end_bit - shift) : width;
        const uint32_t mask = (1u << bits) - 1u;
        uint32_t* ki = cur ? k1 : k0;
        uint32_t* vi = cur ? v1 : v0;
        uint32_t* ko = cur ? k0 : k1;
        uint32_t* vo = cur ? v0 : v1;
        k_radix_hist<<<grid, kSortThreads, 0, stream>>>(ki, n_dev, n_static, capacity, shift, mask, hist, stride, range, live, shift == begin_bit);
        k_radix_scan_rows<<<kSortBins, kSortThreads, 0, stream>>>(hist, n_dev, n_static, capacity, stride, dtotal, range, shift);
        k_radix_scatter<<<grid, kSortThreads, 0, stream>>>(ki, vi, ko, vo, n_dev, n_static, capacity, shift, mask, hist, stride, dtotal, stats, range);
        note_launch(3);
        cur ^= 1;
    }
    return cur;
}

// inclusive scan of n <= 32 * 1024 u32 in one block (one launch instead of
// three for short arrays): thread t owns a contiguous run of ceil(n / 1024)
// items, sums it, the 1024 sums are scanned once, then each run is written.
constexpr uint32_t kScanSingleMax = 32u * 1024u;
static __global__ void __launch_bounds__(1024) k_scan_single(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ out)
{
    __shared__ uint32_t warp_tot[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t per = (n + 1023u) / 1024u;
    const uint32_t b = threadIdx.x * per, e = b + per < n ? b + per : n;
    uint32_t v = 0;
    for (uint32_t i = b; i < e; ++i)
        v += in[i];
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        warp_tot[warp] = x;
    __syncthreads();
    uint32_t run = x - v;
    for (int w = 0; w < warp; ++w)
        run += warp_tot[w];
    for (uint32_t i = b; i < e; ++i) {
        run += in[i];
        out[i] = run;
    }
}

inline size_t scan_temp_bytes(uint32_t n) { return ((size_t(n) + kSortTile - 1) / kSortTile + 1) * sizeof(uint32_t); }

// inclusive scan of n u32 (n known on the host)
inline void inclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, void* temp, cudaStream_t stream)
{
    if (n == 0)
        return;
    const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* sums = static_cast<uint32_t*>(temp);
    k_scan_tile_sums<<<tiles, kSortThreads, 0, stream>>>(in, n, sums);
    k_scan_tile_offsets<<<1, 1024, 0, stream>>>(sums, tiles);
    k_scan_apply<<<tiles, kSortThreads, 0, stream>>>(in, n, sums, out);
    note_launch(3);
}

} // namespace dgmr
