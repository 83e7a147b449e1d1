// Tile binning shared by the splat renderer and the volume marcher.
//
// The reference emits one 64-bit key (tile << 32 | float bits of depth) per
// (tile, Gaussian) pair and radix-sorts all pairs over 32 + msb(tiles) bits
// (splat_forward.cu:159-211).  The sorted order it produces is the order of
// (tile, depth bits, Gaussian index).  Here the same order is reached with
// far less traffic: the N Gaussians are stably sorted once by their 32-bit
// depth bits (N << pairs), pairs are emitted in that depth order, and a
// stable sort over only the msb(tiles) tile bits finishes the job.  The
// result -- point list and tile ranges -- is identical bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dgmr_device_math.cuh"
#include "dgmr_sort.cuh"

namespace dgmr {

// util.h:56-70: next-highest bit of the MSB
inline uint32_t higher_msb(uint32_t n)
{
    uint32_t msb = sizeof(n) * 4;
    uint32_t step = msb;
    while (step > 1) {
        step /= 2;
        if (n >> msb)
            msb += step;
        else
            msb -= step;
    }
    if (n >> msb)
        msb++;
    return msb;
}

inline size_t align_up(size_t v, size_t a = 256) { return (v + a - 1) / a * a; }

// Linear workspace carving with 256-byte alignment.
struct Carver {
    size_t off = 0;
    char* base = nullptr;
    template <class P>
    P* take(size_t count)
    {
        const size_t o = off;
        off = align_up(off + count * sizeof(P));
        return base ? reinterpret_cast<P*>(base + o) : nullptr;
    }
};

// Scratch of the binning stage.
struct BinningBuffers {
    uint32_t* depth_key; // [N]
    uint32_t* perm; // [N]  (holds iota on entry, the depth order on exit)
    uint32_t* key_tmp; // [N]
    uint32_t* perm_tmp; // [N]
    uint32_t* cnt_sorted; // [N]
    uint32_t* off_sorted; // [N]
    uint32_t* pair_tile[2]; // [cap]
    uint32_t* pair_val[2]; // [cap]
    uint32_t* scan_tmp; // scan_temp_bytes(N)
    void* sort_tmp; // radix_temp_bytes(max(N, cap))
    uint32_t* n_sort; // [1] pairs to sort = min(P, cap)
};

// the parts sized by the Gaussian count
inline void carve_binning_gaussians(Carver& c, BinningBuffers& b, uint32_t N)
{
    b.depth_key = c.take<uint32_t>(N);
    b.perm = c.take<uint32_t>(N);
    b.key_tmp = c.take<uint32_t>(N);
    b.perm_tmp = c.take<uint32_t>(N);
    b.cnt_sorted = c.take<uint32_t>(N);
    b.off_sorted = c.take<uint32_t>(N);
    b.scan_tmp = c.take<uint32_t>(scan_temp_bytes(N) / 4 + 1);
    b.n_sort = c.take<uint32_t>(4);
}

// the parts sized by the pair capacity (and the sort scratch)
inline void carve_binning_pairs(Carver& c, BinningBuffers& b, uint32_t N, uint32_t cap)
{
    for (int i = 0; i < 2; ++i) {
        b.pair_tile[i] = c.take<uint32_t>(cap);
        b.pair_val[i] = c.take<uint32_t>(cap);
    }
    b.sort_tmp = c.take<char>(radix_temp_bytes(N > cap ? N : cap));
}

inline void carve_binning(Carver& c, BinningBuffers& b, uint32_t N, uint32_t cap)
{
    carve_binning_gaussians(c, b, N);
    carve_binning_pairs(c, b, N, cap);
}

// parity of the buffer that holds the tile-sorted pairs
inline int tile_sort_parity(uint32_t n_tiles)
{
    const int bits = int(higher_msb(n_tiles));
    return ((bits + 7) / 8) & 1;
}

static __global__ void k_pair_count(const uint32_t* __restrict__ point_offsets, uint32_t N, uint32_t cap, uint32_t* __restrict__ stats, uint32_t* __restrict__ n_sort)
{
    const uint32_t P = N ? point_offsets[N - 1] : 0u;
    stats[0] = P;
    if (P > cap)
        atomicOr(&stats[1], 1u);
    *n_sort = P < cap ? P : cap;
}

static __global__ void k_gather_counts(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ tiles_touched, uint32_t N, uint32_t* __restrict__ cnt_sorted,
    uint32_t* __restrict__ stats)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < N) {
        const uint32_t g = perm[j];
        if (g < N) {
            cnt_sorted[j] = tiles_touched[g];
        } else {
            cnt_sorted[j] = 0;
            flag_bounds(stats, 0x21u);
        }
    }
}

// Tile grid of the frame a Gaussian slot belongs to: its size and the offset
// of its first tile in the (possibly multi-frame) tile numbering.
struct TileGrid {
    unsigned gx, gy, off;
};

// One frame: every slot uses the same grid.
struct SingleGrid {
    unsigned gx, gy;
    __device__ __forceinline__ TileGrid grid(uint32_t) const { return TileGrid { gx, gy, 0u }; }
};

// Pairs in depth order: for the j-th Gaussian by depth, one entry per tile
// its rectangle touches, row-major (util.h:42-52 applied to the cached rect
// and centroid).  The 32 Gaussians of a warp own one contiguous output range
// (their offsets come from an inclusive scan in the same order), so the warp
// writes that range together: in each round lane l takes slot base + l and
// finds its owner -- the first lane whose inclusive end exceeds the slot -- by
// a five-step binary search over the lanes' ends, done with shuffles.
template <class T, class Grids>
static __global__ void __launch_bounds__(256) k_emit_pairs(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ cnt_sorted,
    const uint32_t* __restrict__ off_sorted, const int32_t* __restrict__ rects, const T* __restrict__ xy, uint32_t N, uint32_t cap,
    uint32_t* __restrict__ pair_tile, uint32_t* __restrict__ pair_val, uint32_t* __restrict__ stats, const __grid_constant__ Grids grids)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    if (__all_sync(0xffffffffu, j >= N))
        return;
    uint32_t c = 0, end = 0, g = 0;
    TileRect r = { 0, 0, 0, 0 };
    TileGrid tg = { 0u, 0u, 0u };
    if (j < N) {
        c = cnt_sorted[j];
        end = off_sorted[j];
        if (c > 0) {
            g = perm[j];
            if (g < N) {
                tg = grids.grid(g);
                r = get_rect(float(xy[2 * g]), float(xy[2 * g + 1]), rects[2 * g], rects[2 * g + 1], tg.gx, tg.gy);
                if ((r.x1 - r.x0) * (r.y1 - r.y0) != c) {
                    flag_bounds(stats, 0x22u);
                    r = { 0, 0, 0, 0 };
                }
            } else {
                flag_bounds(stats, 0x23u);
                g = 0;
            }
        }
    }
    const uint32_t start = end - c;
    // inclusive ends, non-decreasing across the warp; lanes past N sort last
    const uint32_t key = j < N ? end : 0xffffffffu;
    const uint32_t lo = __shfl_sync(0xffffffffu, start, 0);
    uint32_t hi = j < N ? end : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    const uint32_t rw = r.x1 - r.x0;
    for (uint32_t base = lo; base < hi; base += 32) {
        const uint32_t pos = base + lane;
        // first lane with end > pos (that lane's count is > 0 whenever pos < hi)
        int a = 0, b = 31;
#pragma unroll
        for (int it = 0; it < 5; ++it) {
            const int mid = (a + b) >> 1;
            const uint32_t m = __shfl_sync(0xffffffffu, key, mid);
            if (m > pos)
                b = mid;
            else
                a = mid + 1;
        }
        const int src = a;
        const uint32_t s_start = __shfl_sync(0xffffffffu, start, src);
        const uint32_t s_c = __shfl_sync(0xffffffffu, c, src);
        const uint32_t s_g = __shfl_sync(0xffffffffu, g, src);
        const uint32_t s_x0 = __shfl_sync(0xffffffffu, r.x0, src);
        const uint32_t s_y0 = __shfl_sync(0xffffffffu, r.y0, src);
        const uint32_t s_w = __shfl_sync(0xffffffffu, rw, src);
        const uint32_t s_gx = __shfl_sync(0xffffffffu, tg.gx, src);
        const uint32_t s_n = __shfl_sync(0xffffffffu, tg.gx * tg.gy, src);
        const uint32_t s_off = __shfl_sync(0xffffffffu, tg.off, src);
        if (pos < hi && pos < cap) {
            const uint32_t k = pos - s_start;
            const uint32_t t = (s_w && k < s_c) ? (s_y0 + k / s_w) * s_gx + s_x0 + k % s_w : 0xffffffffu;
            if (t < s_n) {
                pair_tile[pos] = s_off + t;
                pair_val[pos] = s_g;
            } else {
                pair_tile[pos] = 0;
                pair_val[pos] = 0;
                flag_bounds(stats, 0x24u);
            }
        }
    }
}

// splat_forward.cu:218-239 on the tile-sorted list (ranges zeroed beforehand)
static __global__ void k_tile_ranges(const uint32_t* __restrict__ tiles_sorted, const uint32_t* __restrict__ n_dev, int32_t* __restrict__ ranges, uint32_t n_tiles,
    uint32_t* __restrict__ stats)
{
    const uint32_t n = *n_dev;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        const uint32_t cur = tiles_sorted[idx];
        const uint32_t prev_t = idx ? tiles_sorted[idx - 1] : 0u;
        if (cur >= n_tiles || prev_t >= n_tiles) {
            flag_bounds(stats, 0x25u);
            continue;
        }
        if (idx == 0)
            ranges[2 * cur] = 0;
        else {
            const uint32_t prev = tiles_sorted[idx - 1];
            if (cur != prev) {
                ranges[2 * prev + 1] = int32_t(idx);
                ranges[2 * cur] = int32_t(idx);
            }
        }
        if (idx == n - 1)
            ranges[2 * cur + 1] = int32_t(n);
    }
}

// Launch order for the per-tile kernels: tiles bucketed by floor(log2(list
// length + 1)), longest first, so the heaviest tiles start at the head of the
// grid instead of stretching its tail.  One block; order inside a bucket is
// arbitrary (it only affects scheduling, never results).
static __global__ void __launch_bounds__(1024) k_tile_order(const int32_t* __restrict__ ranges, uint32_t n_tiles, uint32_t* __restrict__ order)
{
    __shared__ uint32_t count[33];
    __shared__ uint32_t cursor[33];
    if (threadIdx.x < 33)
        count[threadIdx.x] = 0;
    __syncthreads();
    const auto bucket = [&](uint32_t t) {
        const int32_t len = ranges[2 * t + 1] - ranges[2 * t];
        return 32u - uint32_t(32 - __clz(len > 0 ? len : 0)); // 32 - bit length: long lists -> small bucket
    };
    for (uint32_t t = threadIdx.x; t < n_tiles; t += blockDim.x)
        atomicAdd(&count[bucket(t)], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int b = 0; b < 33; ++b) {
            cursor[b] = run;
            run += count[b];
        }
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < n_tiles; t += blockDim.x)
        order[atomicAdd(&cursor[bucket(t)], 1u)] = t;
}

// Full binning: point_offsets (inclusive scan, reference order), depth sort,
// emission, tile sort and ranges.  Returns the buffer index holding the
// sorted (tile, Gaussian) pairs.  Requires b.perm = iota and b.depth_key
// filled by the preprocess.
template <class T, class Grids>
inline int run_binning_grids(uint32_t N, uint32_t n_tiles, const Grids& grids, const uint32_t* tiles_touched, uint32_t* point_offsets, const int32_t* rects,
    const T* xy, uint32_t cap, BinningBuffers& b, int32_t* ranges, uint32_t* stats, int n_sms, cudaStream_t s, bool offsets_ready)
{
    cudaMemsetAsync(ranges, 0, size_t(n_tiles) * 2 * sizeof(int32_t), s);
    if (N == 0) {
        cudaMemsetAsync(b.n_sort, 0, sizeof(uint32_t), s);
        return tile_sort_parity(n_tiles);
    }
    if (!offsets_ready) {
        inclusive_scan_u32(tiles_touched, point_offsets, N, b.scan_tmp, s);
        k_pair_count<<<1, 1, 0, s>>>(point_offsets, N, cap, stats, b.n_sort);
        note_launch();
    } else {
        k_pair_count<<<1, 1, 0, s>>>(point_offsets, N, cap, stats, b.n_sort);
        note_launch();
    }
    const int dpar = radix_sort_pairs(b.depth_key, b.perm, b.key_tmp, b.perm_tmp, nullptr, N, N, 32, b.sort_tmp, n_sms, s, stats);
    const uint32_t* perm = dpar ? b.perm_tmp : b.perm;
    const uint32_t blocks = (N + 255) / 256;
    k_gather_counts<<<blocks, 256, 0, s>>>(perm, tiles_touched, N, b.cnt_sorted, stats);
    note_launch();
    inclusive_scan_u32(b.cnt_sorted, b.off_sorted, N, b.scan_tmp, s);
    k_emit_pairs<T, Grids><<<blocks, 256, 0, s>>>(perm, b.cnt_sorted, b.off_sorted, rects, xy, N, cap, b.pair_tile[0], b.pair_val[0], stats, grids);
    note_launch();
    const int bits = int(higher_msb(n_tiles));
    const int par = radix_sort_pairs(b.pair_tile[0], b.pair_val[0], b.pair_tile[1], b.pair_val[1], b.n_sort, 0, cap, bits, b.sort_tmp, n_sms, s, stats);
    if (cap > 0) {
        const uint32_t want = (cap + 255) / 256, limit = uint32_t(n_sms) * 16;
        k_tile_ranges<<<want < limit ? want : limit, 256, 0, s>>>(b.pair_tile[par], b.n_sort, ranges, n_tiles, stats);
        note_launch();
    }
    return par;
}

template <class T>
inline int run_binning(uint32_t N, unsigned gx, unsigned gy, const uint32_t* tiles_touched, uint32_t* point_offsets, const int32_t* rects, const T* xy,
    uint32_t cap, BinningBuffers& b, int32_t* ranges, uint32_t* stats, int n_sms, cudaStream_t s, bool offsets_ready = false)
{
    return run_binning_grids<T>(N, gx * gy, SingleGrid { gx, gy }, tiles_touched, point_offsets, rects, xy, cap, b, ranges, stats, n_sms, s, offsets_ready);
}

} // namespace dgmr
