// Tile binning shared by the splat renderer, the volume marcher and the
// volume rasteriser.
//
// The reference emits one 64-bit key (tile << 32 | float bits of depth) per
// (tile, Gaussian) pair and radix-sorts all pairs over 32 + msb(tiles) bits
// (splat_forward.cu:159-211).  The sorted order it produces is the order of
// (tile, depth bits, Gaussian index).  Here the same order is reached without
// sorting the pairs at all:
//   1. the N Gaussians are stably sorted once by their 32-bit depth bits;
//   2. each Gaussian, in that order, emits one entry per 8x8-tile super-tile
//      its rectangle touches (about 1.5 per Gaussian instead of ~9 pairs):
//      key = super-tile id << 12 | the part of its tile rectangle inside that
//      super-tile, value = the Gaussian; one stable radix pass over the
//      super-tile bits groups them, every super-tile's entries in depth order;
//   3. each super-tile's entry list is cut into chunks of 1024; a chunk
//      counts, per tile of its super-tile, the entries covering that tile;
//      prefix sums over the chunks and over the tiles (in tile order) give
//      every tile's range and every chunk's start inside it;
//   4. each chunk writes its pairs: an entry's rank inside a tile is the
//      count of earlier entries of the chunk covering that tile (warp
//      ballots, then warps in order), so each tile's pairs land in depth
//      order.
// The result -- point list, its tile ids and the tile ranges -- is identical
// bit for bit to the reference's sorted order.
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

constexpr unsigned kSuper = 8; // tiles per super-tile side
constexpr unsigned kSuperTiles = kSuper * kSuper; // 64: one bit each in a u64 mask
constexpr unsigned kChunk = 1024; // super-tile entries per chunk
constexpr unsigned kChunkThreads = 256;
constexpr int kRectBits = 12; // a rectangle inside a super-tile: x0, width - 1, y0, height - 1, 3 bits each

// Scratch of the binning stage.  n_tiles bounds the super-tile count (every
// super-tile holds at least one tile).
struct BinningBuffers {
    uint32_t* depth_key; // [N]
    uint32_t* perm; // [N]  (holds iota on entry, the depth order on exit)
    uint32_t* key_tmp; // [N]
    uint32_t* perm_tmp; // [N]
    uint32_t* cnt_sorted; // [N] super-tiles touched, in depth order
    uint32_t* off_sorted; // [N] their inclusive scan
    uint32_t* scan_tmp; // scan_temp_bytes(max(N, n_tiles))
    uint32_t* n_sort; // [8] min(P, cap), super entries to sort, chunk count, spare, depth-key min / max,
                      // blocks done in the blend's tile-order kernel, spare
    int32_t* super_ranges; // [n_tiles, 2] each super-tile's entries in the sorted list
    uint32_t* chunk_base; // [n_tiles + 1] first chunk of each super-tile
    uint32_t* tile_total; // [n_tiles] pairs per tile
    uint32_t* tile_incl; // [n_tiles] their inclusive scan in tile order
    uint32_t* pair_tile[2]; // [cap] super-tile entries (keys), then the tile of each pair
    uint32_t* pair_val[2]; // [cap] super-tile entries (depth ranks), then the point list
    void* sort_tmp; // radix_temp_bytes(max(N, cap))
    uint32_t* chunk_lo; // [n_tiles, 64] per-chunk tile counts (then their prefix over chunks), chunks [0, n_tiles)
    uint32_t* chunk_hi; // [ceil(cap / kChunk), 64] the same for chunks [n_tiles, max chunks)
    uint32_t lo_rows, hi_rows;
};

// Chunk count rows, split between the frame workspace (one row per tile) and
// the pair workspace (one row per kChunk pairs of capacity): a super-tile
// with L entries has ceil(L / kChunk) <= L / kChunk + 1 chunks, so there are
// at most cap / kChunk + n_tiles chunks.
struct ChunkRows {
    uint32_t* lo;
    uint32_t* hi;
    uint32_t lo_rows, max_chunks;
    __device__ __forceinline__ uint32_t* row(uint32_t c) const
    {
        return c < lo_rows ? lo + size_t(c) * kSuperTiles : hi + size_t(c - lo_rows) * kSuperTiles;
    }
};

// the parts sized by the Gaussian count and the tile count
inline void carve_binning_gaussians(Carver& c, BinningBuffers& b, uint32_t N, uint32_t n_tiles)
{
    b.depth_key = c.take<uint32_t>(N);
    b.perm = c.take<uint32_t>(N);
    b.key_tmp = c.take<uint32_t>(N);
    b.perm_tmp = c.take<uint32_t>(N);
    b.cnt_sorted = c.take<uint32_t>(N);
    b.off_sorted = c.take<uint32_t>(N);
    b.scan_tmp = c.take<uint32_t>(scan_temp_bytes(N > n_tiles ? N : n_tiles) / 4 + 1);
    b.n_sort = c.take<uint32_t>(8);
    b.super_ranges = c.take<int32_t>(size_t(n_tiles) * 2);
    b.chunk_base = c.take<uint32_t>(size_t(n_tiles) + 1);
    b.tile_total = c.take<uint32_t>(n_tiles);
    b.tile_incl = c.take<uint32_t>(n_tiles);
    b.lo_rows = n_tiles;
    b.chunk_lo = c.take<uint32_t>(size_t(n_tiles) * kSuperTiles);
}

// the parts sized by the pair capacity (and the sort scratch)
inline void carve_binning_pairs(Carver& c, BinningBuffers& b, uint32_t N, uint32_t cap)
{
    for (int i = 0; i < 2; ++i) {
        b.pair_tile[i] = c.take<uint32_t>(cap);
        b.pair_val[i] = c.take<uint32_t>(cap);
    }
    b.hi_rows = (cap + kChunk - 1) / kChunk;
    b.chunk_hi = c.take<uint32_t>(size_t(b.hi_rows) * kSuperTiles);
    b.sort_tmp = c.take<char>(radix_temp_bytes(N > cap ? N : cap));
}

inline void carve_binning(Carver& c, BinningBuffers& b, uint32_t N, uint32_t n_tiles, uint32_t cap)
{
    carve_binning_gaussians(c, b, N, n_tiles);
    carve_binning_pairs(c, b, N, cap);
}

inline ChunkRows chunk_rows(const BinningBuffers& b) { return ChunkRows { b.chunk_lo, b.chunk_hi, b.lo_rows, b.lo_rows + b.hi_rows }; }

inline uint32_t super_count(uint32_t gx, uint32_t gy) { return ((gx + kSuper - 1) / kSuper) * ((gy + kSuper - 1) / kSuper); }

// Buffer index holding the point list and its tile ids: the super-tile
// entries are emitted into buffer 0 and radix-sorted (one pass per 8 bits of
// the super-tile count, ping-ponging), and the pairs are written into the
// buffer the sort did not end in.
inline int tile_sort_parity(uint32_t n_super)
{
    const int bits = int(higher_msb(n_super));
    return 1 - (((bits + 7) / 8) & 1);
}

static __global__ void k_pair_count(const uint32_t* __restrict__ point_offsets, uint32_t N, uint32_t cap, uint32_t* __restrict__ stats, uint32_t* __restrict__ n_sort)
{
    n_sort[4] = 0xffffffffu; // depth-key range, filled by k_key_range
    n_sort[5] = 0u;
    n_sort[6] = 0u; // counter of the blend's tile-order kernel (k_blend_tile_order)
    const uint32_t P = N ? point_offsets[N - 1] : 0u;
    stats[0] = P;
    if (P > cap)
        atomicOr(&stats[1], 1u);
    *n_sort = P < cap ? P : cap;
}

// Tile grid of the frame a Gaussian slot (or a super-tile) belongs to: its
// size, the offset of its first tile in the (possibly multi-frame) tile
// numbering and the offset of its first super-tile in the super-tile numbering.
struct TileGrid {
    unsigned gx, gy, off, soff;
};

// One frame: every slot uses the same grid.
struct SingleGrid {
    unsigned gx, gy;
    __device__ __forceinline__ TileGrid grid(uint32_t) const { return TileGrid { gx, gy, 0u, 0u }; }
    __device__ __forceinline__ TileGrid super_grid(uint32_t) const { return TileGrid { gx, gy, 0u, 0u }; }
};

// Two consecutive values in one load (the address is aligned to their size).
__device__ __forceinline__ V2<float> load_pair(const float* p)
{
    const float2 v = *reinterpret_cast<const float2*>(p);
    return V2<float> { v.x, v.y };
}
__device__ __forceinline__ V2<double> load_pair(const double* p)
{
    const double2 v = *reinterpret_cast<const double2*>(p);
    return V2<double> { v.x, v.y };
}

// A Gaussian's tile rectangle (util.h:42-52 on the cached rect and centroid),
// checked against its tile count; empty when the count is 0 or disagrees.
template <class T>
__device__ __forceinline__ TileRect checked_rect(uint32_t g, const uint32_t* __restrict__ tiles_touched, const int32_t* __restrict__ rects,
    const T* __restrict__ xy, const TileGrid& tg, uint32_t* __restrict__ stats)
{
    TileRect r = { 0, 0, 0, 0 };
    // the count, rectangle and centre are requested together (8-byte loads for
    // the pairs), not one after the other
    const uint32_t c = tiles_touched[g];
    const int2 e = reinterpret_cast<const int2*>(rects)[g];
    const V2<T> p = load_pair(xy + 2 * size_t(g));
    if (c > 0) {
        r = get_rect(float(p.x), float(p.y), e.x, e.y, tg.gx, tg.gy);
        if ((r.x1 - r.x0) * (r.y1 - r.y0) != c) {
            flag_bounds(stats, 0x22u);
            r = { 0, 0, 0, 0 };
        }
    }
    return r;
}

__device__ __forceinline__ TileRect super_rect(const TileRect& r)
{
    if (r.x1 <= r.x0 || r.y1 <= r.y0)
        return TileRect { 0, 0, 0, 0 };
    return TileRect { r.x0 / kSuper, r.y0 / kSuper, (r.x1 - 1) / kSuper + 1, (r.y1 - 1) / kSuper + 1 };
}

// Super-tiles touched by the j-th Gaussian in depth order, and its tile
// rectangle in depth order (x0 | y0 << 16, x1 | y1 << 16), so that the
// emission reads it contiguously.
template <class T, class Grids>
static __global__ void k_super_counts(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ tiles_touched, const int32_t* __restrict__ rects,
    const T* __restrict__ xy, uint32_t N, uint32_t* __restrict__ cnt_sorted, uint32_t* __restrict__ rect_lo, uint32_t* __restrict__ rect_hi,
    uint32_t* __restrict__ stats, const __grid_constant__ Grids grids)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N)
        return;
    uint32_t g = perm[j];
    uint32_t c = 0;
    TileRect r = { 0, 0, 0, 0 };
    if (g < N) {
        r = checked_rect(g, tiles_touched, rects, xy, grids.grid(g), stats);
        const TileRect sr = super_rect(r);
        c = (sr.x1 - sr.x0) * (sr.y1 - sr.y0);
    } else {
        flag_bounds(stats, 0x21u);
    }
    cnt_sorted[j] = c;
    rect_lo[j] = r.x0 | (r.y0 << 16);
    rect_hi[j] = r.x1 | (r.y1 << 16);
}

// n_sort[1] = super-tile entries to sort = min(total, cap)
static __global__ void k_super_total(const uint32_t* __restrict__ off_sorted, uint32_t N, uint32_t cap, uint32_t* __restrict__ n_sort)
{
    const uint32_t n = N ? off_sorted[N - 1] : 0u;
    n_sort[1] = n < cap ? n : cap;
}

// Super-tile entries in depth order: for the j-th Gaussian by depth, one entry
// per super-tile its rectangle touches, row-major: key = super-tile id << 12 |
// the rectangle's part inside it, value = the Gaussian.  The 32
// Gaussians of a warp own one contiguous output range (their offsets come
// from an inclusive scan in the same order), so the warp writes that range
// together: in each round lane l takes slot base + l and finds its owner --
// the first lane whose inclusive end exceeds the slot -- by a five-step
// binary search over the lanes' ends, done with shuffles.
template <class Grids>
static __global__ void __launch_bounds__(256) k_emit_super(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ cnt_sorted,
    const uint32_t* __restrict__ off_sorted, const uint32_t* __restrict__ rect_lo, const uint32_t* __restrict__ rect_hi, uint32_t N, uint32_t cap,
    uint32_t* __restrict__ skey, uint32_t* __restrict__ sval, uint32_t* __restrict__ stats, const __grid_constant__ Grids grids)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    if (__all_sync(0xffffffffu, j >= N))
        return;
    uint32_t c = 0, end = 0, g = 0xffffffffu;
    TileRect tr = { 0, 0, 0, 0 }, sr = { 0, 0, 0, 0 };
    TileGrid tg = { 0u, 0u, 0u, 0u };
    if (j < N) {
        c = cnt_sorted[j];
        end = off_sorted[j];
        if (c > 0) {
            g = perm[j];
            if (g < N) {
                tg = grids.grid(g);
                const uint32_t lo = rect_lo[j], hi = rect_hi[j];
                tr = TileRect { lo & 0xffffu, lo >> 16, hi & 0xffffu, hi >> 16 };
                sr = super_rect(tr);
                if ((sr.x1 - sr.x0) * (sr.y1 - sr.y0) != c) {
                    flag_bounds(stats, 0x26u);
                    sr = { 0, 0, 0, 0 };
                }
            } else {
                flag_bounds(stats, 0x23u);
                g = 0xffffffffu;
            }
        }
    }
    const uint32_t start = end - c;
    const uint32_t key = j < N ? end : 0xffffffffu;
    const uint32_t lo = __shfl_sync(0xffffffffu, start, 0);
    uint32_t hi = j < N ? end : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    const uint32_t rw = sr.x1 - sr.x0;
    const uint32_t sgx = (tg.gx + kSuper - 1) / kSuper, sgy = (tg.gy + kSuper - 1) / kSuper;
    for (uint32_t base = lo; base < hi; base += 32) {
        const uint32_t pos = base + lane;
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
        const uint32_t s_tx0 = __shfl_sync(0xffffffffu, tr.x0, src);
        const uint32_t s_ty0 = __shfl_sync(0xffffffffu, tr.y0, src);
        const uint32_t s_tx1 = __shfl_sync(0xffffffffu, tr.x1, src);
        const uint32_t s_ty1 = __shfl_sync(0xffffffffu, tr.y1, src);
        const uint32_t s_x0 = __shfl_sync(0xffffffffu, sr.x0, src);
        const uint32_t s_y0 = __shfl_sync(0xffffffffu, sr.y0, src);
        const uint32_t s_w = __shfl_sync(0xffffffffu, rw, src);
        const uint32_t s_gx = __shfl_sync(0xffffffffu, sgx, src);
        const uint32_t s_n = __shfl_sync(0xffffffffu, sgx * sgy, src);
        const uint32_t s_off = __shfl_sync(0xffffffffu, tg.soff, src);
        if (pos < hi && pos < cap) {
            const uint32_t k = pos - s_start;
            const uint32_t sx = s_x0 + (s_w ? k % s_w : 0u), sy = s_y0 + (s_w ? k / s_w : 0u);
            const uint32_t t = (s_w && k < s_c) ? sy * s_gx + sx : 0xffffffffu;
            if (t < s_n) {
                // the tile rectangle clipped to this super-tile, in its local coordinates
                const uint32_t bx = sx * kSuper, by = sy * kSuper;
                const uint32_t x0 = s_tx0 > bx ? s_tx0 - bx : 0u, y0 = s_ty0 > by ? s_ty0 - by : 0u;
                const uint32_t x1 = s_tx1 < bx + kSuper ? s_tx1 - bx : kSuper, y1 = s_ty1 < by + kSuper ? s_ty1 - by : kSuper;
                skey[pos] = ((s_off + t) << kRectBits) | x0 | ((x1 - x0 - 1u) << 3) | (y0 << 6) | ((y1 - y0 - 1u) << 9);
                sval[pos] = s_g;
            } else {
                skey[pos] = 0;
                sval[pos] = 0xffffffffu; // an entry that covers no tile
                flag_bounds(stats, 0x24u);
            }
        }
    }
}

// Chunks of every super-tile's entry list: chunk_base[s] = first chunk of
// super-tile s (exclusive scan of ceil(len / kChunk)); n_sort[2] = chunk
// count.  One block.
static __global__ void __launch_bounds__(1024) k_chunk_plan(const int32_t* __restrict__ super_ranges, uint32_t n_super, uint32_t* __restrict__ chunk_base,
    uint32_t* __restrict__ n_sort)
{
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < n_super; b0 += 1024) {
        const uint32_t s = b0 + threadIdx.x;
        uint32_t v = 0;
        if (s < n_super) {
            const int32_t len = super_ranges[2 * s + 1] - super_ranges[2 * s];
            v = len > 0 ? (uint32_t(len) + kChunk - 1) / kChunk : 0u;
        }
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
        for (int w = 0; w < 32; ++w) {
            const uint32_t t = warp_tot[w];
            wex += (w < warp) ? t : 0;
            tot += t;
        }
        if (s < n_super)
            chunk_base[s] = carry + wex + x - v;
        __syncthreads();
        if (threadIdx.x == 0)
            carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        chunk_base[n_super] = carry;
        n_sort[2] = carry;
    }
}

// One chunk of one super-tile, as seen by the per-chunk kernels.
struct ChunkRef {
    uint32_t s; // global super-tile id
    uint32_t a, b; // its entries [a, b) in the sorted list
    TileGrid tg;
    uint32_t sx, sy; // super-tile position inside its frame
};

template <class Grids>
__device__ __forceinline__ ChunkRef chunk_ref(uint32_t c, const uint32_t* __restrict__ chunk_base, uint32_t n_super, const int32_t* __restrict__ super_ranges,
    const Grids& grids)
{
    // largest s < n_super with chunk_base[s] <= c (super-tiles without chunks are skipped over)
    uint32_t lo = 0, hi = n_super;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (chunk_base[mid] <= c)
            lo = mid;
        else
            hi = mid;
    }
    ChunkRef r;
    r.s = lo;
    const uint32_t seg_a = uint32_t(super_ranges[2 * lo]), seg_b = uint32_t(super_ranges[2 * lo + 1]);
    r.a = seg_a + (c - chunk_base[lo]) * kChunk;
    r.b = r.a + kChunk < seg_b ? r.a + kChunk : seg_b;
    r.tg = grids.super_grid(lo);
    const uint32_t sgx = (r.tg.gx + kSuper - 1) / kSuper;
    const uint32_t local = lo - r.tg.soff;
    r.sx = local % sgx;
    r.sy = local / sgx;
    return r;
}

// Tiles of the chunk's super-tile covered by an entry: bit (ly * 8 + lx) for
// local tile (lx, ly), from the rectangle in the key's low 12 bits.  An entry
// whose value is not a Gaussian covers nothing.
__device__ __forceinline__ unsigned long long entry_mask(uint32_t key, uint32_t g, uint32_t N, uint32_t* __restrict__ stats)
{
    if (g >= N) {
        if (g != 0xffffffffu)
            flag_bounds(stats, 0x27u);
        return 0ull;
    }
    const uint32_t x0 = key & 7u, w = ((key >> 3) & 7u) + 1u, y0 = (key >> 6) & 7u, h = ((key >> 9) & 7u) + 1u;
    const uint32_t ww = x0 + w <= kSuper ? w : kSuper - x0, hh = y0 + h <= kSuper ? h : kSuper - y0;
    const unsigned long long row = ((1ull << ww) - 1ull) << x0; // one row of the rectangle
    const unsigned long long col = 0x0101010101010101ull >> (kSuper * (kSuper - hh)); // bit 0 of its hh rows
    return (row * col) << (kSuper * y0);
}

__device__ __forceinline__ uint32_t chunk_tile(const ChunkRef& ch, uint32_t k, bool* exists)
{
    const uint32_t tx = ch.sx * kSuper + (k % kSuper), ty = ch.sy * kSuper + (k / kSuper);
    *exists = tx < ch.tg.gx && ty < ch.tg.gy;
    return ch.tg.off + ty * ch.tg.gx + tx;
}

// Transpose of a 32 x 32 bit matrix held one row per lane: returns, for lane
// l, the word whose bit r is bit l of lane r's row.  Five levels of 2 x 2
// block swaps, each one shuffle exchange.
__device__ __forceinline__ uint32_t warp_bit_transpose(uint32_t x, int lane)
{
    const uint32_t masks[5] = { 0x0000ffffu, 0x00ff00ffu, 0x0f0f0f0fu, 0x33333333u, 0x55555555u };
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const int j = 16 >> i;
        const uint32_t lo = masks[i];
        const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
        x = (lane & j) ? ((x & ~lo) | ((y & ~lo) >> j)) : ((x & lo) | ((y & lo) << j));
    }
    return x;
}

// Per chunk: how many of its entries cover each of the super-tile's 64 tiles.
template <class Grids>
static __global__ void __launch_bounds__(kChunkThreads) k_chunk_counts(const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sval, uint32_t N,
    const int32_t* __restrict__ super_ranges, const uint32_t* __restrict__ chunk_base, uint32_t n_super, const uint32_t* __restrict__ n_sort,
    const ChunkRows rows, uint32_t* __restrict__ stats, const __grid_constant__ Grids grids)
{
    __shared__ uint32_t cnt[kSuperTiles];
    uint32_t n_chunks = n_sort[2];
    if (n_chunks > rows.max_chunks) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            flag_bounds(stats, 0x28u);
        n_chunks = rows.max_chunks;
    }
    for (uint32_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        if (threadIdx.x < kSuperTiles)
            cnt[threadIdx.x] = 0;
        __syncthreads();
        const ChunkRef ch = chunk_ref(c, chunk_base, n_super, super_ranges, grids);
        const int lane = threadIdx.x & 31;
        for (uint32_t r0 = ch.a; r0 < ch.b; r0 += kChunkThreads) {
            const uint32_t e = r0 + threadIdx.x;
            const unsigned long long m = e < ch.b ? entry_mask(skey[e], sval[e], N, stats) : 0ull;
            // lane l: how many of the warp's entries cover tiles l and l + 32
            const uint32_t n_lo = __popc(warp_bit_transpose(uint32_t(m), lane));
            const uint32_t n_hi = __popc(warp_bit_transpose(uint32_t(m >> 32), lane));
            if (n_lo)
                atomicAdd(&cnt[lane], n_lo);
            if (n_hi)
                atomicAdd(&cnt[lane + 32], n_hi);
        }
        __syncthreads();
        if (threadIdx.x < kSuperTiles)
            rows.row(c)[threadIdx.x] = cnt[threadIdx.x];
        __syncthreads();
    }
}

// Per (super-tile, local tile): exclusive prefix of the chunk counts over the
// super-tile's chunks (in place) and the tile's total.  One block of
// 64 x 16 threads per super-tile: thread (k, q) owns the q-th sixteenth of
// the chunks for tile k -- sums it, takes the sums of the earlier sixteenths,
// then writes its prefixes.
constexpr int kPrefixParts = 16;
template <class Grids>
static __global__ void __launch_bounds__(kSuperTiles* kPrefixParts) k_chunk_prefix(const uint32_t* __restrict__ chunk_base, uint32_t n_super,
    const ChunkRows rows, uint32_t* __restrict__ tile_total, uint32_t n_tiles, uint32_t* __restrict__ stats, const __grid_constant__ Grids grids)
{
    __shared__ uint32_t part[kPrefixParts][kSuperTiles];
    const uint32_t s = blockIdx.x;
    const uint32_t k = threadIdx.x % kSuperTiles, q = threadIdx.x / kSuperTiles;
    const uint32_t c0 = chunk_base[s];
    uint32_t c1 = chunk_base[s + 1];
    if (c1 > rows.max_chunks) {
        if (threadIdx.x == 0)
            flag_bounds(stats, 0x28u);
        c1 = rows.max_chunks;
    }
    const uint32_t n = c1 > c0 ? c1 - c0 : 0u;
    const uint32_t per = (n + kPrefixParts - 1) / kPrefixParts;
    const uint32_t a = c0 + (q * per < n ? q * per : n), b = c0 + ((q + 1) * per < n ? (q + 1) * per : n);
    uint32_t sum = 0;
    for (uint32_t c = a; c < b; ++c)
        sum += rows.row(c)[k];
    part[q][k] = sum;
    __syncthreads();
    uint32_t run = 0, total = 0;
    for (uint32_t p = 0; p < kPrefixParts; ++p) {
        const uint32_t v = part[p][k];
        run += p < q ? v : 0u;
        total += v;
    }
    for (uint32_t c = a; c < b; ++c) {
        uint32_t* r = rows.row(c);
        const uint32_t v = r[k];
        r[k] = run;
        run += v;
    }
    if (q != 0)
        return;
    const TileGrid tg = grids.super_grid(s);
    const uint32_t sgx = (tg.gx + kSuper - 1) / kSuper, local = s - tg.soff;
    const uint32_t tx = (local % sgx) * kSuper + (k % kSuper), ty = (local / sgx) * kSuper + (k / kSuper);
    if (tx < tg.gx && ty < tg.gy) {
        const uint32_t t = tg.off + ty * tg.gx + tx;
        if (t < n_tiles)
            tile_total[t] = total;
        else
            flag_bounds(stats, 0x29u);
    } else if (total) {
        flag_bounds(stats, 0x2au);
    }
}

// splat_forward.cu:218-239: [start, end) of each tile's run, (0, 0) for an
// empty tile; clamped to the pair capacity.
static __global__ void k_tile_ranges_from_counts(const uint32_t* __restrict__ tile_total, const uint32_t* __restrict__ tile_incl, uint32_t n_tiles,
    uint32_t cap, int32_t* __restrict__ ranges)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tiles)
        return;
    const uint32_t tot = tile_total[t], end = tile_incl[t];
    const uint32_t start = end - tot;
    ranges[2 * t] = tot ? int32_t(start < cap ? start : cap) : 0;
    ranges[2 * t + 1] = tot ? int32_t(end < cap ? end : cap) : 0;
}

// Per chunk: every entry's pairs at their final positions.  Rounds of 256
// entries in list order; in a round, warp w's ballot of tile k says which of
// its lanes cover k, and the warps' counts are summed in warp order, so the
// rank of an entry in tile k is (pairs of earlier rounds) + (earlier warps) +
// (earlier lanes).  A round's pairs (typically ~1.5-2k) are first staged in
// shared memory grouped by tile, then copied out run by run, so that
// consecutive threads store consecutive addresses of one tile's run; a round
// with more pairs than the stage holds writes them directly.  Three barriers
// per round: after the ballots (which also ends the previous copy-out, so warp
// 0 then advances the tile positions by the previous round's counts), after
// the offsets, and after the staging.
constexpr unsigned kEmitStage = 4096;
template <class Grids>
static __global__ void __launch_bounds__(kChunkThreads) k_chunk_emit(const uint32_t* __restrict__ skey, const uint32_t* __restrict__ sval, uint32_t N,
    const int32_t* __restrict__ super_ranges, const uint32_t* __restrict__ chunk_base, uint32_t n_super, const uint32_t* __restrict__ n_sort,
    const ChunkRows rows, const uint32_t* __restrict__ tile_total, const uint32_t* __restrict__ tile_incl, uint32_t cap, uint32_t* __restrict__ out_tile,
    uint32_t* __restrict__ out_val, uint32_t* __restrict__ stats, const __grid_constant__ Grids grids)
{
    constexpr int kWarps = kChunkThreads / 32;
    extern __shared__ uint32_t stage_val[]; // [kEmitStage]
    uint8_t* stage_k = reinterpret_cast<uint8_t*>(stage_val + kEmitStage); // [kEmitStage]
    __shared__ uint32_t base[kSuperTiles]; // next global position of each tile
    __shared__ uint32_t tile_id[kSuperTiles];
    __shared__ uint32_t roff[kSuperTiles + 1]; // start of each tile's run in the stage
    __shared__ uint32_t bal[kWarps][kSuperTiles];
    __shared__ uint32_t wpre[kWarps][kSuperTiles];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t n_chunks = n_sort[2];
    n_chunks = n_chunks < rows.max_chunks ? n_chunks : rows.max_chunks;
    for (uint32_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const ChunkRef ch = chunk_ref(c, chunk_base, n_super, super_ranges, grids);
        if (threadIdx.x < kSuperTiles) {
            bool ex;
            const uint32_t t = chunk_tile(ch, threadIdx.x, &ex);
            tile_id[threadIdx.x] = ex ? t : 0xffffffffu;
            base[threadIdx.x] = ex ? (tile_incl[t] - tile_total[t]) + rows.row(c)[threadIdx.x] : 0u;
        }
        __syncthreads();
        for (uint32_t r0 = ch.a; r0 < ch.b; r0 += kChunkThreads) {
            const uint32_t e = r0 + threadIdx.x;
            const uint32_t g = e < ch.b ? sval[e] : 0xffffffffu;
            const unsigned long long m = e < ch.b ? entry_mask(skey[e], g, N, stats) : 0ull;
            // the ballots of all 64 tiles: lane l gets those of tiles l and l + 32
            // by transposing the warp's 32 x 32 bit matrices (row = lane, column
            // = tile) with five shuffle exchanges each
            const uint32_t b_lo = warp_bit_transpose(uint32_t(m), lane);
            const uint32_t b_hi = warp_bit_transpose(uint32_t(m >> 32), lane);
            bal[warp][lane] = b_lo;
            bal[warp][lane + 32] = b_hi;
            __syncthreads(); // also ends the previous round's copy-out
            if (warp == 0) {
                if (r0 != ch.a) { // the previous round's pairs advance each tile's position
                    base[lane] += roff[lane + 1] - roff[lane];
                    base[lane + 32] += roff[lane + 33] - roff[lane + 32];
                }
                // per tile: prefix over warps, then the exclusive scan over the 64 tiles
                uint32_t run_lo = 0, run_hi = 0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) {
                    wpre[w][lane] = run_lo;
                    wpre[w][lane + 32] = run_hi;
                    run_lo += __popc(bal[w][lane]);
                    run_hi += __popc(bal[w][lane + 32]);
                }
                uint32_t x = run_lo, y = run_hi;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t xs = __shfl_up_sync(0xffffffffu, x, o);
                    const uint32_t ys = __shfl_up_sync(0xffffffffu, y, o);
                    if (lane >= o) {
                        x += xs;
                        y += ys;
                    }
                }
                const uint32_t lo_total = __shfl_sync(0xffffffffu, x, 31);
                __syncwarp(); // the base update above read the old offsets
                roff[lane + 1] = x;
                roff[lane + 33] = lo_total + y;
                if (lane == 0)
                    roff[0] = 0;
            }
            __syncthreads();
            const uint32_t total = roff[kSuperTiles];
            const bool staged = total <= kEmitStage;
            unsigned long long own = m;
            while (own) {
                const int k = __ffsll(static_cast<long long>(own)) - 1;
                own &= own - 1ull;
                const uint32_t rank = wpre[warp][k] + __popc(bal[warp][k] & lt);
                if (staged) {
                    stage_val[roff[k] + rank] = g;
                    stage_k[roff[k] + rank] = uint8_t(k);
                } else {
                    const uint32_t t = tile_id[k];
                    const uint32_t pos = base[k] + rank;
                    if (t == 0xffffffffu) {
                        flag_bounds(stats, 0x2bu);
                    } else if (pos < cap) {
                        out_tile[pos] = t;
                        out_val[pos] = g;
                    }
                }
            }
            __syncthreads();
            for (uint32_t i = threadIdx.x; staged && i < total; i += kChunkThreads) {
                const uint32_t k = stage_k[i];
                const uint32_t t = tile_id[k];
                const uint32_t pos = base[k] + (i - roff[k]);
                if (t == 0xffffffffu) {
                    flag_bounds(stats, 0x2bu);
                } else if (pos < cap) {
                    out_tile[pos] = t;
                    out_val[pos] = stage_val[i];
                }
            }
        }
        __syncthreads(); // the last copy-out reads base and tile_id
    }
}

inline size_t chunk_emit_smem() { return size_t(kEmitStage) * (sizeof(uint32_t) + sizeof(uint8_t)); }

// [start, end) of every run of equal keys in a sorted key list (the tile
// ranges of splat_forward.cu:218-239; here applied to the sorted super-tile
// entries, whose keys carry the super-tile id above bit `shift`).  ranges
// must be zeroed beforehand.
static __global__ void k_tile_ranges(const uint32_t* __restrict__ tiles_sorted, const uint32_t* __restrict__ n_dev, int32_t* __restrict__ ranges, uint32_t n_tiles,
    uint32_t* __restrict__ stats, int shift)
{
    const uint32_t n = *n_dev;
    // four items per thread and step, every load issued before the first is used
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 4u * stride) {
        uint32_t cur_v[4], prev_v[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t idx = i0 + uint32_t(r) * stride;
            cur_v[r] = idx < n ? tiles_sorted[idx] >> shift : 0u;
            prev_v[r] = (idx < n && idx) ? tiles_sorted[idx - 1] >> shift : 0u;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t idx = i0 + uint32_t(r) * stride;
            if (idx >= n)
                break;
            const uint32_t cur = cur_v[r], prev = prev_v[r];
            if (cur >= n_tiles || prev >= n_tiles) {
                flag_bounds(stats, 0x25u);
                continue;
            }
            if (idx == 0)
                ranges[2 * cur] = 0;
            else if (cur != prev) {
                ranges[2 * prev + 1] = int32_t(idx);
                ranges[2 * cur] = int32_t(idx);
            }
            if (idx == n - 1)
                ranges[2 * cur + 1] = int32_t(n);
        }
    }
}

// Launch order for the marcher's per-tile kernels: tiles bucketed by
// floor(log2(list length + 1)), longest first, so the heaviest tiles start at
// the head of the grid instead of stretching its tail.  One block; order
// inside a bucket is arbitrary (it only affects scheduling, never results).
// The splat blend orders its tiles by a predicted cost instead
// (k_blend_tile_order): there the longest lists saturate early.
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
// super-tile entries and their sort, chunk counts, tile ranges and the point
// list.  Returns the buffer index holding the point list (pair_val) and its
// tile ids (pair_tile).  Requires b.perm = iota and b.depth_key filled by the
// preprocess.  n_super = super-tiles of all frames (super_count per frame).
template <class T, class Grids>
inline int run_binning_grids(uint32_t N, uint32_t n_tiles, uint32_t n_super, const Grids& grids, const uint32_t* tiles_touched, uint32_t* point_offsets,
    const int32_t* rects, const T* xy, uint32_t cap, BinningBuffers& b, int32_t* ranges, uint32_t* stats, int n_sms, cudaStream_t s, bool offsets_ready)
{
    const int par = tile_sort_parity(n_super);
    if (N == 0) {
        cudaMemsetAsync(ranges, 0, size_t(n_tiles) * 2 * sizeof(int32_t), s);
        cudaMemsetAsync(b.n_sort, 0, 8 * sizeof(uint32_t), s);
        return par;
    }
    if (!offsets_ready)
        inclusive_scan_u32(tiles_touched, point_offsets, N, b.scan_tmp, s);
    k_pair_count<<<1, 1, 0, s>>>(point_offsets, N, cap, stats, b.n_sort);
    note_launch();
    // the depth keys of the Gaussians that touch a tile usually span < 2^24
    // values: rebased, the top pass only copies
    {
        const uint32_t want = (N + 255) / 256, limit = uint32_t(n_sms) * 8;
        k_key_range<<<want < limit ? want : limit, 256, 0, s>>>(b.depth_key, tiles_touched, N, b.n_sort + 4);
        note_launch();
    }
    const int dpar = radix_sort_pairs(b.depth_key, b.perm, b.key_tmp, b.perm_tmp, nullptr, N, N, 32, b.sort_tmp, n_sms, s, stats, 0, b.n_sort + 4,
        tiles_touched);
    const uint32_t* perm = dpar ? b.perm_tmp : b.perm;
    // the pair of N-sized buffers the depth sort did not end in holds the rectangles
    uint32_t* rect_lo = dpar ? b.depth_key : b.key_tmp;
    uint32_t* rect_hi = dpar ? b.perm : b.perm_tmp;
    const uint32_t blocks = (N + 255) / 256;
    k_super_counts<T, Grids><<<blocks, 256, 0, s>>>(perm, tiles_touched, rects, xy, N, b.cnt_sorted, rect_lo, rect_hi, stats, grids);
    inclusive_scan_u32(b.cnt_sorted, b.off_sorted, N, b.scan_tmp, s);
    k_super_total<<<1, 1, 0, s>>>(b.off_sorted, N, cap, b.n_sort);
    note_launch(2);
    cudaMemsetAsync(b.super_ranges, 0, size_t(n_super) * 2 * sizeof(int32_t), s);
    cudaMemsetAsync(b.tile_total, 0, size_t(n_tiles) * sizeof(uint32_t), s);
    if (cap > 0) {
        k_emit_super<Grids><<<blocks, 256, 0, s>>>(perm, b.cnt_sorted, b.off_sorted, rect_lo, rect_hi, N, cap, b.pair_tile[0], b.pair_val[0], stats, grids);
        note_launch();
        const int spar = radix_sort_pairs(b.pair_tile[0], b.pair_val[0], b.pair_tile[1], b.pair_val[1], b.n_sort + 1, 0, cap,
            kRectBits + int(higher_msb(n_super)), b.sort_tmp, n_sms, s, stats, kRectBits);
        const uint32_t want = (cap + 255) / 256, limit = uint32_t(n_sms) * 16;
        k_tile_ranges<<<want < limit ? want : limit, 256, 0, s>>>(b.pair_tile[spar], b.n_sort + 1, b.super_ranges, n_super, stats, kRectBits);
        k_chunk_plan<<<1, 1024, 0, s>>>(b.super_ranges, n_super, b.chunk_base, b.n_sort);
        const ChunkRows rows = chunk_rows(b);
        const uint32_t cgrid = rows.max_chunks < uint32_t(n_sms) * 8 ? rows.max_chunks : uint32_t(n_sms) * 8;
        k_chunk_counts<Grids><<<cgrid, kChunkThreads, 0, s>>>(b.pair_tile[spar], b.pair_val[spar], N, b.super_ranges, b.chunk_base, n_super, b.n_sort, rows,
            stats, grids);
        k_chunk_prefix<Grids><<<n_super, kSuperTiles * kPrefixParts, 0, s>>>(b.chunk_base, n_super, rows, b.tile_total, n_tiles, stats, grids);
        note_launch(4);
        if (n_tiles <= kScanSingleMax) {
            k_scan_single<<<1, 1024, 0, s>>>(b.tile_total, n_tiles, b.tile_incl);
            note_launch();
        } else {
            inclusive_scan_u32(b.tile_total, b.tile_incl, n_tiles, b.scan_tmp, s);
        }
        k_tile_ranges_from_counts<<<(n_tiles + 255) / 256, 256, 0, s>>>(b.tile_total, b.tile_incl, n_tiles, cap, ranges);
        static bool smem_set = false; // one opt-in per instantiation, above the 48 KB default
        if (!smem_set) {
            cudaFuncSetAttribute(k_chunk_emit<Grids>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(chunk_emit_smem()));
            smem_set = true;
        }
        k_chunk_emit<Grids><<<cgrid, kChunkThreads, chunk_emit_smem(), s>>>(b.pair_tile[spar], b.pair_val[spar], N, b.super_ranges, b.chunk_base, n_super,
            b.n_sort, rows, b.tile_total, b.tile_incl, cap, b.pair_tile[1 - spar], b.pair_val[1 - spar], stats, grids);
        note_launch(2);
    } else {
        cudaMemsetAsync(ranges, 0, size_t(n_tiles) * 2 * sizeof(int32_t), s);
    }
    return par;
}

template <class T>
inline int run_binning(uint32_t N, unsigned gx, unsigned gy, const uint32_t* tiles_touched, uint32_t* point_offsets, const int32_t* rects, const T* xy,
    uint32_t cap, BinningBuffers& b, int32_t* ranges, uint32_t* stats, int n_sms, cudaStream_t s, bool offsets_ready = false)
{
    return run_binning_grids<T>(N, gx * gy, super_count(gx, gy), SingleGrid { gx, gy }, tiles_touched, point_offsets, rects, xy, cap, b, ranges, stats, n_sms, s,
        offsets_ready);
}

} // namespace dgmr
