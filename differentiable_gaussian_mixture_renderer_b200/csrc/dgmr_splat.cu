// Tile-based EWA splat renderer: forward (src/dgmr/splat_forward.cu:30-338)
// and a reverse-order backward (no reference kernel), behind the C ABI of
// include/dgmr_b200.h.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <cuda_runtime.h>

#include "../../include/dgmr_b200.h"
#include "dgmr_abi_common.h"
#include "dgmr_batch.cuh"
#include "dgmr_binning.cuh"
#include "dgmr_device_grad.cuh"

namespace dgmr {

// Frame workspace: everything sized by the Gaussian count, tiles and pixels.
// Pair workspace: the (tile, Gaussian) pair buffers and sort scratch.
struct SplatLayout {
    int32_t* rects;
    float* rgb;
    uint8_t* clamped;
    float* depths;
    float* xy;
    float* conic_opacity;
    uint32_t* tiles_touched;
    uint32_t* point_offsets;
    int32_t* ranges;
    float* final_T;
    int32_t* n_contrib;
    double* grad_acc; // [N,9]: xy(2) conic(3) opacity rgb(3), summed over pixels in double
    float4* blend_rec; // [N,2]: (x, y, a, c), (2b, opacity, q_cut, 0) -- the blend's 32-byte record
    uint32_t* tile_order; // [tiles] launch order of the per-tile kernels, heaviest first
    uint32_t* tile_cost; // [tiles] predicted blend cost of each tile as a bucket, 0 = heaviest
    uint32_t* stats; // [4] used when the caller passes none
    BinningBuffers bin;
    size_t bytes; // frame workspace
    size_t pair_bytes; // pair workspace
};

// N Gaussians (or view-Gaussians of a batch), n_tiles tiles and n_px pixels
inline SplatLayout splat_layout_n(uint32_t N, uint32_t n_tiles, size_t n_px, uint32_t cap, void* base, void* pair_base)
{
    SplatLayout L;
    Carver c;
    c.base = static_cast<char*>(base);
    L.rects = c.take<int32_t>(size_t(N) * 2);
    L.rgb = c.take<float>(size_t(N) * 3);
    L.clamped = c.take<uint8_t>(size_t(N) * 3);
    L.depths = c.take<float>(N);
    L.xy = c.take<float>(size_t(N) * 2);
    L.conic_opacity = c.take<float>(size_t(N) * 4);
    L.tiles_touched = c.take<uint32_t>(N);
    L.point_offsets = c.take<uint32_t>(N);
    L.ranges = c.take<int32_t>(size_t(n_tiles) * 2);
    L.final_T = c.take<float>(n_px);
    L.n_contrib = c.take<int32_t>(n_px);
    L.grad_acc = c.take<double>(size_t(N) * 9);
    L.blend_rec = c.take<float4>(size_t(N) * 2);
    L.tile_order = c.take<uint32_t>(n_tiles);
    L.tile_cost = c.take<uint32_t>(n_tiles);
    L.stats = c.take<uint32_t>(4);
    carve_binning_gaussians(c, L.bin, N, n_tiles);
    L.bytes = c.off;
    Carver cp;
    cp.base = static_cast<char*>(pair_base);
    carve_binning_pairs(cp, L.bin, N, cap);
    L.pair_bytes = cp.off;
    return L;
}

inline SplatLayout splat_layout(uint32_t N, uint32_t W, uint32_t H, uint32_t cap, void* base, void* pair_base)
{
    const uint32_t gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
    return splat_layout_n(N, gx * gy, size_t(W) * H, cap, base, pair_base);
}

struct SplatPre {
    uint32_t N;
    const float* centroids;
    const float* sh;
    int sh_stride, sh_degree;
    const float* weights;
    const float* scales;
    const float* rotations;
    int32_t* rects;
    float* rgb;
    uint8_t* clamped;
    float* depths;
    float* xy;
    float* conic_opacity;
    uint32_t* tiles_touched;
    uint32_t* depth_key;
    uint32_t* perm;
    float4* blend_rec;
    Formulation form;
};

// splat_forward.cu:70-118 for Gaussian i of the scene, written to output
// slot o (o = i for one frame; o = the view's offset + i in a batch)
__device__ __forceinline__ void preprocess_one(const SplatPre& p, const CameraT<float>& cam, uint32_t i, uint32_t o)
{
    p.tiles_touched[o] = 0;
    p.perm[o] = o;
    p.depth_key[o] = 0;
    p.rects[2 * o] = 0;
    p.rects[2 * o + 1] = 0;
    p.xy[2 * o] = 0.f;
    p.xy[2 * o + 1] = 0.f;
    p.depths[o] = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        p.rgb[3 * o + c] = 0.f;
        p.clamped[3 * o + c] = 0;
    }
    reinterpret_cast<float4*>(p.conic_opacity)[o] = make_float4(0.f, 0.f, 0.f, 0.f);
    p.blend_rec[2 * o] = make_float4(0.f, 0.f, 0.f, 0.f);
    p.blend_rec[2 * o + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
    const V3<float> mu = { p.centroids[3 * i], p.centroids[3 * i + 1], p.centroids[3 * i + 2] };
    if (view_z(cam.view, mu) < 0.2f)
        return;
    const float w = p.weights[i];
    const V3<float> sc = mul3(V3<float> { p.scales[3 * i], p.scales[3 * i + 1], p.scales[3 * i + 2] }, cam.cov_scale_multiplier);
    const float* q = p.rotations + 4 * size_t(i);
    const M3<float> R = quat_to_mat3(q[0], q[1], q[2], q[3]);
    const Gaussian2d<float> g = splat_project(p.form, w, mu, sc, R, cam, 0.3f);
    const int ex = dgmr_fm::to_int_rz(dgmr_fm::ceil_f(3.f * dgmr_fm::sqrt_f(g.cov.v[0])));
    const int ey = dgmr_fm::to_int_rz(dgmr_fm::ceil_f(3.f * dgmr_fm::sqrt_f(g.cov.v[2])));
    p.rects[2 * o] = ex;
    p.rects[2 * o + 1] = ey;
    const TileRect r = get_rect(g.centroid.x, g.centroid.y, ex, ey, cam.gx, cam.gy);
    const unsigned touched = (r.x1 - r.x0) * (r.y1 - r.y0);
    if (touched == 0)
        return;
    p.tiles_touched[o] = touched;
    p.xy[2 * o] = g.centroid.x;
    p.xy[2 * o + 1] = g.centroid.y;
    const V3<float> campos = { cam.campos[0], cam.campos[1], cam.campos[2] };
    const float depth = len3(sub3(campos, mu));
    p.depths[o] = depth;
    p.depth_key[o] = __float_as_uint(depth);
    const V3<float> v = sub3(mu, campos);
    const V3<float> dir = mul3(v, 1.f / dgmr_fm::sqrt_f(dot3(v, v)));
    uint8_t mask[3];
    const V3<float> col = sh_to_colour(p.sh, i, p.sh_stride, p.sh_degree, dir, mask);
    p.rgb[3 * o] = col.x;
    p.rgb[3 * o + 1] = col.y;
    p.rgb[3 * o + 2] = col.z;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        p.clamped[3 * o + c] = mask[c];
    const S2<float> con = inverse2(g.cov);
    reinterpret_cast<float4*>(p.conic_opacity)[o] = make_float4(con.v[0], con.v[1], con.v[2], g.weight);
    // q_cut: any pixel with d'Qd > q_cut has opacity * exp(-d'Qd/2) < exp(-1e-3) / 255, i.e. alpha < 1/255
    // with a margin far above the rounding of the exponential, so the blend may skip it without changing
    // a single result
    const float q_cut = 2.f * (dgmr_fm::log_f(255.f * g.weight) + 1e-3f);
    p.blend_rec[2 * o] = make_float4(g.centroid.x, g.centroid.y, con.v[0], con.v[2]);
    p.blend_rec[2 * o + 1] = make_float4(2.f * con.v[1], g.weight, q_cut, 0.f);
}

__global__ void __launch_bounds__(256, 6) k_splat_preprocess(SplatPre p, CameraT<float> cam)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < p.N)
        preprocess_one(p, cam, i, i);
}

// d'Qd of one (pixel, splat) pair (splat_forward.cu:302), evaluated as
// dx * (a dx + 2b dy) + (c dy) dy with two fused multiply-adds; r0 = (x, y, a, c), b2 = 2b
__device__ __forceinline__ float splat_q(float4 r0, float b2, float px, float py, float* dx_o, float* dy_o)
{
    const float dx = px - r0.x;
    const float dy = py - r0.y;
    *dx_o = dx;
    *dy_o = dy;
    return __fmaf_rn(__fmaf_rn(r0.z, dx, b2 * dy), dx, (r0.w * dy) * dy);
}

// Per-pixel blend state of the pixel a thread owns (splat_forward.cu:299-321).
struct PixelState {
    float T, c0, c1, c2;
    int32_t last;
    bool done;
};

// One blend step after the cutoff test, given exp(-q/2)
// (splat_forward.cu:303-321): alpha = min(0.99, opacity * exp), skipped below
// 1/255; the pixel saturates (and keeps its state) once T * (1 - alpha) would
// drop below 1e-4.  Written as selects so that a warp can run it for every
// lane, whether or not the lane uses the record (`use`): the arithmetic and
// its order are the reference's, applied only where `use` holds.
__device__ __forceinline__ void blend_alpha_select(PixelState& ps, bool use, float ex, float opacity, float r, float g, float b, int32_t idx)
{
    const float alpha = min_f(0.99f, opacity * ex);
    const float test_T = ps.T * (1.f - alpha);
    const bool live = use && !ps.done && !(alpha < 1.0f / 255.0f);
    const bool stop = live && test_T < 0.0001f;
    const bool take = live && !stop;
    const float w = alpha * ps.T;
    ps.c0 = take ? __fmaf_rn(r, w, ps.c0) : ps.c0;
    ps.c1 = take ? __fmaf_rn(g, w, ps.c1) : ps.c1;
    ps.c2 = take ? __fmaf_rn(b, w, ps.c2) : ps.c2;
    ps.T = take ? test_T : ps.T;
    ps.last = take ? idx : ps.last;
    ps.done = ps.done || stop;
}

// Minimum of d'Qd over the tile's pixel rectangle [x0,x1] x [y0,y1] for a
// splat at (cx, cy) with conic (a, b, c): 0 if the centre is inside, else the
// minimum over the four edges (each a clamped 1-D quadratic).  Returns 0 (keep)
// for a conic that is not positive definite.  Only used to drop splats with a
// wide margin, so approximate division is fine here.
__device__ __forceinline__ float rect_min_q(float cx, float cy, float a, float b, float c, float x0, float x1, float y0, float y1)
{
    if (!(a > 0.f && c > 0.f && a * c - b * b > 0.f))
        return 0.f;
    if (cx >= x0 && cx <= x1 && cy >= y0 && cy <= y1)
        return 0.f;
    const auto q = [&](float dx, float dy) { return a * dx * dx + 2.f * b * dx * dy + c * dy * dy; };
    float m = 3.0e38f;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const float dx = (e == 0 ? x0 : x1) - cx;
        const float dy = fminf(fmaxf(cy - __fdividef(b * dx, c), y0), y1) - cy;
        m = fminf(m, q(dx, dy));
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const float dy = (e == 0 ? y0 : y1) - cy;
        const float dx = fminf(fmaxf(cx - __fdividef(b * dy, a), x0), x1) - cx;
        m = fminf(m, q(dx, dy));
    }
    return m;
}

// One 16x16 tile per block of 256 threads, one pixel per thread.  Each batch
// of up to 256 list entries is loaded one per thread; splats whose cutoff
// ellipse cannot reach the tile are dropped (an exact rectangle minimum with a
// margin, so no pixel that could pass its own cutoff test loses a splat); the
// rest are compacted in list order into shared memory as 32-byte records and
// evaluated by every pixel.  The block stops when every pixel is saturated.
// The kernel's duration is set by its slowest tile (a few tiles with ~2-3k
// unsaturated entries run from the first wave to the end), so a tile's
// pixels are spread over as many threads as it has pixels: two pixels per
// thread made that critical path, and the launch, 12 % longer.

// A single frame: every tile is one of its tiles.
struct SingleFrame {
    unsigned W, H, gx;
    float bg0, bg1, bg2;
    float* fb;
    float* final_T;
    int32_t* n_contrib;
    const float* grad_fb;
    __device__ __forceinline__ FrameRef frame(uint32_t tile) const { return FrameRef { W, H, gx, tile, bg0, bg1, bg2, fb, final_T, n_contrib, grad_fb }; }
};

// Block shapes of the blend: a 16x16 tile per block of 256 threads, or an 8x8
// quarter of a tile per block of 64 threads (four blocks walk the same tile
// list, each culling against its own quarter and stopping when its own pixels
// are saturated; every pixel sees the same records in the same order, so the
// results are the same bits).  __launch_bounds__ keeps both at 48 registers:
// for 16x16, five blocks per SM instead of four at the 52 the compiler picks
// unbounded -- 3 % shorter launches over 8 cameras at 1080p/1M, +2.3 % served
// renders/s.
template <int kSide>
struct BlendShape {
    static_assert(kSide == 16 || kSide == 8, "blend blocks of 16x16 or 8x8 pixels");
    static constexpr int kThreads = kSide * kSide;
    static constexpr int kMinBlocks = kSide == 16 ? 5 : 20;
    static constexpr int kPerTile = (int(kTile) / kSide) * (int(kTile) / kSide); // blocks per 16x16 tile
};

template <int kSide, class Frames>
__global__ void __launch_bounds__(BlendShape<kSide>::kThreads, BlendShape<kSide>::kMinBlocks) k_splat_blend(const int32_t* __restrict__ ranges,
    const uint32_t* __restrict__ list, const float4* __restrict__ rec, const float* __restrict__ rgb, uint32_t N, uint32_t cap, uint32_t* __restrict__ stats,
    const uint32_t* __restrict__ tile_order, const __grid_constant__ Frames frames)
{
    constexpr int kThreads = BlendShape<kSide>::kThreads;
    constexpr int kPerTile = BlendShape<kSide>::kPerTile;
    constexpr int kBatch = kThreads;
    constexpr int kWarps = kThreads / 32;
    constexpr int kGroup = 4;
    static_assert(kBatch % kGroup == 0, "a group never reads past the batch");
    __shared__ float4 s_r0[kBatch];
    __shared__ float4 s_r1[kBatch]; // (2b, opacity, q_cut, 1-based list index as int bits)
    __shared__ float4 s_rgb[kBatch]; // (r, g, b, .): one 16-byte load per record that a warp blends
    __shared__ int s_warp_tot[kWarps];
    const unsigned slot = blockIdx.x / kPerTile, part = blockIdx.x % kPerTile;
    const unsigned tile = tile_order ? tile_order[slot] : slot;
    const FrameRef f = frames.frame(tile);
    const unsigned W = f.W, H = f.H;
    const unsigned tx = f.tile % f.gx, ty = f.tile / f.gx;
    // the block's pixels start at (ox, oy) of the tile; warp w covers the 8x4
    // pixel block (8 (w % kRow), 4 (w / kRow)) of them: a compact footprint, so
    // fewer records pass some lane's cutoff than over a 16x2 strip (a record
    // no lane needs costs one vote)
    constexpr unsigned kRow = unsigned(kSide) / 8u;
    const unsigned ox = unsigned(kSide) * (part % (kTile / unsigned(kSide))), oy = unsigned(kSide) * (part / (kTile / unsigned(kSide)));
    const unsigned wb = threadIdx.x >> 5;
    const unsigned px = tx * kTile + ox + 8u * (wb % kRow) + (threadIdx.x & 7u);
    const unsigned py = ty * kTile + oy + 4u * (wb / kRow) + ((threadIdx.x >> 3) & 3u);
    PixelState p0 { 1.f, 0.f, 0.f, 0.f, 0, !(px < W && py < H) };
    const bool in0 = !p0.done;
    int32_t b = ranges[2 * tile], e = ranges[2 * tile + 1];
    if (b < 0 || e < b || uint32_t(e) > cap) {
        if (threadIdx.x == 0)
            flag_bounds(stats, 0x31u);
        b = e = 0;
    }
    const float fx0 = float(tx * kTile + ox), fx1 = fx0 + float(kSide - 1), fy0 = float(ty * kTile + oy), fy1 = fy0 + float(kSide - 1);
    const float fpx = float(px), fpy = float(py);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int32_t base = b; base < e; base += kBatch) {
        if (__syncthreads_count(p0.done) == kThreads)
            break;
        float4 r0, r1;
        uint32_t id = 0xffffffffu;
        int keep = 0;
        {
            const int32_t k = base + int(threadIdx.x);
            if (k < e) {
                uint32_t g = list[k];
                if (g >= N) {
                    flag_bounds(stats, 0x32u);
                    g = 0;
                }
                r0 = rec[2 * size_t(g)];
                r1 = rec[2 * size_t(g) + 1];
                const float qmin = rect_min_q(r0.x, r0.y, r0.z, 0.5f * r1.x, r0.w, fx0, fx1, fy0, fy1);
                if (!(qmin > r1.z * 1.001f + 0.01f)) {
                    id = g;
                    r1.w = __int_as_float(k - b + 1);
                    keep = 1;
                }
            }
        }
        // order-preserving compaction: warp ballot, then the warps' totals in order
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0)
            s_warp_tot[warp] = __popc(m);
        __syncthreads();
        int slot = __popc(m & ((1u << lane) - 1u));
        int n = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const int t = s_warp_tot[w];
            slot += (w < warp) ? t : 0;
            n += t;
        }
        if (keep) {
            s_r0[slot] = r0;
            s_r1[slot] = r1;
            s_rgb[slot] = make_float4(rgb[3 * size_t(id)], rgb[3 * size_t(id) + 1], rgb[3 * size_t(id) + 2], 0.f);
        }
        // the slots after the last record up to the group boundary: a cutoff below
        // every quadratic form (q = 0 here), so no lane ever uses them
        if (int(threadIdx.x) < kGroup - 1 && n + int(threadIdx.x) < kBatch) {
            s_r0[n + threadIdx.x] = make_float4(0.f, 0.f, 0.f, 0.f);
            s_r1[n + threadIdx.x] = make_float4(0.f, 0.f, -1.f, 0.f);
        }
        __syncthreads();
        if (!__all_sync(0xffffffffu, p0.done)) {
            // kGroup records at a time, with control flow that is uniform over
            // the warp: the group's quadratic forms (independent, so their
            // shared-memory loads and multiply-adds overlap), then, in list
            // order, the exp and the blend step (as selects) of each record
            // that some lane's cutoff admits; a record no lane needs costs a
            // vote, and the warp leaves once all its pixels are saturated.
            for (int j = 0; j < n; j += kGroup) {
                float q[kGroup];
                bool u[kGroup];
#pragma unroll
                for (int i = 0; i < kGroup; ++i) {
                    const float4 a0 = s_r0[j + i], a1 = s_r1[j + i]; // j + i < kBatch (kBatch % kGroup == 0)
                    float dx, dy;
                    q[i] = splat_q(a0, a1.x, fpx, fpy, &dx, &dy);
                    u[i] = !(q[i] > a1.z) && !p0.done;
                }
#pragma unroll
                for (int i = 0; i < kGroup; ++i) {
                    if (!__any_sync(0xffffffffu, u[i]))
                        continue;
                    const float ex = u[i] ? dgmr_fm::exp_f_nonpos(-0.5f * q[i]) : 0.f;
                    const float4 a1 = s_r1[j + i];
                    const float4 c = s_rgb[j + i];
                    blend_alpha_select(p0, u[i], ex, a1.y, c.x, c.y, c.z, __float_as_int(a1.w));
                }
                if (__all_sync(0xffffffffu, p0.done))
                    break;
            }
        }
        __syncthreads();
    }
    const size_t plane = size_t(W) * H;
    if (in0) {
        const size_t pix = size_t(py) * W + px;
        f.fb[pix] = p0.c0 + p0.T * f.bg0;
        f.fb[plane + pix] = p0.c1 + p0.T * f.bg1;
        f.fb[2 * plane + pix] = p0.c2 + p0.T * f.bg2;
        f.final_T[pix] = p0.T;
        f.n_contrib[pix] = p0.last;
    }
}

// The blend over n_tiles tiles with blocks of side x side pixels (16 or 8).
// Single frames use 8x8 blocks: at 1080p with 1M Gaussians the blend takes
// 0.1725 ms against 0.198 ms with 16x16 blocks (the same bits); batches take
// the side from their views (dgmr_batch_view.blend_block).
constexpr int kBlendSide = 8;
template <class Frames>
void launch_blend(int side, uint32_t n_tiles, const int32_t* ranges, const uint32_t* list, const float4* rec, const float* rgb, uint32_t N, uint32_t cap,
    uint32_t* stats, const uint32_t* tile_order, const Frames& frames, cudaStream_t s)
{
    if (n_tiles == 0)
        return;
    if (side == 8)
        k_splat_blend<8, Frames><<<n_tiles * BlendShape<8>::kPerTile, BlendShape<8>::kThreads, 0, s>>>(ranges, list, rec, rgb, N, cap, stats, tile_order, frames);
    else
        k_splat_blend<16, Frames><<<n_tiles, BlendShape<16>::kThreads, 0, s>>>(ranges, list, rec, rgb, N, cap, stats, tile_order, frames);
    note_launch();
}

// Sums of 9 per-lane values over a warp, scattered: halve the slots each lane
// holds at every butterfly level (16 -> 8 -> 4 -> 2 -> 1, the upper half kept
// by the lanes whose level bit is set), then add the partner's copy.  Lane l
// returns the warp total of slot 8 b4 + 4 b3 + 2 b2 + b1 (b = the bits of l;
// slots 9..15 are zero).
__device__ __forceinline__ float warp_reduce_scatter9(const float (&v)[9], int lane)
{
    float a[16];
#pragma unroll
    for (int q = 0; q < 16; ++q)
        a[q] = q < 9 ? v[q] : 0.f;
#pragma unroll
    for (int half = 8; half >= 1; half >>= 1) {
        const int bit = half * 2; // the xor distance: 16, 8, 4, 2
        const bool upper = (lane & bit) != 0;
#pragma unroll
        for (int q = 0; q < half; ++q) {
            const float give = upper ? a[q] : a[q + half];
            const float keep = upper ? a[q + half] : a[q];
            a[q] = keep + __shfl_xor_sync(0xffffffffu, give, bit);
        }
    }
    return a[0] + __shfl_xor_sync(0xffffffffu, a[0], 1);
}

// Reverse-order blend adjoint: each pixel walks its contributors back to
// front, recovering T_i = T_{i+1} / (1 - alpha_i); per-splat gradients are
// summed over the warp with shuffles before one atomic per value.  Tiles run
// in the forward's launch order (heaviest predicted walk first): a tile's
// backward walks the same list up to its last contributor.
// The block shapes of the forward (BlendShape): with 8x8 blocks each block
// walks only up to the last contributor of its own 64 pixels.
// __launch_bounds__: 48 registers (for 16x16, instead of 53: five blocks per
// SM instead of four, backward 2-3 % shorter at 1080p/1M and 200k/1024^2).
template <int kSide, class Frames>
__global__ void __launch_bounds__(BlendShape<kSide>::kThreads, BlendShape<kSide>::kMinBlocks) k_splat_bwd_pixels(const int32_t* __restrict__ ranges,
    const uint32_t* __restrict__ list, const float4* __restrict__ rec, const float* __restrict__ rgb, double* __restrict__ acc,
    const uint32_t* __restrict__ tile_order, const __grid_constant__ Frames frames)
{
    constexpr int kThreads = BlendShape<kSide>::kThreads;
    constexpr int kPerTile = BlendShape<kSide>::kPerTile;
    constexpr int kWarps = kThreads / 32;
    __shared__ float4 s_r0[kThreads]; // the blend records: (x, y, a, c), (2b, opacity, q_cut, list index as int bits)
    __shared__ float4 s_r1[kThreads];
    __shared__ float s_rgb[3][kThreads];
    __shared__ uint32_t s_id[kThreads];
    __shared__ int s_warp_tot[kWarps];
    __shared__ int s_max;
    const unsigned slot = blockIdx.x / kPerTile, part = blockIdx.x % kPerTile, n_tiles = gridDim.x / kPerTile;
    const unsigned ordered = tile_order ? tile_order[slot] : slot;
    const unsigned tile = ordered < n_tiles ? ordered : slot; // the order is a permutation of the tiles
    const FrameRef f = frames.frame(tile);
    if (!f.grad_fb) // a view without an image gradient (batched renders that only asked for the image)
        return;
    const unsigned W = f.W, H = f.H;
    const unsigned tx = f.tile % f.gx, ty = f.tile / f.gx;
    // the forward's pixel blocks: the block's pixels start at (ox, oy) of the
    // tile, warp w covers the 8x4 block (8 (w % kRow), 4 (w / kRow)) of them
    constexpr unsigned kRow = unsigned(kSide) / 8u;
    const unsigned ox = unsigned(kSide) * (part % (kTile / unsigned(kSide))), oy = unsigned(kSide) * (part / (kTile / unsigned(kSide)));
    const unsigned wb = threadIdx.x >> 5;
    const unsigned px = tx * kTile + ox + 8u * (wb % kRow) + (threadIdx.x & 7u);
    const unsigned py = ty * kTile + oy + 4u * (wb / kRow) + ((threadIdx.x >> 3) & 3u);
    const bool inside = px < W && py < H;
    const int32_t b = ranges[2 * tile];
    const size_t pix = size_t(py) * W + px;
    const int32_t my_n = inside ? f.n_contrib[pix] : 0;
    if (threadIdx.x == 0)
        s_max = 0;
    __syncthreads();
    atomicMax(&s_max, my_n);
    __syncthreads();
    const int32_t max_n = s_max;
    float g0 = 0.f, g1 = 0.f, g2 = 0.f, Tf = 1.f;
    if (inside) {
        g0 = f.grad_fb[pix];
        g1 = f.grad_fb[size_t(W) * H + pix];
        g2 = f.grad_fb[2 * size_t(W) * H + pix];
        Tf = f.final_T[pix];
    }
    const float bg_dot = (f.bg0 * g0 + f.bg1 * g1) + f.bg2 * g2;
    float Tr = Tf;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f; // accumulated colour behind the current splat
    const float fpx = float(px), fpy = float(py);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float fx0 = float(tx * kTile + ox), fx1 = fx0 + float(kSide - 1), fy0 = float(ty * kTile + oy), fy1 = fy0 + float(kSide - 1);
    for (int32_t hi = max_n; hi > 0; hi -= kThreads) {
        const int32_t lo = hi > kThreads ? hi - kThreads : 0;
        __syncthreads();
        // the batch's records that can reach a pixel of this block (the
        // forward's exact rectangle cull), compacted in list order with their
        // list positions; the others add nothing to any pixel here
        const int32_t k = lo + int32_t(threadIdx.x);
        uint32_t id = 0;
        float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0;
        int keep = 0;
        if (k < hi) {
            id = list[b + k];
            r0 = rec[2 * size_t(id)];
            r1 = rec[2 * size_t(id) + 1];
            const float qmin = rect_min_q(r0.x, r0.y, r0.z, 0.5f * r1.x, r0.w, fx0, fx1, fy0, fy1);
            keep = !(qmin > r1.z * 1.001f + 0.01f);
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0)
            s_warp_tot[warp] = __popc(m);
        __syncthreads();
        int pos = __popc(m & ((1u << lane) - 1u));
        int n = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const int t = s_warp_tot[w];
            pos += (w < warp) ? t : 0;
            n += t;
        }
        if (keep) {
            r1.w = __int_as_float(k);
            s_id[pos] = id;
            s_r0[pos] = r0;
            s_r1[pos] = r1;
            s_rgb[0][pos] = rgb[3 * size_t(id)];
            s_rgb[1][pos] = rgb[3 * size_t(id) + 1];
            s_rgb[2][pos] = rgb[3 * size_t(id) + 2];
        }
        __syncthreads();
        for (int j = n - 1; j >= 0; --j) {
            float v[9] = { 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f };
            bool any = false;
            const float4 r0 = s_r0[j], r1 = s_r1[j];
            const int32_t kk = __float_as_int(r1.w);
            float dx, dy;
            const float q = splat_q(r0, r1.x, fpx, fpy, &dx, &dy);
            // the forward's cutoff: past q_cut alpha < 1/255, so exp is not
            // needed; a record no lane of the warp needs costs one vote
            const bool need = kk < my_n && !(q > r1.z);
            if (!__any_sync(0xffffffffu, need))
                continue;
            if (need) {
                const float4 co = make_float4(r0.z, 0.5f * r1.x, r0.w, r1.y); // conic a, b, c and opacity
                const float g = dgmr_fm::exp_f_nonpos(-0.5f * q);
                const float alpha = min_f(0.99f, co.w * g);
                if (!(alpha < 1.0f / 255.0f)) {
                    any = true;
                    // T before this splat, and the background term's 1 / (1 - alpha): one reciprocal
                    const float inv = 1.f / (1.f - alpha);
                    Tr = Tr * inv;
                    const float c0 = s_rgb[0][j], c1 = s_rgb[1][j], c2 = s_rgb[2][j];
                    const float aT = alpha * Tr;
                    v[6] = aT * g0;
                    v[7] = aT * g1;
                    v[8] = aT * g2;
                    const float g_alpha = Tr * (((c0 - a0) * g0 + (c1 - a1) * g1) + (c2 - a2) * g2) - (Tf * bg_dot) * inv;
                    a0 = alpha * c0 + (1.f - alpha) * a0;
                    a1 = alpha * c1 + (1.f - alpha) * a1;
                    a2 = alpha * c2 + (1.f - alpha) * a2;
                    if (co.w * g < 0.99f) {
                        v[5] = g_alpha * g;
                        const float g_q = -0.5f * g * (g_alpha * co.w);
                        v[2] = g_q * dx * dx;
                        v[3] = g_q * 2.f * dx * dy;
                        v[4] = g_q * dy * dy;
                        v[0] = -(g_q * (2.f * co.x * dx + 2.f * co.y * dy));
                        v[1] = -(g_q * (2.f * co.z * dy + 2.f * co.y * dx));
                    }
                }
            }
            if (__any_sync(0xffffffffu, any)) {
                // reduce-scatter of the 9 partials over the warp (16 shuffles, not
                // 9 x 5): lane l ends with the warp's sum of partial slot(l) and
                // the lanes of slots 0..8 add them, one atomic each.  The totals
                // over warps are double: in float, the order in which the
                // atomics of many cancelling terms land moved single elements by
                // ~1e-3 relative from run to run at 200k Gaussians, 1024^2.
                float w = warp_reduce_scatter9(v, lane);
                const int slot = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
                if ((lane & 1) == 0 && slot < 9 && w != 0.f)
                    atomicAdd(acc + size_t(s_id[j]) * 9 + slot, double(w));
            }
        }
    }
}

// The per-pixel adjoint over n_tiles tiles with the forward's block shape.
template <class Frames>
void launch_blend_bwd(int side, uint32_t n_tiles, const int32_t* ranges, const uint32_t* list, const float4* rec, const float* rgb, double* acc,
    const uint32_t* tile_order, const Frames& frames, cudaStream_t s)
{
    if (n_tiles == 0)
        return;
    if (side == 8)
        k_splat_bwd_pixels<8, Frames><<<n_tiles * BlendShape<8>::kPerTile, BlendShape<8>::kThreads, 0, s>>>(ranges, list, rec, rgb, acc, tile_order, frames);
    else
        k_splat_bwd_pixels<16, Frames><<<n_tiles, BlendShape<16>::kThreads, 0, s>>>(ranges, list, rec, rgb, acc, tile_order, frames);
}

struct SplatBwdGauss {
    uint32_t N;
    const float* centroids;
    const float* sh;
    int sh_stride, sh_degree;
    const float* weights;
    const float* scales;
    const float* rotations;
    const uint8_t* clamped;
    const uint32_t* tiles_touched;
    const double* acc;
    float* g_sh;
    float* g_weights;
    float* g_centroids;
    float* g_scales;
    float* g_rotations;
    Formulation form;
};

__device__ __forceinline__ void zero_gaussian_grads(const SplatBwdGauss& p, uint32_t i)
{
    for (int k = 0; k < p.sh_stride * 3; ++k)
        p.g_sh[size_t(i) * p.sh_stride * 3 + k] = 0.f;
    p.g_weights[i] = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p.g_centroids[3 * i + k] = 0.f;
        p.g_scales[3 * i + k] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
        p.g_rotations[4 * i + k] = 0.f;
}

// per-Gaussian chain rule: conic -> 2-D covariance -> projection adjoint, SH.
// Gaussian i of the scene, per-view state at slot o; the result is added to
// the (zeroed) gradient rows of i, so several views of one scene sum up.
__device__ __forceinline__ void bwd_gaussian_one(const SplatBwdGauss& p, const CameraT<float>& cam, uint32_t i, uint32_t o)
{
    if (p.tiles_touched[o] == 0)
        return;
    float a[9];
#pragma unroll
    for (int k = 0; k < 9; ++k)
        a[k] = float(p.acc[size_t(o) * 9 + k]);
    const V3<float> mu = { p.centroids[3 * i], p.centroids[3 * i + 1], p.centroids[3 * i + 2] };
    const V3<float> sc = mul3(V3<float> { p.scales[3 * i], p.scales[3 * i + 1], p.scales[3 * i + 2] }, cam.cov_scale_multiplier);
    const float* q = p.rotations + 4 * size_t(i);
    const M3<float> R = quat_to_mat3(q[0], q[1], q[2], q[3]);
    const Gaussian2d<float> g2 = splat_project(p.form, p.weights[i], mu, sc, R, cam, 0.3f);
    const S2<float> M = inverse2(g2.cov);
    const float G00 = a[2], G01 = a[3] * 0.5f, G11 = a[4];
    // H = -M G M (2x2 symmetric)
    const float MG00 = M.v[0] * G00 + M.v[1] * G01, MG01 = M.v[0] * G01 + M.v[1] * G11;
    const float MG10 = M.v[1] * G00 + M.v[2] * G01, MG11 = M.v[1] * G01 + M.v[2] * G11;
    const float H00 = -(MG00 * M.v[0] + MG01 * M.v[1]);
    const float H01 = -(MG00 * M.v[1] + MG01 * M.v[2]);
    const float H11 = -(MG10 * M.v[1] + MG11 * M.v[2]);
    const S2<float> g_cov = { { H00, 2.f * H01, H11 } };
    float g_weight = 0.f;
    V3<float> g_mu = { 0.f, 0.f, 0.f }, g_s = { 0.f, 0.f, 0.f };
    float g_q[4] = { 0.f, 0.f, 0.f, 0.f };
    grad_splat(p.form, p.weights[i], mu, sc, q[0], q[1], q[2], q[3], cam, 0.3f, a[5], V2<float> { a[0], a[1] }, g_cov, &g_weight, &g_mu, &g_s, g_q);
    const V3<float> campos = { cam.campos[0], cam.campos[1], cam.campos[2] };
    const V3<float> v = sub3(mu, campos);
    const float vl = dgmr_fm::sqrt_f(dot3(v, v));
    const V3<float> dir = mul3(v, 1.f / vl);
    const V3<float> g_dir = grad_sh_to_colour(p.sh, i, p.sh_stride, p.sh_degree, dir, V3<float> { a[6], a[7], a[8] }, p.clamped + 3 * size_t(o), 0.f, p.g_sh,
        true);
    const float gd = dot3(g_dir, dir);
    g_mu = add3(g_mu, mul3(sub3(g_dir, mul3(dir, gd)), 1.f / vl));
    p.g_weights[i] += g_weight;
    p.g_centroids[3 * i] += g_mu.x;
    p.g_centroids[3 * i + 1] += g_mu.y;
    p.g_centroids[3 * i + 2] += g_mu.z;
    p.g_scales[3 * i] += g_s.x * cam.cov_scale_multiplier;
    p.g_scales[3 * i + 1] += g_s.y * cam.cov_scale_multiplier;
    p.g_scales[3 * i + 2] += g_s.z * cam.cov_scale_multiplier;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        p.g_rotations[4 * i + k] += g_q[k];
}

__global__ void __launch_bounds__(128) k_splat_bwd_gaussians(SplatBwdGauss p, CameraT<float> cam)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.N)
        return;
    zero_gaussian_grads(p, i);
    bwd_gaussian_one(p, cam, i, i);
}

} // namespace dgmr

using namespace dgmr;

namespace {

bool bad_sizes(int32_t n, int32_t w, int32_t h, int64_t cap)
{
    return n < 0 || w <= 0 || h <= 0 || w > 65536 || h > 65536 || cap < 0 || cap > int64_t(0x7fffffff);
}

SplatPre make_pre(const dgmr_scene* scene, const SplatLayout& L)
{
    return SplatPre { uint32_t(scene->n_gaussians), static_cast<const float*>(scene->centroids), static_cast<const float*>(scene->sh), scene->sh_stride,
        scene->sh_degree, static_cast<const float*>(scene->weights), static_cast<const float*>(scene->scales), static_cast<const float*>(scene->rotations),
        L.rects, L.rgb, L.clamped, L.depths, L.xy, L.conic_opacity, L.tiles_touched, L.bin.depth_key, L.bin.perm, L.blend_rec,
        scene_formulation(scene, Formulation::Ots) };
}

SingleFrame single_frame(const CameraT<float>& cam, float* fb, const SplatLayout& L, const float* grad_fb = nullptr)
{
    return SingleFrame { cam.W, cam.H, cam.gx, cam.bg[0], cam.bg[1], cam.bg[2], fb, L.final_T, L.n_contrib, grad_fb };
}

// per-Gaussian preprocess and the inclusive scan (splat_forward.cu:70-139)
void launch_preprocess(const dgmr_scene* scene, const CameraT<float>& cam, const SplatLayout& L, uint32_t* st_dev, cudaStream_t s)
{
    const uint32_t N = uint32_t(scene->n_gaussians);
    cudaMemsetAsync(st_dev, 0, 16, s);
    if (N == 0)
        return;
    k_splat_preprocess<<<(N + 255) / 256, 256, 0, s>>>(make_pre(scene, L), cam);
    note_launch();
    inclusive_scan_u32(L.tiles_touched, L.point_offsets, N, L.bin.scan_tmp, s);
}

// Launch order of the blend's tiles, heaviest first, from a predicted cost
// (scheduling only: results never depend on it).  A tile's block walks its
// list until every pixel is saturated, so the cost is the list length L for a
// tile that some pixel never saturates, and far less for one that is densely
// covered: the longest lists belong to dense tiles that saturate within a few
// hundred entries, and ordering by length alone starts the truly slow tiles
// late.  From the first 128 entries of its list, one warp per tile estimates
// the coverage of each 8x8 quadrant (summed opacity of the splats whose cutoff
// ellipse holds the quadrant's centre pixel, per entry); the least covered
// quadrant inside the frame sets the walk: cost = min(L, 100 / density), kept
// as a bucket of a quarter octave (0 = heaviest).  The last block to finish
// (counter n_sort[6], zeroed by the binning) counting-sorts the tiles by bucket
// with warp-aggregated shared atomics (most tiles share the "empty" bucket)
// and resets the counter.  On 1080p frames of 1M Gaussians this order ends
// the blend 5-26 % sooner than ordering by list length.
constexpr int kCostBuckets = 128;
constexpr uint32_t kOrderWarps = 8;
constexpr uint32_t kOrderPerThread = 16; // buckets a thread of the last block loads at once

template <class Frames>
__global__ void __launch_bounds__(kOrderWarps * 32) k_blend_tile_order(const int32_t* __restrict__ ranges, const uint32_t* __restrict__ list,
    const float4* __restrict__ rec, uint32_t N, uint32_t cap, uint32_t n_tiles, uint32_t* __restrict__ bucket, uint32_t* __restrict__ blocks_done,
    uint32_t* __restrict__ order, const __grid_constant__ Frames frames)
{
    constexpr int kSample = 128;
    __shared__ uint32_t count[kCostBuckets];
    __shared__ uint32_t cursor[kCostBuckets];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31;
    const uint32_t tile = blockIdx.x * kOrderWarps + (threadIdx.x >> 5);
    if (tile < n_tiles) {
        const FrameRef f = frames.frame(tile);
        const int32_t b = ranges[2 * tile], e = ranges[2 * tile + 1];
        uint32_t bk = kCostBuckets - 1; // empty (or flagged by the blend): lightest
        if (b >= 0 && e > b && uint32_t(e) <= cap) {
            const unsigned tx = f.tile % f.gx, ty = f.tile / f.gx;
            const float x0 = float(tx * kTile), y0 = float(ty * kTile);
            const int n = min(e - b, kSample);
            float hit[4] = { 0.f, 0.f, 0.f, 0.f };
            // the sample's list entries, then their records, all requested
            // before the first is used (kSample / 32 entries per lane)
            constexpr int kPerLane = kSample / 32;
            uint32_t gs[kPerLane];
#pragma unroll
            for (int i = 0; i < kPerLane; ++i) {
                const int k = lane + 32 * i;
                gs[i] = k < n ? list[b + k] : 0xffffffffu;
            }
            float4 r0s[kPerLane], r1s[kPerLane];
#pragma unroll
            for (int i = 0; i < kPerLane; ++i) {
                const size_t g = gs[i] < N ? gs[i] : 0u;
                r0s[i] = rec[2 * g];
                r1s[i] = rec[2 * g + 1];
            }
#pragma unroll
            for (int i = 0; i < kPerLane; ++i) {
                if (gs[i] >= N)
                    continue;
                const float4 r0 = r0s[i], r1 = r1s[i];
#pragma unroll
                for (int qd = 0; qd < 4; ++qd) {
                    const float dx = x0 + ((qd & 1) ? 12.f : 4.f) - r0.x;
                    const float dy = y0 + ((qd & 2) ? 12.f : 4.f) - r0.y;
                    const float q = r0.z * dx * dx + r1.x * dx * dy + r0.w * dy * dy;
                    hit[qd] += q <= r1.z ? r1.y : 0.f;
                }
            }
#pragma unroll
            for (int qd = 0; qd < 4; ++qd)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                    hit[qd] += __shfl_xor_sync(0xffffffffu, hit[qd], o);
            float dmin = 3.0e38f;
#pragma unroll
            for (int qd = 0; qd < 4; ++qd)
                if (tx * kTile + ((qd & 1) ? 12u : 4u) < f.W && ty * kTile + ((qd & 2) ? 12u : 4u) < f.H)
                    dmin = fminf(dmin, hit[qd] / float(n));
            const float cost = dmin > 1.0e37f ? 0.f : fminf(float(e - b), 100.f / fmaxf(dmin, 1.0e-4f));
            const int level = int(4.f * __log2f(cost + 1.f));
            bk = uint32_t(kCostBuckets - 1 - min(max(level, 0), kCostBuckets - 1));
        }
        if (lane == 0)
            bucket[tile] = bk;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        is_last = atomicAdd(blocks_done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last)
        return;
    __threadfence();
    // counting sort by bucket: count every tile, an exclusive prefix over the
    // buckets, then scatter; each sweep loads kOrderPerThread buckets per
    // thread at once so that their latencies overlap
    const unsigned below = (1u << lane) - 1u;
    const uint32_t sweep = kOrderPerThread * blockDim.x;
    const auto load = [&](uint32_t s0, uint32_t (&bk)[kOrderPerThread]) {
#pragma unroll
        for (uint32_t i = 0; i < kOrderPerThread; ++i) {
            const uint32_t t = s0 + i * blockDim.x + threadIdx.x;
            bk[i] = t < n_tiles ? min(__ldcg(bucket + t), uint32_t(kCostBuckets - 1)) : 0xffffffffu;
        }
    };
    if (threadIdx.x < kCostBuckets)
        count[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t s0 = 0; s0 < n_tiles; s0 += sweep) {
        uint32_t bk[kOrderPerThread];
        load(s0, bk);
#pragma unroll
        for (uint32_t i = 0; i < kOrderPerThread; ++i) {
            const unsigned peers = __match_any_sync(0xffffffffu, bk[i]);
            if (bk[i] != 0xffffffffu && lane == __ffs(peers) - 1)
                atomicAdd(&count[bk[i]], uint32_t(__popc(peers)));
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) { // exclusive prefix of the counts, kCostBuckets / 32 per lane
        constexpr int kPer = kCostBuckets / 32;
        uint32_t v[kPer];
        uint32_t sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            v[k] = count[lane * kPer + k];
            sum += v[k];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t up = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += up;
        }
        uint32_t run = incl - sum;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            cursor[lane * kPer + k] = run;
            run += v[k];
        }
    }
    __syncthreads();
    for (uint32_t s0 = 0; s0 < n_tiles; s0 += sweep) {
        uint32_t bk[kOrderPerThread];
        load(s0, bk);
#pragma unroll
        for (uint32_t i = 0; i < kOrderPerThread; ++i) {
            const unsigned peers = __match_any_sync(0xffffffffu, bk[i]);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (bk[i] != 0xffffffffu && lane == leader)
                base = atomicAdd(&cursor[bk[i]], uint32_t(__popc(peers)));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (bk[i] != 0xffffffffu)
                order[base + uint32_t(__popc(peers & below))] = s0 + i * blockDim.x + threadIdx.x;
        }
    }
    if (threadIdx.x == 0)
        *blocks_done = 0u;
}

template <class Frames>
void launch_tile_order(const SplatLayout& L, int par, uint32_t N, uint32_t cap, uint32_t n_tiles, const Frames& frames, cudaStream_t s)
{
    if (n_tiles == 0)
        return;
    k_blend_tile_order<Frames><<<(n_tiles + kOrderWarps - 1) / kOrderWarps, kOrderWarps * 32, 0, s>>>(L.ranges, L.bin.pair_val[par], L.blend_rec, N, cap,
        n_tiles, L.tile_cost, L.bin.n_sort + 6, L.tile_order, frames);
    note_launch();
}

// binning (after the preprocess) and the blend
void launch_render(const dgmr_scene* scene, const CameraT<float>& cam, float* fb, SplatLayout& L, uint32_t cap, uint32_t* st_dev, cudaStream_t s)
{
    const uint32_t N = uint32_t(scene->n_gaussians);
    const int par
        = run_binning<float>(N, cam.gx, cam.gy, L.tiles_touched, L.point_offsets, L.rects, L.xy, cap, L.bin, L.ranges, st_dev, num_sms(), s, true);
    launch_tile_order(L, par, N, cap, cam.gx * cam.gy, single_frame(cam, fb, L), s);
    launch_blend(kBlendSide, cam.gx * cam.gy, L.ranges, L.bin.pair_val[par], L.blend_rec, L.rgb, N, cap, st_dev, L.tile_order, single_frame(cam, fb, L), s);
}

} // namespace

extern "C" {

size_t dgmr_splat_frame_workspace_size(int32_t n_gaussians, int32_t width, int32_t height)
{
    if (bad_sizes(n_gaussians, width, height, 0))
        return 0;
    return splat_layout(uint32_t(n_gaussians), uint32_t(width), uint32_t(height), 0, nullptr, nullptr).bytes;
}

size_t dgmr_splat_pair_workspace_size(int32_t n_gaussians, int64_t pair_capacity)
{
    if (bad_sizes(n_gaussians, 1, 1, pair_capacity))
        return 0;
    return splat_layout(uint32_t(n_gaussians), 1, 1, uint32_t(pair_capacity), nullptr, nullptr).pair_bytes;
}

dgmr_status dgmr_splat_workspace_views(int32_t n_gaussians, int32_t width, int32_t height, int64_t pair_capacity, void* frame_workspace,
    size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, dgmr_splat_views* views)
{
    if (!views || !frame_workspace || bad_sizes(n_gaussians, width, height, pair_capacity) || (pair_capacity > 0 && !pair_workspace))
        return DGMR_ERR_BAD_ARG;
    const uint32_t W = uint32_t(width), H = uint32_t(height);
    const SplatLayout L = splat_layout(uint32_t(n_gaussians), W, H, uint32_t(pair_capacity), frame_workspace, pair_workspace);
    if (frame_workspace_bytes < L.bytes || pair_workspace_bytes < L.pair_bytes)
        return DGMR_ERR_WORKSPACE;
    const uint32_t gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
    const int par = tile_sort_parity(super_count(gx, gy));
    views->rects = L.rects;
    views->rgb = L.rgb;
    views->rgb_sh_clamped = L.clamped;
    views->depths = L.depths;
    views->points_xy_image = L.xy;
    views->conic_opacity = L.conic_opacity;
    views->tiles_touched = reinterpret_cast<int32_t*>(L.tiles_touched);
    views->point_offsets = reinterpret_cast<int32_t*>(L.point_offsets);
    views->i_ranges = L.ranges;
    views->point_list = pair_workspace ? reinterpret_cast<int32_t*>(L.bin.pair_val[par]) : nullptr;
    views->point_list_tiles = pair_workspace ? L.bin.pair_tile[par] : nullptr;
    views->final_transmittance = L.final_T;
    views->n_contrib = L.n_contrib;
    return DGMR_OK;
}

dgmr_status dgmr_splat_preprocess(const dgmr_scene* scene, const dgmr_camera* camera, void* frame_workspace, size_t frame_workspace_bytes,
    dgmr_frame_stats* stats, dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, DGMR_F32);
    if (st != DGMR_OK)
        return st;
    if (!frame_workspace)
        return DGMR_ERR_BAD_ARG;
    const SplatLayout L = splat_layout(uint32_t(scene->n_gaussians), uint32_t(camera->width), uint32_t(camera->height), 0, frame_workspace, nullptr);
    if (frame_workspace_bytes < L.bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<float> cam = make_camera<float>(*camera);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    launch_preprocess(scene, cam, L, st_dev, s);
    if (scene->n_gaussians > 0) {
        k_pair_count<<<1, 1, 0, s>>>(L.point_offsets, uint32_t(scene->n_gaussians), 0xffffffffu, st_dev, L.bin.n_sort);
        note_launch();
    }
    return launch_status();
}

dgmr_status dgmr_splat_render(const dgmr_scene* scene, const dgmr_camera* camera, float* framebuffer, void* frame_workspace, size_t frame_workspace_bytes,
    void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, DGMR_F32);
    if (st != DGMR_OK)
        return st;
    if (!framebuffer || !frame_workspace || pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff) || (pair_capacity > 0 && !pair_workspace))
        return DGMR_ERR_BAD_ARG;
    SplatLayout L = splat_layout(uint32_t(scene->n_gaussians), uint32_t(camera->width), uint32_t(camera->height), uint32_t(pair_capacity), frame_workspace,
        pair_workspace);
    if (frame_workspace_bytes < L.bytes || pair_workspace_bytes < L.pair_bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<float> cam = make_camera<float>(*camera);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    launch_render(scene, cam, framebuffer, L, uint32_t(pair_capacity), st_dev, s);
    return launch_status();
}

dgmr_status dgmr_splat_forward(const dgmr_scene* scene, const dgmr_camera* camera, float* framebuffer, void* frame_workspace, size_t frame_workspace_bytes,
    void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, DGMR_F32);
    if (st != DGMR_OK)
        return st;
    if (!framebuffer || !frame_workspace || pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff) || (pair_capacity > 0 && !pair_workspace))
        return DGMR_ERR_BAD_ARG;
    SplatLayout L = splat_layout(uint32_t(scene->n_gaussians), uint32_t(camera->width), uint32_t(camera->height), uint32_t(pair_capacity), frame_workspace,
        pair_workspace);
    if (frame_workspace_bytes < L.bytes || pair_workspace_bytes < L.pair_bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<float> cam = make_camera<float>(*camera);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    launch_preprocess(scene, cam, L, st_dev, s);
    launch_render(scene, cam, framebuffer, L, uint32_t(pair_capacity), st_dev, s);
    return launch_status();
}

dgmr_status dgmr_splat_blend(const dgmr_camera* camera, int32_t n_gaussians, float* framebuffer, void* frame_workspace, size_t frame_workspace_bytes,
    void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_stream stream)
{
    if (!camera || !framebuffer || !frame_workspace || bad_sizes(n_gaussians, camera->width, camera->height, pair_capacity)
        || (pair_capacity > 0 && !pair_workspace))
        return DGMR_ERR_BAD_ARG;
    const SplatLayout L = splat_layout(uint32_t(n_gaussians), uint32_t(camera->width), uint32_t(camera->height), uint32_t(pair_capacity), frame_workspace,
        pair_workspace);
    if (frame_workspace_bytes < L.bytes || pair_workspace_bytes < L.pair_bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<float> cam = make_camera<float>(*camera);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int par = tile_sort_parity(super_count(cam.gx, cam.gy));
    launch_blend(kBlendSide, cam.gx * cam.gy, L.ranges, L.bin.pair_val[par], L.blend_rec, L.rgb, uint32_t(n_gaussians), uint32_t(pair_capacity), L.stats,
        L.tile_order, single_frame(cam, framebuffer, L), s);
    return launch_status();
}

dgmr_status dgmr_splat_backward(const dgmr_scene* scene, const dgmr_camera* camera, const float* grad_framebuffer, float* grad_sh, float* grad_weights,
    float* grad_centroids, float* grad_scales, float* grad_rotations, void* frame_workspace, size_t frame_workspace_bytes, void* pair_workspace,
    size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, DGMR_F32);
    if (st != DGMR_OK)
        return st;
    // per-Gaussian outputs may have no address when there are no Gaussians
    const bool grads_ok = scene->n_gaussians == 0 || (grad_sh && grad_weights && grad_centroids && grad_scales && grad_rotations);
    if (!grad_framebuffer || !grads_ok || !frame_workspace || pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff)
        || (pair_capacity > 0 && !pair_workspace))
        return DGMR_ERR_BAD_ARG;
    const uint32_t N = uint32_t(scene->n_gaussians);
    const SplatLayout L = splat_layout(N, uint32_t(camera->width), uint32_t(camera->height), uint32_t(pair_capacity), frame_workspace, pair_workspace);
    if (frame_workspace_bytes < L.bytes || pair_workspace_bytes < L.pair_bytes)
        return DGMR_ERR_WORKSPACE;
    if (N == 0)
        return DGMR_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const CameraT<float> cam = make_camera<float>(*camera);
    const int par = tile_sort_parity(super_count(cam.gx, cam.gy));
    cudaMemsetAsync(L.grad_acc, 0, size_t(N) * 9 * sizeof(double), s);
    launch_blend_bwd(kBlendSide, cam.gx * cam.gy, L.ranges, L.bin.pair_val[par], L.blend_rec, L.rgb, L.grad_acc, L.tile_order,
        single_frame(cam, nullptr, L, grad_framebuffer), s);
    SplatBwdGauss p { N, static_cast<const float*>(scene->centroids), static_cast<const float*>(scene->sh), scene->sh_stride, scene->sh_degree,
        static_cast<const float*>(scene->weights), static_cast<const float*>(scene->scales), static_cast<const float*>(scene->rotations), L.clamped,
        L.tiles_touched, L.grad_acc, grad_sh, grad_weights, grad_centroids, grad_scales, grad_rotations, scene_formulation(scene, Formulation::Ots) };
    k_splat_bwd_gaussians<<<(N + 127) / 128, 128, 0, s>>>(p, cam);
    note_launch(2);
    return launch_status();
}

} // extern "C"

// ---------------------------------------------------------------------------
// Batched multi-view rendering over the view table of dgmr_batch.cuh.

namespace dgmr {

__global__ void __launch_bounds__(256) k_batch_preprocess(SplatPre out, const __grid_constant__ BatchTable tab)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= tab.G)
        return;
    const uint32_t v = BatchTable::owner(tab.g_off, tab.n_views, g);
    const BatchView& bv = tab.views[v];
    const BatchScene& sc = tab.scenes[bv.scene];
    SplatPre p = out;
    p.N = sc.n;
    p.centroids = sc.centroids;
    p.sh = sc.sh;
    p.sh_stride = sc.sh_stride;
    p.sh_degree = sc.sh_degree;
    p.weights = sc.weights;
    p.scales = sc.scales;
    p.rotations = sc.rotations;
    p.form = sc.form;
    preprocess_one(p, bv.cam, g - tab.g_off[v], g);
}

// per scene Gaussian: zero its gradient rows, then add the chain rule of
// every view of its scene, in view order (deterministic, no atomics)
__global__ void __launch_bounds__(128) k_batch_bwd_gaussians(SplatBwdGauss state, const __grid_constant__ BatchTable tab)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= tab.scene_off[tab.n_scenes])
        return;
    const uint32_t s = BatchTable::owner(tab.scene_off, tab.n_scenes, k);
    const BatchScene& sc = tab.scenes[s];
    const uint32_t i = k - tab.scene_off[s];
    if (!sc.g_sh) // a scene entry without gradient outputs
        return;
    SplatBwdGauss p = state;
    p.N = sc.n;
    p.centroids = sc.centroids;
    p.sh = sc.sh;
    p.sh_stride = sc.sh_stride;
    p.sh_degree = sc.sh_degree;
    p.weights = sc.weights;
    p.scales = sc.scales;
    p.rotations = sc.rotations;
    p.g_sh = sc.g_sh;
    p.g_weights = sc.g_weights;
    p.g_centroids = sc.g_centroids;
    p.g_scales = sc.g_scales;
    p.g_rotations = sc.g_rotations;
    p.form = sc.form;
    zero_gaussian_grads(p, i);
    for (uint32_t q = sc.view_begin; q < sc.view_end; ++q) {
        const uint32_t v = tab.view_by_scene[q];
        if (tab.views[v].grad_fb)
            bwd_gaussian_one(p, tab.views[v].cam, i, tab.g_off[v] + i);
    }
}

} // namespace dgmr

namespace {

struct BatchPlan {
    BatchTable tab;
    SplatLayout L;
    size_t px_total;
    int blend_side; // the blend's block side (dgmr_batch_view.blend_block)
};

// Validates the batch and builds its table and workspace layout.  grads may be
// null (forward).  Bases may be null (size query).
dgmr_status make_batch(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, const dgmr_scene_grads* grads,
    int64_t pair_capacity, void* frame_ws, void* pair_ws, BatchPlan& plan)
{
    if (pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff))
        return DGMR_ERR_BAD_ARG;
    BatchTable& t = plan.tab;
    const dgmr_status st = build_batch_table(scenes, n_scenes, views, n_views, grads, Formulation::Ots, t);
    if (st != DGMR_OK)
        return st;
    const int side = views[0].blend_block;
    if (side != 0 && side != 8 && side != 16)
        return DGMR_ERR_BAD_ARG;
    for (int v = 1; v < n_views; ++v)
        if (views[v].blend_block != 0 && views[v].blend_block != side)
            return DGMR_ERR_BAD_ARG;
    plan.blend_side = side ? side : kBlendSide;
    plan.px_total = t.px_total;
    plan.L = splat_layout_n(t.G, t.n_tiles, plan.px_total, uint32_t(pair_capacity), frame_ws, pair_ws);
    t.final_T = plan.L.final_T;
    t.n_contrib = plan.L.n_contrib;
    return DGMR_OK;
}

SplatPre batch_pre(const SplatLayout& L, uint32_t G)
{
    return SplatPre { G, nullptr, nullptr, 1, 0, nullptr, nullptr, nullptr, L.rects, L.rgb, L.clamped, L.depths, L.xy, L.conic_opacity, L.tiles_touched,
        L.bin.depth_key, L.bin.perm, L.blend_rec, Formulation::Ots };
}

// need_pairs = false for the preprocess alone, which touches no pair buffer
dgmr_status batch_check_ws(const BatchPlan& plan, void* frame_ws, size_t frame_bytes, void* pair_ws, size_t pair_bytes, int64_t pair_capacity,
    bool need_pairs = true)
{
    if (!frame_ws || (need_pairs && pair_capacity > 0 && !pair_ws))
        return DGMR_ERR_BAD_ARG;
    if (frame_bytes < plan.L.bytes || (need_pairs && pair_bytes < plan.L.pair_bytes))
        return DGMR_ERR_WORKSPACE;
    return DGMR_OK;
}

void batch_preprocess(const BatchPlan& plan, uint32_t* st_dev, cudaStream_t s)
{
    const SplatLayout& L = plan.L;
    const uint32_t G = plan.tab.G;
    cudaMemsetAsync(st_dev, 0, 16, s);
    if (G == 0)
        return;
    k_batch_preprocess<<<(G + 255) / 256, 256, 0, s>>>(batch_pre(L, G), plan.tab);
    note_launch();
    inclusive_scan_u32(L.tiles_touched, L.point_offsets, G, L.bin.scan_tmp, s);
}

} // namespace

extern "C" {

dgmr_status dgmr_splat_batch_workspace_size(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, int64_t pair_capacity,
    size_t* frame_workspace_bytes, size_t* pair_workspace_bytes)
{
    if (!frame_workspace_bytes || !pair_workspace_bytes)
        return DGMR_ERR_BAD_ARG;
    static thread_local BatchPlan plan;
    const dgmr_status st = make_batch(scenes, n_scenes, views, n_views, nullptr, pair_capacity, nullptr, nullptr, plan);
    if (st != DGMR_OK)
        return st;
    *frame_workspace_bytes = plan.L.bytes;
    *pair_workspace_bytes = plan.L.pair_bytes;
    return DGMR_OK;
}

dgmr_status dgmr_splat_batch_preprocess(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, void* frame_workspace,
    size_t frame_workspace_bytes, dgmr_frame_stats* stats, dgmr_stream stream)
{
    static thread_local BatchPlan plan;
    dgmr_status st = make_batch(scenes, n_scenes, views, n_views, nullptr, 0, frame_workspace, nullptr, plan);
    if (st != DGMR_OK)
        return st;
    st = batch_check_ws(plan, frame_workspace, frame_workspace_bytes, nullptr, 0, 0, false);
    if (st != DGMR_OK)
        return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : plan.L.stats;
    batch_preprocess(plan, st_dev, s);
    if (plan.tab.G > 0) {
        k_pair_count<<<1, 1, 0, s>>>(plan.L.point_offsets, plan.tab.G, 0xffffffffu, st_dev, plan.L.bin.n_sort);
        note_launch();
    }
    return launch_status();
}

dgmr_status dgmr_splat_batch_forward(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, void* frame_workspace,
    size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream)
{
    static thread_local BatchPlan plan;
    dgmr_status st = make_batch(scenes, n_scenes, views, n_views, nullptr, pair_capacity, frame_workspace, pair_workspace, plan);
    if (st != DGMR_OK)
        return st;
    st = batch_check_ws(plan, frame_workspace, frame_workspace_bytes, pair_workspace, pair_workspace_bytes, pair_capacity);
    if (st != DGMR_OK)
        return st;
    for (int v = 0; v < n_views; ++v)
        if (!views[v].framebuffer)
            return DGMR_ERR_BAD_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    SplatLayout& L = plan.L;
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    const uint32_t G = plan.tab.G, cap = uint32_t(pair_capacity);
    batch_preprocess(plan, st_dev, s);
    const int par = run_binning_grids<float>(G, plan.tab.n_tiles, plan.tab.n_stiles, plan.tab, L.tiles_touched, L.point_offsets, L.rects, L.xy, cap, L.bin, L.ranges, st_dev,
        num_sms(), s, true);
    launch_tile_order(L, par, G, cap, plan.tab.n_tiles, plan.tab, s);
    launch_blend(plan.blend_side, plan.tab.n_tiles, L.ranges, L.bin.pair_val[par], L.blend_rec, L.rgb, G, cap, st_dev, L.tile_order, plan.tab, s);
    note_launch();
    return launch_status();
}

dgmr_status dgmr_splat_batch_backward(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views,
    const dgmr_scene_grads* grads, void* frame_workspace, size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes,
    int64_t pair_capacity, dgmr_stream stream)
{
    if (!grads)
        return DGMR_ERR_BAD_ARG;
    static thread_local BatchPlan plan;
    dgmr_status st = make_batch(scenes, n_scenes, views, n_views, grads, pair_capacity, frame_workspace, pair_workspace, plan);
    if (st != DGMR_OK)
        return st;
    st = batch_check_ws(plan, frame_workspace, frame_workspace_bytes, pair_workspace, pair_workspace_bytes, pair_capacity);
    if (st != DGMR_OK)
        return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const SplatLayout& L = plan.L;
    const uint32_t G = plan.tab.G;
    const uint32_t n_scene_gaussians = plan.tab.scene_off[n_scenes];
    if (n_scene_gaussians == 0)
        return DGMR_OK;
    const int par = tile_sort_parity(plan.tab.n_stiles);
    cudaMemsetAsync(L.grad_acc, 0, size_t(G) * 9 * sizeof(double), s);
    launch_blend_bwd(plan.blend_side, plan.tab.n_tiles, L.ranges, L.bin.pair_val[par], L.blend_rec, L.rgb, L.grad_acc, L.tile_order, plan.tab, s);
    SplatBwdGauss state { 0, nullptr, nullptr, 1, 0, nullptr, nullptr, nullptr, L.clamped, L.tiles_touched, L.grad_acc, nullptr, nullptr, nullptr, nullptr,
        nullptr, Formulation::Ots };
    k_batch_bwd_gaussians<<<(n_scene_gaussians + 127) / 128, 128, 0, s>>>(state, plan.tab);
    note_launch(2);
    return launch_status();
}

} // extern "C"

// ---------------------------------------------------------------------------
// Splat forward without any device allocation.
//
// Some callers cannot hand this library a workspace: a plugin inside a host
// application that owns every byte of GPU memory through its own pool, or
// code running in a per-frame callback where a cudaMalloc would synchronise
// the whole device and stall everything else in flight.  For them the frame
// and pair workspaces live in one fixed-size array in device memory, defined
// below, which every GPU that loads this library keeps until the process
// exits.  A call whose two workspaces do not fit is rejected with
// DGMR_ERR_STATIC_SCRATCH; nothing else is allocated.
//
// The array is shared by every call on a device and keeps whatever the last
// call left in it.  The forward writes everything it later reads (the frame
// statistics and tile ranges are cleared on the stream at the start of each
// frame), so consecutive calls are independent -- but two calls that overlap
// on the GPU (different streams, no ordering between them) race on the array
// and corrupt each other's frame.

namespace {

constexpr size_t kStaticScratchBytes = size_t(64) << 20; // 64 MiB per device

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_mutex;
void* g_static_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  Host code must
// not pass g_static_scratch itself to a kernel: on the host that name is only
// a stand-in for the device symbol.  Looked up once per device, on the first
// call made with that device current.
dgmr_status static_scratch(void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return DGMR_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p)
            return DGMR_ERR_CUDA;
        g_static_ptr[dev] = p;
    }
    *out = g_static_ptr[dev];
    return DGMR_OK;
}

} // namespace

extern "C" dgmr_status dgmr_splat_forward_noalloc(const dgmr_scene* scene, const dgmr_camera* camera, float* framebuffer, int64_t pair_capacity,
    dgmr_frame_stats* stats, dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, DGMR_F32);
    if (st != DGMR_OK)
        return st;
    if (!framebuffer || pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff))
        return DGMR_ERR_BAD_ARG;
    const uint32_t N = uint32_t(scene->n_gaussians), W = uint32_t(camera->width), H = uint32_t(camera->height), cap = uint32_t(pair_capacity);
    const SplatLayout sizes = splat_layout(N, W, H, cap, nullptr, nullptr);
    const size_t frame_bytes = align_up(sizes.bytes);
    if (frame_bytes + sizes.pair_bytes > kStaticScratchBytes)
        return DGMR_ERR_STATIC_SCRATCH;
    void* base = nullptr;
    st = static_scratch(&base);
    if (st != DGMR_OK)
        return st;
    char* frame_ws = static_cast<char*>(base);
    char* pair_ws = frame_ws + frame_bytes;
    SplatLayout L = splat_layout(N, W, H, cap, frame_ws, pair_ws);
    const CameraT<float> cam = make_camera<float>(*camera);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    launch_preprocess(scene, cam, L, st_dev, s);
    launch_render(scene, cam, framebuffer, L, cap, st_dev, s);
    st = launch_status();
    if (st != DGMR_OK || stats)
        return st;
    // No caller-visible statistics: the overflow flag sits in the static
    // array, so wait for the frame and report it as the call's status.
    uint32_t flags = 0;
    if (cudaMemcpyAsync(&flags, L.stats + 1, sizeof(flags), cudaMemcpyDeviceToHost, s) != cudaSuccess
        || cudaStreamSynchronize(s) != cudaSuccess)
        return DGMR_ERR_CUDA;
    return (flags & DGMR_FLAG_PAIR_OVERFLOW) ? DGMR_ERR_PAIR_OVERFLOW : DGMR_OK;
}
