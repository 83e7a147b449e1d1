// The view table of a batch of frames, shared by the batched splat renderer
// and the batched volume marcher.
#pragma once
#include <cstdint>
#include <cstring>

#include "../../include/dgmr_b200.h"
#include "dgmr_abi_common.h"
#include "dgmr_binning.cuh"

// Many views -- cameras of one or several resident scenes, each at its own
// resolution -- go through ONE launch sequence: one preprocess over every
// (view, Gaussian) slot, one depth sort, one pair emission, one tile sort and
// one blend (or march) over the tiles of all views, ordered heaviest-first
// across views.
// Slots of view v are [g_off[v], g_off[v+1]); its tiles are numbered from
// tile_off[v].  The stable depth sort over all slots keeps every view's
// Gaussians in their own (depth, index) order and a global tile holds pairs
// of one view only, so each view's point list, ranges and image are the same,
// bit for bit, as when it is rendered alone.  The view table travels as a
// __grid_constant__ kernel parameter (no host copy, nothing to keep alive,
// capturable in a CUDA graph).

namespace dgmr {

// Where one tile's pixels live: the frame it belongs to and the tile's index
// inside that frame's grid.  final_T / n_contrib / grad_fb point at the
// frame's own planes.
struct FrameRef {
    unsigned W, H, gx, tile;
    float bg0, bg1, bg2;
    float* fb;
    float* final_T;
    int32_t* n_contrib;
    const float* grad_fb;
};

constexpr int kMaxBatchViews = DGMR_BATCH_MAX_VIEWS;
constexpr int kMaxBatchScenes = DGMR_BATCH_MAX_SCENES;

struct BatchScene {
    const float* centroids;
    const float* sh;
    const float* weights;
    const float* scales;
    const float* rotations;
    uint32_t n;
    int sh_stride, sh_degree;
    uint32_t view_begin, view_end; // range in BatchTable::view_by_scene
    Formulation form;
    float* g_sh;
    float* g_weights;
    float* g_centroids;
    float* g_scales;
    float* g_rotations;
};

struct BatchView {
    CameraT<float> cam;
    float* fb;
    const float* grad_fb;
    uint32_t scene, g_off, tile_off;
    size_t px_off;
};

struct BatchTable {
    uint32_t n_views, n_scenes, G, n_tiles, n_stiles;
    size_t px_total; // pixels of all views
    uint32_t g_off[kMaxBatchViews + 1];
    uint32_t tile_off[kMaxBatchViews + 1];
    uint32_t stile_off[kMaxBatchViews + 1]; // first super-tile of each view
    uint32_t scene_off[kMaxBatchScenes + 1];
    uint8_t view_by_scene[kMaxBatchViews];
    float* final_T;
    int32_t* n_contrib;
    BatchScene scenes[kMaxBatchScenes];
    BatchView views[kMaxBatchViews];

    // largest v with off[v] <= x (views that own nothing are skipped over)
    __device__ __forceinline__ static uint32_t owner(const uint32_t* off, uint32_t n, uint32_t x)
    {
        uint32_t lo = 0, hi = n;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (off[mid] <= x)
                lo = mid;
            else
                hi = mid;
        }
        return lo;
    }
    __device__ __forceinline__ TileGrid grid(uint32_t g) const
    {
        const uint32_t v = owner(g_off, n_views, g);
        return TileGrid { views[v].cam.gx, views[v].cam.gy, tile_off[v], stile_off[v] };
    }
    __device__ __forceinline__ TileGrid super_grid(uint32_t s) const
    {
        const uint32_t v = owner(stile_off, n_views, s);
        return TileGrid { views[v].cam.gx, views[v].cam.gy, tile_off[v], stile_off[v] };
    }
    __device__ __forceinline__ FrameRef frame(uint32_t t) const
    {
        const uint32_t v = owner(tile_off, n_views, t);
        const BatchView& bv = views[v];
        return FrameRef { bv.cam.W, bv.cam.H, bv.cam.gx, t - tile_off[v], bv.cam.bg[0], bv.cam.bg[1], bv.cam.bg[2], bv.fb, final_T + bv.px_off,
            n_contrib + bv.px_off, bv.grad_fb };
    }
};
static_assert(sizeof(BatchTable) < 32000, "the view table must fit in the kernel parameter space");

// Validates a batch and fills its view table: scenes (float32, with their
// gradient outputs when grads is not null), views grouped by scene, and the
// slot, tile, super-tile and pixel offsets of every view.  default_form is the
// formulation a scene with DGMR_FORMULATION_DEFAULT gets (each renderer has
// its own, as in the reference).
inline dgmr_status build_batch_table(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views,
    const dgmr_scene_grads* grads, Formulation default_form, BatchTable& t)
{
    if (!scenes || !views || n_scenes <= 0 || n_views <= 0 || n_scenes > kMaxBatchScenes || n_views > kMaxBatchViews)
        return DGMR_ERR_BAD_ARG;
    std::memset(&t, 0, sizeof(t));
    t.n_views = uint32_t(n_views);
    t.n_scenes = uint32_t(n_scenes);
    uint64_t G = 0, T = 0, ST = 0, px = 0, gs = 0;
    for (int s = 0; s < n_scenes; ++s) {
        const dgmr_scene& sc = scenes[s];
        if (sc.dtype != DGMR_F32 || sc.n_gaussians < 0 || sc.sh_stride < 1 || sc.sh_stride > 16 || sc.sh_degree < 0 || sc.sh_degree > 3
            || sc.formulation < DGMR_FORMULATION_DEFAULT || sc.formulation > DGMR_FORMULATION_OLS)
            return DGMR_ERR_BAD_ARG;
        if (sc.n_gaussians > 0 && (!sc.centroids || !sc.sh || !sc.weights || !sc.scales || !sc.rotations))
            return DGMR_ERR_BAD_ARG;
        BatchScene& b = t.scenes[s];
        b.centroids = static_cast<const float*>(sc.centroids);
        b.sh = static_cast<const float*>(sc.sh);
        b.weights = static_cast<const float*>(sc.weights);
        b.scales = static_cast<const float*>(sc.scales);
        b.rotations = static_cast<const float*>(sc.rotations);
        b.n = uint32_t(sc.n_gaussians);
        b.sh_stride = sc.sh_stride;
        b.sh_degree = sc.sh_degree;
        b.form = scene_formulation(&sc, default_form);
        if (grads && grads[s].sh) {
            const dgmr_scene_grads& g = grads[s];
            if (sc.n_gaussians > 0 && (!g.weights || !g.centroids || !g.scales || !g.rotations))
                return DGMR_ERR_BAD_ARG;
            b.g_sh = g.sh;
            b.g_weights = g.weights;
            b.g_centroids = g.centroids;
            b.g_scales = g.scales;
            b.g_rotations = g.rotations;
        }
        t.scene_off[s] = uint32_t(gs);
        gs += uint64_t(sc.n_gaussians);
    }
    t.scene_off[n_scenes] = uint32_t(gs);
    // views grouped by scene, each group in view order
    uint32_t q = 0;
    for (int s = 0; s < n_scenes; ++s) {
        t.scenes[s].view_begin = q;
        for (int v = 0; v < n_views; ++v)
            if (views[v].scene == s)
                t.view_by_scene[q++] = uint8_t(v);
        t.scenes[s].view_end = q;
    }
    for (int v = 0; v < n_views; ++v) {
        const dgmr_batch_view& bv = views[v];
        if (bv.scene < 0 || bv.scene >= n_scenes)
            return DGMR_ERR_BAD_ARG;
        const dgmr_camera& c = bv.camera;
        if (c.width <= 0 || c.height <= 0 || c.width > 65536 || c.height > 65536)
            return DGMR_ERR_BAD_ARG;
        BatchView& w = t.views[v];
        w.cam = make_camera<float>(c);
        w.fb = bv.framebuffer;
        w.grad_fb = bv.grad_framebuffer;
        w.scene = uint32_t(bv.scene);
        w.g_off = uint32_t(G);
        w.tile_off = uint32_t(T);
        w.px_off = size_t(px);
        t.g_off[v] = uint32_t(G);
        t.tile_off[v] = uint32_t(T);
        t.stile_off[v] = uint32_t(ST);
        G += uint64_t(scenes[bv.scene].n_gaussians);
        T += uint64_t(w.cam.gx) * w.cam.gy;
        ST += super_count(w.cam.gx, w.cam.gy);
        px += uint64_t(c.width) * uint64_t(c.height);
    }
    t.g_off[n_views] = uint32_t(G);
    t.tile_off[n_views] = uint32_t(T);
    t.stile_off[n_views] = uint32_t(ST);
    t.n_stiles = uint32_t(ST);
    // super-tile ids share a 32-bit sort key with a 12-bit rectangle
    if (G > 0x7fffffffull || T > (1ull << 30) || ST >= (1ull << 20) || gs > 0x7fffffffull)
        return DGMR_ERR_BAD_ARG;
    t.G = uint32_t(G);
    t.n_tiles = uint32_t(T);
    t.px_total = size_t(px);
    return DGMR_OK;
}

} // namespace dgmr
