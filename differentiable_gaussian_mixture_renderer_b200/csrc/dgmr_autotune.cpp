// Batch autotuner, host C++ over the library's C ABI (no reference
// counterpart: the reference renders one view per call).
//
// A view set can be launched as one batch or cut into several, and the splat
// blend can run on 8x8 or 16x16 pixel blocks; every choice gives the same
// images and gradients, only the time differs.  dgmr_batch_autotune times
// each (batch depth, blend block) candidate on the caller's stream with CUDA
// events -- the whole set, cut into consecutive batches of at most `depth`
// views, forward and (with gradient outputs) backward, once untimed and
// `reps` times timed -- and reports the best time of each and the fastest.
// Each batch carries only the scenes its views use (scene indices remapped),
// as a caller batching the set that way would pass them.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <vector>

#include "../../include/dgmr_b200.h"

namespace {

struct Batch {
    std::vector<dgmr_scene> scenes;
    std::vector<dgmr_scene_grads> grads;
    std::vector<dgmr_batch_view> views;
};

// Consecutive batches of at most `depth` views with blend block `block`.
std::vector<Batch> cut(const dgmr_scene* scenes, const dgmr_batch_view* views, int32_t n_views, const dgmr_scene_grads* grads, int32_t depth,
    int32_t block)
{
    std::vector<Batch> out;
    std::vector<int32_t> local; // scene index -> index in the current batch, -1 if absent
    for (int32_t v = 0; v < n_views; ++v) {
        if (out.empty() || int32_t(out.back().views.size()) >= depth) {
            out.emplace_back();
            local.assign(DGMR_BATCH_MAX_SCENES, -1);
        }
        Batch& b = out.back();
        const int32_t s = views[v].scene;
        if (local[size_t(s)] < 0) {
            local[size_t(s)] = int32_t(b.scenes.size());
            b.scenes.push_back(scenes[s]);
            if (grads)
                b.grads.push_back(grads[s]);
        }
        dgmr_batch_view w = views[v];
        w.scene = local[size_t(s)];
        w.blend_block = block;
        b.views.push_back(w);
    }
    return out;
}

dgmr_status run(int32_t kind, std::vector<Batch>& batches, bool backward, void* fws, size_t fbytes, void* pws, size_t pbytes, int64_t cap,
    dgmr_stream stream)
{
    for (Batch& b : batches) {
        const int32_t ns = int32_t(b.scenes.size()), nv = int32_t(b.views.size());
        dgmr_status st = kind == DGMR_SERVE_SPLAT
            ? dgmr_splat_batch_forward(b.scenes.data(), ns, b.views.data(), nv, fws, fbytes, pws, pbytes, cap, nullptr, stream)
            : dgmr_vm_batch_forward(b.scenes.data(), ns, b.views.data(), nv, fws, fbytes, pws, pbytes, cap, nullptr, stream);
        if (st == DGMR_OK && backward)
            st = kind == DGMR_SERVE_SPLAT
                ? dgmr_splat_batch_backward(b.scenes.data(), ns, b.views.data(), nv, b.grads.data(), fws, fbytes, pws, pbytes, cap, stream)
                : dgmr_vm_batch_backward(b.scenes.data(), ns, b.views.data(), nv, b.grads.data(), fws, fbytes, pws, pbytes, cap, nullptr, stream);
        if (st != DGMR_OK)
            return st;
    }
    return DGMR_OK;
}

} // namespace

extern "C" dgmr_status dgmr_batch_autotune(int32_t kind, const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views,
    const dgmr_scene_grads* grads, const int32_t* depths, int32_t n_depths, const int32_t* blend_blocks, int32_t n_blocks, int32_t reps,
    void* frame_workspace, size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, float* ms,
    int32_t* best_depth, int32_t* best_block, dgmr_stream stream)
{
    if ((kind != DGMR_SERVE_SPLAT && kind != DGMR_SERVE_MARCH) || !scenes || !views || n_scenes < 1 || n_scenes > DGMR_BATCH_MAX_SCENES || n_views < 1
        || n_views > DGMR_BATCH_MAX_VIEWS || !depths || n_depths < 1 || !blend_blocks || n_blocks < 1 || reps < 1 || !ms || !best_depth || !best_block)
        return DGMR_ERR_BAD_ARG;
    for (int32_t v = 0; v < n_views; ++v)
        if (views[v].scene < 0 || views[v].scene >= n_scenes)
            return DGMR_ERR_BAD_ARG;
    for (int32_t d = 0; d < n_depths; ++d)
        if (depths[d] < 1)
            return DGMR_ERR_BAD_ARG;
    for (int32_t b = 0; b < n_blocks; ++b) {
        const int32_t blk = blend_blocks[b];
        if (kind == DGMR_SERVE_SPLAT ? (blk != 0 && blk != 8 && blk != 16) : blk != 0)
            return DGMR_ERR_BAD_ARG;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0)
            cudaEventDestroy(e0);
        return DGMR_ERR_CUDA;
    }
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    dgmr_status st = DGMR_OK;
    float best = FLT_MAX;
    for (int32_t d = 0; d < n_depths && st == DGMR_OK; ++d) {
        for (int32_t b = 0; b < n_blocks && st == DGMR_OK; ++b) {
            std::vector<Batch> batches = cut(scenes, views, n_views, grads, depths[d], blend_blocks[b]);
            st = run(kind, batches, grads != nullptr, frame_workspace, frame_workspace_bytes, pair_workspace, pair_workspace_bytes, pair_capacity, stream);
            float t_best = FLT_MAX;
            for (int32_t r = 0; r < reps && st == DGMR_OK; ++r) {
                if (cudaEventRecord(e0, s) != cudaSuccess) {
                    st = DGMR_ERR_CUDA;
                    break;
                }
                st = run(kind, batches, grads != nullptr, frame_workspace, frame_workspace_bytes, pair_workspace, pair_workspace_bytes, pair_capacity,
                    stream);
                float t = 0.f;
                if (st == DGMR_OK
                    && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
                    st = DGMR_ERR_CUDA;
                if (st == DGMR_OK && t < t_best)
                    t_best = t;
            }
            if (st != DGMR_OK)
                break;
            ms[size_t(d) * size_t(n_blocks) + size_t(b)] = t_best;
            if (t_best < best) {
                best = t_best;
                *best_depth = depths[d];
                *best_block = blend_blocks[b];
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}
