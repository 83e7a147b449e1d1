// Continuous-batching request server, host C++ over the library's C ABI.
//
// No reference counterpart: the reference renders one view per call from a
// training loop or its viewer.  A server holds resident scenes (caller-owned
// device tensors) and a queue of requests -- a splat render (optionally with
// the gradient against a caller image gradient) or a vol_marcher render
// (optionally with its backward).  Each of n_slots slots owns a CUDA stream,
// grow-only workspaces and an event; whenever a slot is free the queue head
// is cut into one batch:
//   * requests of one kind (splat or marcher) in arrival order, as many as
//     fit the view / scene-entry limits of one batched launch sequence
//     (dgmr_splat_batch_* or dgmr_vm_batch_*), the batch's pixel cap and the
//     HBM budget (a gradient request gets its own scene entry, so its
//     gradients never mix with another request's); small marcher frames gain
//     most from sharing a launch (a few rays with long tile lists each do not
//     fill the GPU);
//   * a batch of one request goes through the single-frame entry points
//     (dgmr_splat_forward / _backward; dgmr_vm_forward_preprocess /
//     _render_options / dgmr_vm_backward): the same bits, a shorter sequence.
// Pair capacities are learnt per (scene, resolution, renderer): the first
// request of a key sizes itself with one synchronous read of its pair count,
// later ones launch with the learnt capacity and no host synchronisation; a
// batch whose pairs overflowed is rendered again, exactly sized, before it
// completes, so every result equals the plain call.  Completions are
// reported by dgmr_server_poll / _wait; the caller's buffers are written when
// a request completes (device framebuffer, optional pinned host copy,
// gradients).  One thread drives a server; servers are independent.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <tuple>
#include <vector>

#include "../../include/dgmr_b200.h"

namespace {

constexpr double kHeadroom = 1.25; // workspace growth factor

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// grow-only device buffer (freed only when it must grow or the server goes)
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool ensure(size_t need, int* reallocs)
    {
        if (need <= bytes && p)
            return true;
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
        const size_t n = std::max<size_t>(256, size_t(double(need) * kHeadroom) + 256);
        if (cudaMalloc(&p, n) != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return false;
        }
        bytes = n;
        ++*reallocs;
        return true;
    }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

struct Request {
    dgmr_server_request r;
    double t_submit = 0, t_launch = 0;
    int rerendered = 0;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    DevBuf frame_ws, pair_ws, cache; // cache: the marcher's per-Gaussian / per-tile / per-pixel arrays
    dgmr_frame_stats* stats_dev = nullptr;
    dgmr_frame_stats* stats_host = nullptr; // pinned
    std::vector<Request> batch;
    int64_t capacity = 0;
    size_t reserved = 0;
    bool busy = false;
    // tables of the batch in flight (kept for a re-render)
    std::vector<dgmr_scene> scenes;
    std::vector<dgmr_batch_view> views;
    std::vector<dgmr_scene_grads> grads;
    dgmr_vm_cache vm {};
};

using Key = std::tuple<int32_t, int32_t, int32_t, int32_t>; // scene, width, height, kind

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// the marcher cache arrays of one frame, carved from one buffer
size_t vm_cache_bytes(int64_t n, int64_t w, int64_t h, int64_t cap, size_t* off /* [12] or null */)
{
    const int64_t tiles = ((w + 15) / 16) * ((h + 15) / 16);
    const size_t sizes[12] = { size_t(n) * 8, size_t(n) * 12, size_t(n) * 3, size_t(n) * 4, size_t(n) * 8, size_t(n) * 24, size_t(n) * 4,
        size_t(n) * 4, size_t(n) * 4, size_t(tiles) * 8, size_t(cap) * 4 + 4, size_t(w * h) * 4 };
    size_t total = 0;
    for (int i = 0; i < 12; ++i) {
        if (off)
            off[i] = total;
        total += align256(sizes[i]);
    }
    return total;
}

} // namespace

struct dgmr_server {
    dgmr_server_config cfg {};
    int device = 0;
    std::vector<dgmr_scene> scenes;
    std::vector<size_t> scene_bytes;
    std::deque<Request> queue;
    std::vector<Slot> slots;
    std::vector<dgmr_server_completion> done;
    std::map<Key, int64_t> capacity; // pairs per frame of a key (with the margin)
    std::map<std::tuple<int32_t, int32_t, int32_t, int32_t, int32_t>, size_t> unit_cost;
    size_t budget = 0, in_use = 0, peak = 0;
    dgmr_server_stats st {};
    double t0 = 0;
    cudaStream_t probe = nullptr; // first-sight pair counts
    DevBuf probe_ws, probe_cache;
    dgmr_frame_stats* probe_stats_dev = nullptr;
    dgmr_frame_stats* probe_stats_host = nullptr;
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess)
            prev = -1;
        cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0)
            cudaSetDevice(prev);
    }
};

bool is_march(const dgmr_server_request& r) { return r.kind == DGMR_SERVE_MARCH; }
bool wants_grad(const dgmr_server_request& r) { return r.grad_image != nullptr; }
Key key_of(const dgmr_server_request& r) { return Key { r.scene, r.camera.width, r.camera.height, r.kind }; }

void set_vm_cache(dgmr_vm_cache& c, char* base, int64_t n, int64_t w, int64_t h, int64_t cap, void* fb)
{
    size_t off[12];
    vm_cache_bytes(n, w, h, cap, off);
    c.framebuffer = fb;
    c.rects = reinterpret_cast<int32_t*>(base + off[0]);
    c.rgb = base + off[1];
    c.rgb_sh_clamped = reinterpret_cast<uint8_t*>(base + off[2]);
    c.depths = base + off[3];
    c.points_xy_image = base + off[4];
    c.inverse_filtered_cov3d = base + off[5];
    c.filtered_masses = base + off[6];
    c.tiles_touched = reinterpret_cast<int32_t*>(base + off[7]);
    c.point_offsets = reinterpret_cast<int32_t*>(base + off[8]);
    c.i_ranges = reinterpret_cast<int32_t*>(base + off[9]);
    c.b_point_list = reinterpret_cast<int32_t*>(base + off[10]);
    c.remaining_transparency = base + off[11];
}

// Pair count of a key's frame, read once (synchronously) on the probe stream.
dgmr_status learn_capacity(dgmr_server* s, const dgmr_server_request& r, int64_t* out)
{
    const Key k = key_of(r);
    auto it = s->capacity.find(k);
    if (it != s->capacity.end()) {
        *out = it->second;
        return DGMR_OK;
    }
    const dgmr_scene& sc = s->scenes[size_t(r.scene)];
    const int n = sc.n_gaussians, w = r.camera.width, h = r.camera.height;
    dgmr_status st;
    if (is_march(r)) {
        const size_t ws = dgmr_vm_workspace_size(n, w, h, 0, DGMR_F32);
        if (!ws)
            return DGMR_ERR_BAD_ARG;
        if (!s->probe_ws.ensure(ws, &s->st.reallocs) || !s->probe_cache.ensure(vm_cache_bytes(n, w, h, 0, nullptr), &s->st.reallocs))
            return DGMR_ERR_CUDA;
        dgmr_vm_cache c {};
        // the framebuffer is not written by the preprocess; any valid device address will do
        set_vm_cache(c, static_cast<char*>(s->probe_cache.p), n, w, h, 0, s->probe_cache.p);
        st = dgmr_vm_forward_preprocess(&sc, &r.camera, &c, s->probe_ws.p, s->probe_ws.bytes, s->probe_stats_dev, reinterpret_cast<dgmr_stream>(s->probe));
    } else {
        const size_t ws = dgmr_splat_frame_workspace_size(n, w, h);
        if (!ws)
            return DGMR_ERR_BAD_ARG;
        if (!s->probe_ws.ensure(ws, &s->st.reallocs))
            return DGMR_ERR_CUDA;
        st = dgmr_splat_preprocess(&sc, &r.camera, s->probe_ws.p, s->probe_ws.bytes, s->probe_stats_dev, reinterpret_cast<dgmr_stream>(s->probe));
    }
    if (st != DGMR_OK)
        return st;
    if (cudaMemcpyAsync(s->probe_stats_host, s->probe_stats_dev, sizeof(dgmr_frame_stats), cudaMemcpyDeviceToHost, s->probe) != cudaSuccess
        || cudaStreamSynchronize(s->probe) != cudaSuccess)
        return DGMR_ERR_CUDA;
    const int64_t cap = int64_t(std::ceil(double(s->probe_stats_host->n_pairs) * s->cfg.capacity_margin)) + 1024;
    s->capacity[k] = cap;
    *out = cap;
    return DGMR_OK;
}

// Tables of a batch: a scene entry per scene of render-only requests, one of
// its own per gradient request.
void batch_tables(dgmr_server* s, Slot& sl)
{
    sl.scenes.clear();
    sl.views.clear();
    sl.grads.clear();
    std::map<int32_t, int32_t> entry_of; // render-only entries by scene
    for (const Request& q : sl.batch) {
        const dgmr_server_request& r = q.r;
        int32_t e;
        if (!wants_grad(r) && entry_of.count(r.scene)) {
            e = entry_of[r.scene];
        } else {
            e = int32_t(sl.scenes.size());
            sl.scenes.push_back(s->scenes[size_t(r.scene)]);
            dgmr_scene_grads g {};
            if (wants_grad(r))
                g = r.grads;
            sl.grads.push_back(g);
            if (!wants_grad(r))
                entry_of[r.scene] = e;
        }
        dgmr_batch_view v {};
        v.scene = e;
        v.camera = r.camera;
        v.framebuffer = r.framebuffer;
        v.grad_framebuffer = r.grad_image;
        sl.views.push_back(v);
    }
}

// Bytes a one-request batch holds (workspaces, outputs, gradients): the
// admission cost of each request, summed over a batch.
dgmr_status unit_cost(dgmr_server* s, const dgmr_server_request& r, size_t* out)
{
    const auto k = std::make_tuple(r.scene, r.camera.width, r.camera.height, r.kind, int32_t(wants_grad(r)));
    auto it = s->unit_cost.find(k);
    if (it != s->unit_cost.end()) {
        *out = it->second;
        return DGMR_OK;
    }
    int64_t cap = 0;
    dgmr_status st = learn_capacity(s, r, &cap);
    if (st != DGMR_OK)
        return st;
    const dgmr_scene& sc = s->scenes[size_t(r.scene)];
    const size_t px = size_t(r.camera.width) * size_t(r.camera.height);
    size_t bytes = 12 * px + (wants_grad(r) ? s->scene_bytes[size_t(r.scene)] : 0);
    if (is_march(r)) {
        bytes += dgmr_vm_workspace_size(sc.n_gaussians, r.camera.width, r.camera.height, cap, DGMR_F32)
            + vm_cache_bytes(sc.n_gaussians, r.camera.width, r.camera.height, cap, nullptr);
    } else {
        dgmr_batch_view v {};
        v.camera = r.camera;
        size_t fb = 0, pb = 0;
        st = dgmr_splat_batch_workspace_size(&sc, 1, &v, 1, cap, &fb, &pb);
        if (st != DGMR_OK)
            return st;
        bytes += fb + pb;
    }
    s->unit_cost[k] = bytes;
    *out = bytes;
    return DGMR_OK;
}

dgmr_status launch(dgmr_server* s, Slot& sl)
{
    const cudaStream_t cs = sl.stream;
    const dgmr_stream ds = reinterpret_cast<dgmr_stream>(cs);
    dgmr_status st = DGMR_OK;
    const dgmr_server_request& head = sl.batch.front().r;
    if (is_march(head) && sl.batch.size() == 1) {
        const dgmr_scene& sc = s->scenes[size_t(head.scene)];
        const int n = sc.n_gaussians, w = head.camera.width, h = head.camera.height;
        const size_t ws = dgmr_vm_workspace_size(n, w, h, sl.capacity, DGMR_F32);
        if (!sl.frame_ws.ensure(ws, &s->st.reallocs) || !sl.cache.ensure(vm_cache_bytes(n, w, h, sl.capacity, nullptr), &s->st.reallocs))
            return DGMR_ERR_CUDA;
        set_vm_cache(sl.vm, static_cast<char*>(sl.cache.p), n, w, h, sl.capacity, head.framebuffer);
        st = dgmr_vm_forward_preprocess(&sc, &head.camera, &sl.vm, sl.frame_ws.p, sl.frame_ws.bytes, sl.stats_dev, ds);
        if (st == DGMR_OK)
            st = dgmr_vm_forward_render_options(&sc, &head.camera, nullptr, &sl.vm, sl.capacity, sl.frame_ws.p, sl.frame_ws.bytes, sl.stats_dev, ds);
        if (st == DGMR_OK)
            cudaMemcpyAsync(sl.stats_host, sl.stats_dev, sizeof(dgmr_frame_stats), cudaMemcpyDeviceToHost, cs);
        if (st == DGMR_OK && wants_grad(head))
            st = dgmr_vm_backward(&sc, &head.camera, &sl.vm, head.grad_image, head.grads.sh, head.grads.weights, head.grads.centroids,
                head.grads.scales, head.grads.rotations, sl.frame_ws.p, sl.frame_ws.bytes, nullptr, ds);
    } else if (sl.batch.size() == 1) {
        // one view: the single-frame entry points (the same bits as the batched ones, a
        // shorter launch sequence)
        const dgmr_scene& sc = s->scenes[size_t(head.scene)];
        const int n = sc.n_gaussians;
        const size_t fb = dgmr_splat_frame_workspace_size(n, head.camera.width, head.camera.height);
        const size_t pb = std::max<size_t>(1, dgmr_splat_pair_workspace_size(n, sl.capacity));
        if (!fb)
            return DGMR_ERR_BAD_ARG;
        if (!sl.frame_ws.ensure(fb, &s->st.reallocs) || !sl.pair_ws.ensure(pb, &s->st.reallocs))
            return DGMR_ERR_CUDA;
        st = dgmr_splat_forward(&sc, &head.camera, head.framebuffer, sl.frame_ws.p, sl.frame_ws.bytes, sl.pair_ws.p, sl.pair_ws.bytes, sl.capacity,
            sl.stats_dev, ds);
        if (st == DGMR_OK)
            cudaMemcpyAsync(sl.stats_host, sl.stats_dev, sizeof(dgmr_frame_stats), cudaMemcpyDeviceToHost, cs);
        if (st == DGMR_OK && wants_grad(head))
            st = dgmr_splat_backward(&sc, &head.camera, head.grad_image, head.grads.sh, head.grads.weights, head.grads.centroids, head.grads.scales,
                head.grads.rotations, sl.frame_ws.p, sl.frame_ws.bytes, sl.pair_ws.p, sl.pair_ws.bytes, sl.capacity, ds);
    } else if (is_march(head)) {
        batch_tables(s, sl);
        const int32_t nv = int32_t(sl.views.size()), ns = int32_t(sl.scenes.size());
        size_t fb = 0, pb = 0;
        st = dgmr_vm_batch_workspace_size(sl.scenes.data(), ns, sl.views.data(), nv, sl.capacity, &fb, &pb);
        if (st != DGMR_OK)
            return st;
        if (!sl.frame_ws.ensure(fb, &s->st.reallocs) || !sl.pair_ws.ensure(std::max<size_t>(pb, 1), &s->st.reallocs))
            return DGMR_ERR_CUDA;
        st = dgmr_vm_batch_forward(sl.scenes.data(), ns, sl.views.data(), nv, sl.frame_ws.p, sl.frame_ws.bytes, sl.pair_ws.p, sl.pair_ws.bytes,
            sl.capacity, sl.stats_dev, ds);
        if (st == DGMR_OK)
            cudaMemcpyAsync(sl.stats_host, sl.stats_dev, sizeof(dgmr_frame_stats), cudaMemcpyDeviceToHost, cs);
        bool any_grad = false;
        for (const Request& q : sl.batch)
            any_grad = any_grad || wants_grad(q.r);
        if (st == DGMR_OK && any_grad)
            st = dgmr_vm_batch_backward(sl.scenes.data(), ns, sl.views.data(), nv, sl.grads.data(), sl.frame_ws.p, sl.frame_ws.bytes, sl.pair_ws.p,
                sl.pair_ws.bytes, sl.capacity, nullptr, ds);
    } else {
        batch_tables(s, sl);
        const int32_t nv = int32_t(sl.views.size()), ns = int32_t(sl.scenes.size());
        size_t fb = 0, pb = 0;
        st = dgmr_splat_batch_workspace_size(sl.scenes.data(), ns, sl.views.data(), nv, sl.capacity, &fb, &pb);
        if (st != DGMR_OK)
            return st;
        if (!sl.frame_ws.ensure(fb, &s->st.reallocs) || !sl.pair_ws.ensure(pb, &s->st.reallocs))
            return DGMR_ERR_CUDA;
        st = dgmr_splat_batch_forward(sl.scenes.data(), ns, sl.views.data(), nv, sl.frame_ws.p, sl.frame_ws.bytes, sl.pair_ws.p, sl.pair_ws.bytes,
            sl.capacity, sl.stats_dev, ds);
        if (st == DGMR_OK)
            cudaMemcpyAsync(sl.stats_host, sl.stats_dev, sizeof(dgmr_frame_stats), cudaMemcpyDeviceToHost, cs);
        bool any_grad = false;
        for (const Request& q : sl.batch)
            any_grad = any_grad || wants_grad(q.r);
        if (st == DGMR_OK && any_grad)
            st = dgmr_splat_batch_backward(sl.scenes.data(), ns, sl.views.data(), nv, sl.grads.data(), sl.frame_ws.p, sl.frame_ws.bytes, sl.pair_ws.p,
                sl.pair_ws.bytes, sl.capacity, ds);
    }
    if (st != DGMR_OK)
        return st;
    for (const Request& q : sl.batch)
        if (q.r.host_image
            && cudaMemcpyAsync(q.r.host_image, q.r.framebuffer, size_t(12) * size_t(q.r.camera.width) * size_t(q.r.camera.height), cudaMemcpyDeviceToHost, cs)
                != cudaSuccess)
            return DGMR_ERR_CUDA;
    if (cudaEventRecord(sl.done, cs) != cudaSuccess)
        return DGMR_ERR_CUDA;
    sl.busy = true;
    return DGMR_OK;
}

void complete(dgmr_server* s, Slot& sl, dgmr_status status)
{
    const double t = now_s() - s->t0;
    for (const Request& q : sl.batch) {
        dgmr_server_completion c {};
        c.tag = q.r.tag;
        c.status = status;
        c.n_pairs = sl.stats_host->n_pairs;
        c.batch_size = int32_t(sl.batch.size());
        c.rerendered = q.rerendered;
        c.submit_s = q.t_submit;
        c.launch_s = q.t_launch;
        c.done_s = t;
        s->done.push_back(c);
    }
    s->in_use -= std::min(s->in_use, sl.reserved);
    sl.reserved = 0;
    sl.batch.clear();
    sl.busy = false;
}

// Finished batches complete (or render again, exactly sized, after an overflow).
void reap(dgmr_server* s)
{
    for (Slot& sl : s->slots) {
        if (!sl.busy)
            continue;
        const cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaErrorNotReady)
            continue;
        if (q != cudaSuccess) {
            cudaGetLastError();
            complete(s, sl, DGMR_ERR_CUDA);
            continue;
        }
        const uint32_t pairs = sl.stats_host->n_pairs, flags = sl.stats_host->flags;
        if (flags & DGMR_FLAG_PAIR_OVERFLOW) {
            // more pairs than the learnt capacities: grow them, render the batch again
            ++s->st.rerenders;
            const double grow = double(pairs) / double(std::max<int64_t>(sl.capacity, 1));
            std::vector<Key> grown; // each key of the batch grows once, however many of its requests the batch holds
            for (Request& q2 : sl.batch) {
                const Key k = key_of(q2.r);
                q2.rerendered = 1;
                if (std::find(grown.begin(), grown.end(), k) != grown.end())
                    continue;
                grown.push_back(k);
                s->capacity[k] = std::min<int64_t>(int64_t(std::ceil(double(s->capacity[k]) * std::max(s->cfg.capacity_margin, grow))), 0x7fffffff);
                for (int g = 0; g < 2; ++g)
                    s->unit_cost.erase(std::make_tuple(q2.r.scene, q2.r.camera.width, q2.r.camera.height, q2.r.kind, int32_t(g)));
            }
            sl.capacity = int64_t(pairs) + 1024;
            const dgmr_status st = launch(s, sl);
            if (st != DGMR_OK)
                complete(s, sl, st);
            continue;
        }
        ++s->st.batches;
        complete(s, sl, DGMR_OK);
    }
}

// Batches cut from the queue head onto free slots.
void dispatch(dgmr_server* s)
{
    for (Slot& sl : s->slots) {
        if (sl.busy || s->queue.empty())
            continue;
        std::vector<Request> batch;
        size_t bytes = 0;
        int64_t cap = 0, pixels = 0;
        int entries = 0;
        std::vector<int32_t> render_scenes;
        dgmr_status err = DGMR_OK;
        while (!s->queue.empty()) {
            const Request& q = s->queue.front();
            const bool march = is_march(q.r);
            const int64_t px = int64_t(q.r.camera.width) * int64_t(q.r.camera.height);
            if (!batch.empty()
                && (march != is_march(batch.front().r) || int32_t(batch.size()) >= s->cfg.max_views
                    || (s->cfg.max_batch_pixels > 0 && pixels + px > s->cfg.max_batch_pixels)))
                break;
            const bool new_entry = wants_grad(q.r) || std::find(render_scenes.begin(), render_scenes.end(), q.r.scene) == render_scenes.end();
            if (new_entry && entries + 1 > DGMR_BATCH_MAX_SCENES)
                break;
            size_t c = 0;
            int64_t kc = 0;
            err = unit_cost(s, q.r, &c);
            if (err == DGMR_OK)
                err = learn_capacity(s, q.r, &kc);
            if (err != DGMR_OK)
                break;
            if (s->in_use + bytes + c > s->budget || cap + kc > int64_t(0x7fffffff))
                break;
            bytes += c;
            cap += kc;
            pixels += px;
            if (new_entry)
                ++entries;
            if (!wants_grad(q.r))
                render_scenes.push_back(q.r.scene);
            batch.push_back(q);
            batch.back().t_launch = now_s() - s->t0;
            s->queue.pop_front();
        }
        if (err != DGMR_OK && batch.empty()) {
            // the head cannot run at all: complete it with the error
            sl.batch.assign(1, s->queue.front());
            s->queue.pop_front();
            sl.stats_host->n_pairs = 0;
            complete(s, sl, err);
            continue;
        }
        if (batch.empty()) {
            bool any_busy = false;
            for (const Slot& o : s->slots)
                any_busy = any_busy || o.busy;
            if (!any_busy) { // nothing in flight and the head alone exceeds the budget
                sl.batch.assign(1, s->queue.front());
                s->queue.pop_front();
                sl.stats_host->n_pairs = 0;
                complete(s, sl, DGMR_ERR_WORKSPACE);
                continue;
            }
            ++s->st.deferred;
            break;
        }
        s->in_use += bytes;
        s->peak = std::max(s->peak, s->in_use);
        sl.reserved = bytes;
        sl.batch = std::move(batch);
        sl.capacity = cap;
        const dgmr_status st = launch(s, sl);
        if (st != DGMR_OK)
            complete(s, sl, st);
    }
}

int32_t take_completions(dgmr_server* s, dgmr_server_completion* out, int32_t max_out)
{
    const int32_t n = int32_t(std::min<size_t>(s->done.size(), size_t(std::max(max_out, 0))));
    if (out && n > 0)
        std::memcpy(out, s->done.data(), size_t(n) * sizeof(dgmr_server_completion));
    s->done.erase(s->done.begin(), s->done.begin() + n);
    return n;
}

} // namespace

extern "C" {

dgmr_status dgmr_server_create(const dgmr_server_config* config, dgmr_server** out)
{
    if (!out)
        return DGMR_ERR_BAD_ARG;
    *out = nullptr;
    dgmr_server_config cfg {};
    if (config)
        cfg = *config;
    if (cfg.n_slots <= 0)
        cfg.n_slots = 4;
    if (cfg.max_views <= 0 || cfg.max_views > DGMR_BATCH_MAX_VIEWS)
        cfg.max_views = cfg.max_views <= 0 ? 8 : DGMR_BATCH_MAX_VIEWS;
    // 2.0: a pair count grows with 1 / distance^2, 2.5x across the camera radii
    // a request mix may hold, so a key's first frames rarely bound its later ones
    // (c4 serving: 13 -> 1 re-renders per 200 requests against 1.3, HBM peak
    // 17.7 -> 22.0 GB); the pair workspaces cost memory only
    if (!(cfg.capacity_margin > 0.0))
        cfg.capacity_margin = 2.0;
    if (cfg.n_slots > 64)
        return DGMR_ERR_BAD_ARG;
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || cfg.device < 0 || cfg.device >= n_dev) {
        cudaGetLastError();
        return DGMR_ERR_CUDA;
    }
    DeviceGuard g(cfg.device);
    dgmr_server* s = new (std::nothrow) dgmr_server();
    if (!s)
        return DGMR_ERR_BAD_ARG;
    s->cfg = cfg;
    s->device = cfg.device;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        delete s;
        return DGMR_ERR_CUDA;
    }
    s->budget = cfg.hbm_budget_bytes ? cfg.hbm_budget_bytes : size_t(double(free_b) * 0.8);
    bool ok = cudaStreamCreateWithFlags(&s->probe, cudaStreamNonBlocking) == cudaSuccess
        && cudaMalloc(&s->probe_stats_dev, sizeof(dgmr_frame_stats)) == cudaSuccess
        && cudaMallocHost(&s->probe_stats_host, sizeof(dgmr_frame_stats)) == cudaSuccess;
    s->slots.resize(size_t(cfg.n_slots));
    for (Slot& sl : s->slots) {
        ok = ok && cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) == cudaSuccess
            && cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) == cudaSuccess
            && cudaMalloc(&sl.stats_dev, sizeof(dgmr_frame_stats)) == cudaSuccess
            && cudaMallocHost(&sl.stats_host, sizeof(dgmr_frame_stats)) == cudaSuccess;
        if (ok)
            std::memset(sl.stats_host, 0, sizeof(dgmr_frame_stats));
    }
    if (!ok) {
        cudaGetLastError();
        dgmr_server_destroy(s);
        return DGMR_ERR_CUDA;
    }
    s->t0 = now_s(); // the completions' clock starts once the server exists
    *out = s;
    return DGMR_OK;
}

double dgmr_server_now(const dgmr_server* s) { return s ? now_s() - s->t0 : -1.0; }

dgmr_status dgmr_server_add_scene(dgmr_server* s, const dgmr_scene* scene, int32_t* index)
{
    if (!s || !scene || !index || scene->dtype != DGMR_F32 || scene->n_gaussians < 0 || scene->sh_stride < 1 || scene->sh_stride > 16
        || (scene->n_gaussians > 0 && (!scene->centroids || !scene->sh || !scene->weights || !scene->scales || !scene->rotations)))
        return DGMR_ERR_BAD_ARG;
    s->scenes.push_back(*scene);
    s->scene_bytes.push_back(size_t(scene->n_gaussians) * (size_t(scene->sh_stride) * 12 + 4 + 12 + 12 + 16));
    *index = int32_t(s->scenes.size()) - 1;
    return DGMR_OK;
}

dgmr_status dgmr_server_submit(dgmr_server* s, const dgmr_server_request* request)
{
    if (!s || !request)
        return DGMR_ERR_BAD_ARG;
    const dgmr_server_request& r = *request;
    if (r.scene < 0 || size_t(r.scene) >= s->scenes.size() || !r.framebuffer || r.camera.width <= 0 || r.camera.height <= 0
        || (r.kind != DGMR_SERVE_SPLAT && r.kind != DGMR_SERVE_MARCH))
        return DGMR_ERR_BAD_ARG;
    // gradient outputs of a scene without Gaussians may have no address
    if (wants_grad(r) && s->scenes[size_t(r.scene)].n_gaussians > 0
        && (!r.grads.sh || !r.grads.weights || !r.grads.centroids || !r.grads.scales || !r.grads.rotations))
        return DGMR_ERR_BAD_ARG;
    Request q;
    q.r = r;
    q.t_submit = now_s() - s->t0;
    s->queue.push_back(q);
    ++s->st.submitted;
    return DGMR_OK;
}

int32_t dgmr_server_poll(dgmr_server* s, dgmr_server_completion* out, int32_t max_out)
{
    if (!s)
        return -1;
    DeviceGuard g(s->device);
    reap(s);
    dispatch(s);
    return take_completions(s, out, max_out);
}

int32_t dgmr_server_wait(dgmr_server* s, dgmr_server_completion* out, int32_t max_out)
{
    if (!s)
        return -1;
    DeviceGuard g(s->device);
    for (;;) {
        reap(s);
        dispatch(s);
        if (!s->done.empty())
            return take_completions(s, out, max_out);
        bool any_busy = false;
        for (Slot& sl : s->slots)
            if (sl.busy) {
                any_busy = true;
                cudaEventSynchronize(sl.done); // the oldest batch in flight
                break;
            }
        if (!any_busy && s->queue.empty())
            return 0;
    }
}

int64_t dgmr_server_pending(const dgmr_server* s)
{
    if (!s)
        return -1;
    int64_t n = int64_t(s->queue.size()) + int64_t(s->done.size());
    for (const Slot& sl : s->slots)
        n += int64_t(sl.batch.size());
    return n;
}

dgmr_status dgmr_server_get_stats(const dgmr_server* s, dgmr_server_stats* out)
{
    if (!s || !out)
        return DGMR_ERR_BAD_ARG;
    *out = s->st;
    out->hbm_budget_bytes = s->budget;
    out->hbm_in_use_bytes = s->in_use;
    out->hbm_peak_bytes = s->peak;
    return DGMR_OK;
}

dgmr_status dgmr_server_destroy(dgmr_server* s)
{
    if (!s)
        return DGMR_ERR_BAD_ARG;
    DeviceGuard g(s->device);
    for (Slot& sl : s->slots) {
        if (sl.stream)
            cudaStreamSynchronize(sl.stream);
        sl.frame_ws.release();
        sl.pair_ws.release();
        sl.cache.release();
        if (sl.stats_dev)
            cudaFree(sl.stats_dev);
        if (sl.stats_host)
            cudaFreeHost(sl.stats_host);
        if (sl.done)
            cudaEventDestroy(sl.done);
        if (sl.stream)
            cudaStreamDestroy(sl.stream);
    }
    if (s->probe)
        cudaStreamSynchronize(s->probe);
    s->probe_ws.release();
    s->probe_cache.release();
    if (s->probe_stats_dev)
        cudaFree(s->probe_stats_dev);
    if (s->probe_stats_host)
        cudaFreeHost(s->probe_stats_host);
    if (s->probe)
        cudaStreamDestroy(s->probe);
    delete s;
    return DGMR_OK;
}

} // extern "C"
