/* C++ viewer interface over the C ABI (libdgmr_b200.so), headless.
 *
 * Mirrors the reference's C++ entry points for its viewer plugin
 * (src/dgmr/sibr_interfaces.h:24-28, src/dgmr/sibr_interfaces.cpp:26-44):
 *
 *   dgmr::sibr_interfaces::splat(SplatForwardData&)
 *   dgmr::sibr_interfaces::vol_march(framebuffer, vol_marcher::ForwardData<float>&)
 *
 * and the forward-data structs they take (splat_forward.h:37-54,
 * vol_marcher.h:29-56, vol_raster_forward.h:30-55) with the same field names
 * and defaults.  The glm / whack types become plain device pointers and glm
 * matrices become float[16] in glm memory order (element (row r, col c) at
 * c*4+r); quaternions are stored (w,x,y,z), as with GLM_FORCE_QUAT_DATA_WXYZ
 * (src/CMakeLists.txt:51).  There is no window or texture: the framebuffer is a
 * caller-owned device buffer [3,H,W] float, which a viewer uploads with
 * whatever interop it has.
 *
 * The reference allocates its temporaries per call through torch; here a
 * Context owns grow-only workspaces (one per stream), so steady-state frames
 * allocate nothing.  Like the reference, each frame reads the pair count back
 * to the host once (splat_forward.cu:141, vol_marcher_forward.cu:193), which
 * synchronises the context's stream.  Errors throw dgmr_b200::Error (the
 * reference throws from CHECK_CUDA in debug mode); no exception crosses the C
 * ABI itself.
 */
#ifndef DGMR_B200_SIBR_HPP
#define DGMR_B200_SIBR_HPP

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "dgmr_b200.h"

namespace dgmr_b200 {

class Error : public std::runtime_error {
public:
    Error(const std::string& what, dgmr_status status)
        : std::runtime_error(what + ": " + dgmr_status_string(status))
        , status(status)
    {
    }
    dgmr_status status;
};

/* splat_forward.h:26-28; n_rendered is never set by the reference (always 0).
 * n_pairs and flags are the dgmr_frame_stats of the frame. */
struct Statistics {
    unsigned n_rendered = 0;
    uint32_t n_pairs = 0;
    uint32_t flags = 0;
};

/* whack::TensorView<float, 3> framebuffer: device [3, height, width] */
struct Framebuffer {
    float* data = nullptr;
    int32_t height = 0;
    int32_t width = 0;
};

enum class RenderMode { Full, Bins, Depth }; /* vol_marcher.h:50-54 */

/* The Gaussian mixture and camera fields every forward-data struct shares. */
struct MixtureAndCamera {
    const float* gm_centroids = nullptr; /* [N,3] */
    const float* gm_sh_params = nullptr; /* [N,sh_stride,3]; SHs<3,float> is 16 coefficients */
    const float* gm_weights = nullptr; /* [N] */
    const float* gm_cov_scales = nullptr; /* [N,3] */
    const float* gm_cov_rotations = nullptr; /* [N,4] (w,x,y,z) */
    int32_t n_gaussians = 0; /* the TensorViews' size */
    int32_t sh_stride = 16;

    float view_matrix[16] = {};
    float proj_matrix[16] = {}; /* full view-projection */
    float cam_poition[3] = {}; /* (sic) the reference's field name */
    float background[3] = {};
    int sh_degree = 3;
    float cov_scale_multiplier = 1.f;
    float tan_fovy = 0.f;
    float tan_fovx = 0.f;
    bool debug = true; /* the reference's CHECK_CUDA switch; errors are always checked here */
    dgmr_formulation formulation = DGMR_FORMULATION_DEFAULT; /* the renderer's reference formulation */
};

/* splat_forward.h:37-54 */
struct SplatForwardData : MixtureAndCamera {
    Framebuffer framebuffer;
};

/* vol_marcher.h:29-56 (float instantiation) */
struct VolMarcherForwardData : MixtureAndCamera {
    float max_depth = 20.f;
    RenderMode debug_render_mode = RenderMode::Full;
    int debug_render_bin = -1;
};

/* vol_raster_forward.h:30-55 */
struct VolRasterForwardData : MixtureAndCamera {
    Framebuffer framebuffer;
    float max_depth = 20.f;
    RenderMode debug_render_mode = RenderMode::Full;
    int debug_render_bin = -1;
};

namespace detail {
    inline void check(dgmr_status st, const char* what)
    {
        if (st != DGMR_OK)
            throw Error(what, st);
    }
    inline void check_cuda(cudaError_t e, const char* what)
    {
        if (e != cudaSuccess)
            throw Error(std::string(what) + " (" + cudaGetErrorString(e) + ")", DGMR_ERR_CUDA);
    }
    inline size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

    /* Grow-only device buffer. */
    class DeviceBuffer {
    public:
        DeviceBuffer() = default;
        DeviceBuffer(const DeviceBuffer&) = delete;
        DeviceBuffer& operator=(const DeviceBuffer&) = delete;
        ~DeviceBuffer()
        {
            if (ptr_)
                cudaFree(ptr_);
        }
        void* ensure(size_t bytes, cudaStream_t stream)
        {
            if (bytes <= bytes_ && ptr_)
                return ptr_;
            if (ptr_) {
                // earlier frames on this stream may still read the old buffer
                check_cuda(cudaStreamSynchronize(stream), "workspace growth");
                check_cuda(cudaFree(ptr_), "workspace growth");
                ptr_ = nullptr;
                bytes_ = 0;
            }
            const size_t want = bytes + bytes / 4 + 256; // 25 % headroom for the next frames
            check_cuda(cudaMalloc(&ptr_, want), "workspace allocation");
            bytes_ = want;
            return ptr_;
        }
        size_t bytes() const { return bytes_; }

    private:
        void* ptr_ = nullptr;
        size_t bytes_ = 0;
    };

    inline dgmr_scene scene_of(const MixtureAndCamera& d)
    {
        dgmr_scene s {};
        s.n_gaussians = d.n_gaussians;
        s.sh_stride = d.sh_stride;
        s.sh_degree = d.sh_degree;
        s.dtype = DGMR_F32;
        s.centroids = d.gm_centroids;
        s.sh = d.gm_sh_params;
        s.weights = d.gm_weights;
        s.scales = d.gm_cov_scales;
        s.rotations = d.gm_cov_rotations;
        s.formulation = d.formulation;
        return s;
    }

    inline dgmr_camera camera_of(const MixtureAndCamera& d, int32_t width, int32_t height)
    {
        dgmr_camera c {};
        c.width = width;
        c.height = height;
        for (int i = 0; i < 16; ++i) {
            c.view[i] = d.view_matrix[i];
            c.proj[i] = d.proj_matrix[i];
        }
        for (int i = 0; i < 3; ++i) {
            c.campos[i] = d.cam_poition[i];
            c.background[i] = d.background[i];
        }
        c.tan_fovx = d.tan_fovx;
        c.tan_fovy = d.tan_fovy;
        c.cov_scale_multiplier = d.cov_scale_multiplier;
        return c;
    }

    inline dgmr_render_options options_of(RenderMode mode, int bin, float max_depth)
    {
        dgmr_render_options o {};
        o.render_mode = mode == RenderMode::Full ? DGMR_RENDER_FULL : mode == RenderMode::Bins ? DGMR_RENDER_BINS : DGMR_RENDER_DEPTH;
        o.debug_bin = bin;
        o.max_depth = max_depth;
        return o;
    }
} // namespace detail

/* One stream's workspaces.  Not thread-safe; use one Context per thread or
 * stream.  Frames issued through one Context run in order on its stream. */
class Context {
public:
    explicit Context(cudaStream_t stream = nullptr)
        : stream_(stream)
    {
        detail::check_cuda(cudaMallocHost(&host_stats_, sizeof(dgmr_frame_stats)), "pinned statistics");
        detail::check_cuda(cudaMalloc(&device_stats_, sizeof(dgmr_frame_stats)), "device statistics");
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    ~Context()
    {
        cudaStreamSynchronize(stream_); // frames still in flight read the workspaces
        cudaFree(device_stats_);
        cudaFreeHost(host_stats_);
    }

    cudaStream_t stream() const { return stream_; }

    /* dgmr::splat_forward (splat_forward.cu:41-338) */
    Statistics splat(const SplatForwardData& d)
    {
        const dgmr_scene scene = detail::scene_of(d);
        const dgmr_camera cam = detail::camera_of(d, d.framebuffer.width, d.framebuffer.height);
        const dgmr_stream s = reinterpret_cast<dgmr_stream>(stream_);
        const size_t fbytes = dgmr_splat_frame_workspace_size(d.n_gaussians, cam.width, cam.height);
        if (fbytes == 0)
            throw Error("splat", DGMR_ERR_BAD_ARG);
        void* fws = frame_.ensure(fbytes, stream_);
        detail::check(dgmr_splat_preprocess(&scene, &cam, fws, frame_.bytes(), device_stats_, s), "splat preprocess");
        const int64_t pairs = read_stats().n_pairs;
        void* pws = pairs_.ensure(dgmr_splat_pair_workspace_size(d.n_gaussians, pairs), stream_);
        detail::check(dgmr_splat_render(&scene, &cam, d.framebuffer.data, fws, frame_.bytes(), pws, pairs_.bytes(), pairs, device_stats_, s),
            "splat render");
        return finish();
    }

    /* dgmr::vol_marcher::forward (vol_marcher_forward.cu:41-505) into the
     * caller's framebuffer; the cache stays in the Context until the next frame. */
    Statistics vol_march(Framebuffer framebuffer, const VolMarcherForwardData& d)
    {
        const dgmr_scene scene = detail::scene_of(d);
        const dgmr_camera cam = detail::camera_of(d, framebuffer.width, framebuffer.height);
        const dgmr_stream s = reinterpret_cast<dgmr_stream>(stream_);
        const int64_t n = d.n_gaussians, px = int64_t(cam.width) * cam.height;
        const int64_t tiles = int64_t((cam.width + 15) / 16) * ((cam.height + 15) / 16);
        // the cache arena: every per-Gaussian, per-tile and per-pixel output of the reference's cache
        const size_t sizes[12] = { size_t(n) * 8, size_t(n) * 12, size_t(n) * 3, size_t(n) * 4, size_t(n) * 8, size_t(n) * 24, size_t(n) * 4,
            size_t(n) * 4, size_t(n) * 4, size_t(tiles) * 8, size_t(px) * 4, 0 };
        size_t total = 0;
        for (size_t b : sizes)
            total += detail::align_up(b);
        char* base = static_cast<char*>(cache_.ensure(total, stream_));
        char* at[12];
        for (int i = 0; i < 12; ++i) {
            at[i] = base;
            base += detail::align_up(sizes[i]);
        }
        dgmr_vm_cache c {};
        c.framebuffer = framebuffer.data;
        c.rects = reinterpret_cast<int32_t*>(at[0]);
        c.rgb = at[1];
        c.rgb_sh_clamped = reinterpret_cast<uint8_t*>(at[2]);
        c.depths = at[3];
        c.points_xy_image = at[4];
        c.inverse_filtered_cov3d = at[5];
        c.filtered_masses = at[6];
        c.tiles_touched = reinterpret_cast<int32_t*>(at[7]);
        c.point_offsets = reinterpret_cast<int32_t*>(at[8]);
        c.i_ranges = reinterpret_cast<int32_t*>(at[9]);
        c.remaining_transparency = at[10];
        void* ws = frame_.ensure(dgmr_vm_workspace_size(d.n_gaussians, cam.width, cam.height, 0, DGMR_F32), stream_);
        detail::check(dgmr_vm_forward_preprocess(&scene, &cam, &c, ws, frame_.bytes(), device_stats_, s), "vol_march preprocess");
        const int64_t pairs = read_stats().n_pairs;
        c.b_point_list = static_cast<int32_t*>(pairs_.ensure(size_t(pairs > 0 ? pairs : 1) * 4, stream_));
        ws = frame_.ensure(dgmr_vm_workspace_size(d.n_gaussians, cam.width, cam.height, pairs, DGMR_F32), stream_);
        const dgmr_render_options o = detail::options_of(d.debug_render_mode, d.debug_render_bin, d.max_depth);
        detail::check(dgmr_vm_forward_render_options(&scene, &cam, &o, &c, pairs, ws, frame_.bytes(), device_stats_, s), "vol_march render");
        return finish();
    }

    /* dgmr::vol_raster_forward (vol_raster_forward.cu:39-520) */
    Statistics vol_raster(const VolRasterForwardData& d)
    {
        const dgmr_scene scene = detail::scene_of(d);
        const dgmr_camera cam = detail::camera_of(d, d.framebuffer.width, d.framebuffer.height);
        const dgmr_stream s = reinterpret_cast<dgmr_stream>(stream_);
        const size_t fbytes = dgmr_vr_frame_workspace_size(d.n_gaussians, cam.width, cam.height);
        if (fbytes == 0)
            throw Error("vol_raster", DGMR_ERR_BAD_ARG);
        void* fws = frame_.ensure(fbytes, stream_);
        detail::check(dgmr_vr_preprocess(&scene, &cam, fws, frame_.bytes(), device_stats_, s), "vol_raster preprocess");
        const int64_t pairs = read_stats().n_pairs;
        void* pws = pairs_.ensure(dgmr_vr_pair_workspace_size(d.n_gaussians, pairs), stream_);
        const dgmr_render_options o = detail::options_of(d.debug_render_mode, d.debug_render_bin, d.max_depth);
        detail::check(dgmr_vr_forward(&scene, &cam, &o, d.framebuffer.data, fws, frame_.bytes(), pws, pairs_.bytes(), pairs, device_stats_, s),
            "vol_raster forward");
        return finish();
    }

private:
    const dgmr_frame_stats& read_stats()
    {
        detail::check_cuda(cudaMemcpyAsync(host_stats_, device_stats_, sizeof(dgmr_frame_stats), cudaMemcpyDeviceToHost, stream_), "statistics read");
        detail::check_cuda(cudaStreamSynchronize(stream_), "statistics read");
        return *host_stats_;
    }
    Statistics finish()
    {
        const dgmr_frame_stats& st = read_stats();
        Statistics out;
        out.n_pairs = st.n_pairs;
        out.flags = st.flags;
        return out;
    }

    cudaStream_t stream_;
    dgmr_frame_stats* host_stats_ = nullptr;
    dgmr_frame_stats* device_stats_ = nullptr;
    detail::DeviceBuffer frame_, pairs_, cache_;
};

/* The reference's free functions (sibr_interfaces.h:24-28), on a per-thread
 * Context over the legacy default stream, as the reference runs. */
namespace sibr_interfaces {
    inline Context& default_context()
    {
        thread_local Context ctx;
        return ctx;
    }
    inline Statistics splat(SplatForwardData& forward_data) { return default_context().splat(forward_data); }
    inline Statistics vol_march(Framebuffer framebuffer, VolMarcherForwardData& forward_data)
    {
        return default_context().vol_march(framebuffer, forward_data);
    }
    inline Statistics vol_raster(VolRasterForwardData& forward_data) { return default_context().vol_raster(forward_data); }
} // namespace sibr_interfaces

} // namespace dgmr_b200

#endif
