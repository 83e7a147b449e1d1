// Volume rasteriser: src/dgmr/vol_raster_forward.cu:39-520 (forward only,
// float, as in the reference) behind the C ABI of include/dgmr_b200.h.
//
// Per pixel: (A) a RasterBinSizer places 32 depth bins from the tile's
// Gaussians in depth order until the accumulated mass reaches -log(0.005);
// (B) every Gaussian of the tile adds its CDF mass and its border values to
// the bins; (blend) each bin is fitted with the four-channel piecewise-linear
// model (create_approximation) and integrated with 256 midpoint steps.  The
// binning (tile | depth order) is the splat renderer's; the render runs one
// warp per pixel, a lane per bin (dgmr_raster_warp.cuh).
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/dgmr_b200.h"
#include "dgmr_abi_common.h"
#include "dgmr_binning.cuh"
#include "dgmr_volume_fit.h"

namespace dgmr {

constexpr unsigned kVrBins = 32; // vol_raster_forward.h:61
constexpr unsigned kVrStepsPerBin = 256; // vol_raster_forward.h:62
constexpr float kVrTransmission = 0.005f; // vol_raster_forward.h:63
constexpr float kVrRelevanceSigma = 3.f; // vol_raster_forward.h:64
constexpr float kVrFilterSD = 0.55f; // vol_raster_forward.h:60

// Frame workspace: per-Gaussian preprocess, tile ranges and binning scratch;
// pair workspace: the (tile, Gaussian) pairs and sort scratch.
struct VrLayout {
    int32_t* rects;
    float* rgb;
    uint8_t* clamped;
    float* depths;
    float* xy;
    float* inv_cov; // [N,6]
    float* masses;
    uint32_t* tiles_touched;
    uint32_t* point_offsets;
    int32_t* ranges;
    uint32_t* stats;
    BinningBuffers bin;
    size_t bytes;
    size_t pair_bytes;
};

inline VrLayout vr_layout(uint32_t N, uint32_t W, uint32_t H, uint32_t cap, void* base, void* pair_base)
{
    VrLayout L;
    Carver c;
    c.base = static_cast<char*>(base);
    const uint32_t gx = (W + kTile - 1) / kTile, gy = (H + kTile - 1) / kTile;
    L.rects = c.take<int32_t>(size_t(N) * 2);
    L.rgb = c.take<float>(size_t(N) * 3);
    L.clamped = c.take<uint8_t>(size_t(N) * 3);
    L.depths = c.take<float>(N);
    L.xy = c.take<float>(size_t(N) * 2);
    L.inv_cov = c.take<float>(size_t(N) * 6);
    L.masses = c.take<float>(N);
    L.tiles_touched = c.take<uint32_t>(N);
    L.point_offsets = c.take<uint32_t>(N);
    L.ranges = c.take<int32_t>(size_t(gx) * gy * 2);
    L.stats = c.take<uint32_t>(4);
    carve_binning_gaussians(c, L.bin, N, gx * gy);
    L.bytes = c.off;
    Carver cp;
    cp.base = static_cast<char*>(pair_base);
    carve_binning_pairs(cp, L.bin, N, cap);
    L.pair_bytes = cp.off;
    return L;
}

struct VrPre {
    uint32_t N;
    const float* centroids;
    const float* sh;
    int sh_stride, sh_degree;
    const float* weights;
    const float* scales;
    const float* rotations;
    VrLayout L;
    float aa; // filter size per unit distance
    Formulation form;
};

// vol_raster_forward.cu:86-136
__global__ void __launch_bounds__(128) k_vr_preprocess(VrPre p, CameraT<float> cam)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.N)
        return;
    const VrLayout& L = p.L;
    L.tiles_touched[i] = 0;
    L.bin.perm[i] = i;
    L.bin.depth_key[i] = 0;
    L.rects[2 * i] = 0;
    L.rects[2 * i + 1] = 0;
    L.xy[2 * i] = 0.f;
    L.xy[2 * i + 1] = 0.f;
    L.depths[i] = 0.f;
    L.masses[i] = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        L.rgb[3 * i + c] = 0.f;
        L.clamped[3 * i + c] = 0;
    }
#pragma unroll
    for (int c = 0; c < 6; ++c)
        L.inv_cov[6 * i + c] = 0.f;
    const V3<float> mu = { p.centroids[3 * i], p.centroids[3 * i + 1], p.centroids[3 * i + 2] };
    if (view_z(cam.view, mu) < 0.2f)
        return;
    const float w = p.weights[i];
    const V3<float> sc = mul3(V3<float> { p.scales[3 * i], p.scales[3 * i + 1], p.scales[3 * i + 2] }, cam.cov_scale_multiplier);
    const float* q = p.rotations + 4 * size_t(i);
    const M3<float> R = quat_to_mat3(q[0], q[1], q[2], q[3]);
    const Gaussian2d<float> g = splat_project(p.form, w, mu, sc, R, cam, 0.3f);
    const S3<float> cov3 = compute_cov(sc, R);
    const V3<float> campos = { cam.campos[0], cam.campos[1], cam.campos[2] };
    const float fks = len3(sub3(mu, campos)) * p.aa;
    const float fks2 = fks * fks;
    S3<float> filtered = cov3;
    filtered.v[0] = filtered.v[0] + fks2;
    filtered.v[3] = filtered.v[3] + fks2;
    filtered.v[5] = filtered.v[5] + fks2;
    // weight_to_mass of the scales plus the squared filter size (vol_raster_forward.cu:106)
    L.masses[i] = weight_to_mass(p.form, w, V3<float> { sc.x + fks2, sc.y + fks2, sc.z + fks2 }, g.cov);
    const int ex = dgmr_fm::to_int_rz(dgmr_fm::ceil_f(3.f * dgmr_fm::sqrt_f(g.cov.v[0])));
    const int ey = dgmr_fm::to_int_rz(dgmr_fm::ceil_f(3.f * dgmr_fm::sqrt_f(g.cov.v[2])));
    L.rects[2 * i] = ex;
    L.rects[2 * i + 1] = ey;
    const TileRect r = get_rect(g.centroid.x, g.centroid.y, ex, ey, cam.gx, cam.gy);
    const unsigned touched = (r.x1 - r.x0) * (r.y1 - r.y0);
    if (touched == 0)
        return;
    L.tiles_touched[i] = touched;
    L.xy[2 * i] = g.centroid.x;
    L.xy[2 * i + 1] = g.centroid.y;
    const float depth = len3(sub3(campos, mu));
    L.depths[i] = depth;
    L.bin.depth_key[i] = __float_as_uint(depth);
    const V3<float> v = sub3(mu, campos);
    const V3<float> dir = mul3(v, 1.f / dgmr_fm::sqrt_f(dot3(v, v)));
    uint8_t mask[3];
    const V3<float> col = sh_to_colour(p.sh, i, p.sh_stride, p.sh_degree, dir, mask);
    L.rgb[3 * i] = col.x;
    L.rgb[3 * i + 1] = col.y;
    L.rgb[3 * i + 2] = col.z;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        L.clamped[3 * i + c] = mask[c];
    const S3<float> inv = inverse_sym3(filtered);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        L.inv_cov[6 * i + c] = inv.v[c];
}

} // namespace dgmr

namespace dgmr {

struct VrRender {
    const int32_t* ranges;
    const uint32_t* list;
    const float* centroids;
    const float* inv_cov;
    const float* masses;
    const float* rgb;
    float* fb;
    uint32_t N, cap;
    uint32_t* stats;
    int mode; // dgmr_render_mode
    int debug_bin;
    float max_depth;
};

// exp(-(x - c)^2 / (2 var)), the unnormalised 1-D Gaussian
__device__ __forceinline__ float eval_exponential_1d(float c, float var, float x)
{
    const float dx = x - c;
    return dgmr_fm::exp_f((-0.5f * (dx * dx)) / var);
}

// Ray through the pixel corner at NDC z = -1 (vol_raster_forward.cu:263-268)
__device__ __forceinline__ V3<float> vr_pixel_dir(const CameraT<float>& cam, unsigned px, unsigned py)
{
    const float nx = float(px * 2u) / float(cam.W) - 1.f;
    const float ny = float(py * 2u) / float(cam.H) - 1.f;
    const float* m = cam.inv_proj;
    const float z = -1.f, o = 1.f;
    float vx = ((m[0] * nx + m[4] * ny) + m[8] * z) + m[12] * o;
    float vy = ((m[1] * nx + m[5] * ny) + m[9] * z) + m[13] * o;
    float vz = ((m[2] * nx + m[6] * ny) + m[10] * z) + m[14] * o;
    const float vw = ((m[3] * nx + m[7] * ny) + m[11] * z) + m[15] * o;
    vx = vx / vw;
    vy = vy / vw;
    vz = vz / vw;
    const V3<float> d = { vx - cam.campos[0], vy - cam.campos[1], vz - cam.campos[2] };
    const float il = 1.f / dgmr_fm::sqrt_f(dot3(d, d));
    return mul3(d, il);
}


} // namespace dgmr

#include "dgmr_raster_warp.cuh"

using namespace dgmr;

namespace {

bool vr_bad(const dgmr_scene* scene, const dgmr_camera* camera, int64_t cap)
{
    return check_scene(scene, camera, DGMR_F32) != DGMR_OK || cap < 0 || cap > int64_t(0x7fffffff);
}

void vr_launch_preprocess(const dgmr_scene* scene, const CameraT<float>& cam, const VrLayout& L, uint32_t* st_dev, cudaStream_t s)
{
    const uint32_t N = uint32_t(scene->n_gaussians);
    cudaMemsetAsync(st_dev, 0, 16, s);
    if (N == 0)
        return;
    VrPre p { N, static_cast<const float*>(scene->centroids), static_cast<const float*>(scene->sh), scene->sh_stride, scene->sh_degree,
        static_cast<const float*>(scene->weights), static_cast<const float*>(scene->scales), static_cast<const float*>(scene->rotations), L,
        ((kVrFilterSD * cam.tan_fovx) * 2.f) / float(cam.W), scene_formulation(scene, Formulation::Ots) };
    k_vr_preprocess<<<(N + 127) / 128, 128, 0, s>>>(p, cam);
    note_launch();
    inclusive_scan_u32(L.tiles_touched, L.point_offsets, N, L.bin.scan_tmp, s);
}

} // namespace

extern "C" {

size_t dgmr_vr_frame_workspace_size(int32_t n_gaussians, int32_t width, int32_t height)
{
    if (n_gaussians < 0 || width <= 0 || height <= 0 || width > 65536 || height > 65536)
        return 0;
    return vr_layout(uint32_t(n_gaussians), uint32_t(width), uint32_t(height), 0, nullptr, nullptr).bytes;
}

size_t dgmr_vr_pair_workspace_size(int32_t n_gaussians, int64_t pair_capacity)
{
    if (n_gaussians < 0 || pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff))
        return 0;
    return vr_layout(uint32_t(n_gaussians), 16, 16, uint32_t(pair_capacity), nullptr, nullptr).pair_bytes;
}

dgmr_status dgmr_vr_preprocess(const dgmr_scene* scene, const dgmr_camera* camera, void* frame_workspace, size_t frame_workspace_bytes,
    dgmr_frame_stats* stats, dgmr_stream stream)
{
    if (vr_bad(scene, camera, 0) || !frame_workspace)
        return DGMR_ERR_BAD_ARG;
    const VrLayout L = vr_layout(uint32_t(scene->n_gaussians), uint32_t(camera->width), uint32_t(camera->height), 0, frame_workspace, nullptr);
    if (frame_workspace_bytes < L.bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<float> cam = make_camera<float>(*camera);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    vr_launch_preprocess(scene, cam, L, st_dev, s);
    if (scene->n_gaussians > 0) {
        k_pair_count<<<1, 1, 0, s>>>(L.point_offsets, uint32_t(scene->n_gaussians), 0xffffffffu, st_dev, L.bin.n_sort);
        note_launch();
    }
    return launch_status();
}

dgmr_status dgmr_vr_forward(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_render_options* options, float* framebuffer, void* frame_workspace,
    size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream)
{
    if (vr_bad(scene, camera, pair_capacity) || !framebuffer || !frame_workspace || (pair_capacity > 0 && !pair_workspace))
        return DGMR_ERR_BAD_ARG;
    const int mode = options ? options->render_mode : DGMR_RENDER_FULL;
    if (mode != DGMR_RENDER_FULL && mode != DGMR_RENDER_BINS && mode != DGMR_RENDER_DEPTH)
        return DGMR_ERR_BAD_ARG;
    const uint32_t N = uint32_t(scene->n_gaussians), cap = uint32_t(pair_capacity);
    VrLayout L = vr_layout(N, uint32_t(camera->width), uint32_t(camera->height), cap, frame_workspace, pair_workspace);
    if (frame_workspace_bytes < L.bytes || pair_workspace_bytes < L.pair_bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<float> cam = make_camera<float>(*camera);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    vr_launch_preprocess(scene, cam, L, st_dev, s);
    const int par
        = run_binning<float>(N, cam.gx, cam.gy, L.tiles_touched, L.point_offsets, L.rects, L.xy, cap, L.bin, L.ranges, st_dev, num_sms(), s, true);
    VrRender a { L.ranges, L.bin.pair_val[par], static_cast<const float*>(scene->centroids), L.inv_cov, L.masses, L.rgb, framebuffer, N, cap, st_dev, mode,
        options ? options->debug_bin : -1, options ? float(options->max_depth) : 20.f };
    k_vr_render_warp<<<cam.gx * cam.gy * (kTilePixels / kVrRayWarps), kVrRayWarps * 32, 0, s>>>(a, cam);
    note_launch();
    return launch_status();
}

} // extern "C"
