// Volume ray marcher: forward (src/dgmr/vol_marcher_forward.cu:42-503) and
// backward (src/dgmr/vol_marcher_backward.cu:53-386), float and double,
// behind the C ABI of include/dgmr_b200.h.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/dgmr_b200.h"
#include "dgmr_abi_common.h"
#include "dgmr_batch.cuh"
#include "dgmr_binning.cuh"
#include "dgmr_device_grad.cuh"
#include "dgmr_marching.cuh"

namespace dgmr {

// per-Gaussian backward accumulators (double): mass, rgb(3), inverse covariance(6), centroid(3)
constexpr unsigned kVmAcc = 13;

template <class T>
struct ConstSamplesT {
    int n;
    T s[4][3];
};

static ConstSamplesT<double> g_const_samples = { 0, {} };

template <class T>
inline ConstSamplesT<T> const_samples()
{
    ConstSamplesT<T> c;
    c.n = g_const_samples.n;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 3; ++j)
            c.s[i][j] = T(g_const_samples.s[i][j]);
    return c;
}

// Workspace: [stats | preprocess scan scratch | backward accumulators |
// binning].  The first two come first so the preprocess can run on a
// workspace sized for pair_capacity = 0, before the pair count is known.
template <class T>
struct VmLayout {
    uint32_t* stats;
    uint32_t* pre_scan_tmp;
    double* acc; // backward, [N,13]: mass, rgb(3), inverse covariance(6), centroid(3)
    BinningBuffers bin;
    size_t pre_bytes;
    size_t bytes;
};

inline uint32_t frame_tiles(const dgmr_camera* camera)
{
    return ((uint32_t(camera->width) + kTile - 1) / kTile) * ((uint32_t(camera->height) + kTile - 1) / kTile);
}

template <class T>
inline VmLayout<T> vm_layout(uint32_t N, uint32_t n_tiles, uint32_t cap, void* base)
{
    VmLayout<T> L;
    Carver c;
    c.base = static_cast<char*>(base);
    L.stats = c.take<uint32_t>(4);
    L.pre_scan_tmp = c.take<uint32_t>(scan_temp_bytes(N) / 4 + 8); // + room for k_pair_count's eight counters
    L.pre_bytes = c.off;
    L.acc = c.take<double>(size_t(N) * kVmAcc);
    carve_binning(c, L.bin, N, n_tiles, cap);
    L.bytes = c.off;
    return L;
}

// depth keys (float bits of the cached depth) and the identity permutation
template <class T>
__global__ void k_depth_keys(const T* __restrict__ depths, uint32_t N, uint32_t* __restrict__ depth_key, uint32_t* __restrict__ perm)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) {
        depth_key[i] = __float_as_uint(float(depths[i]));
        perm[i] = i;
    }
}

template <class T>
struct VmPre {
    uint32_t N;
    const T* centroids;
    const T* sh;
    int sh_stride, sh_degree;
    const T* weights;
    const T* scales;
    const T* rotations;
    int32_t* rects;
    T* rgb;
    uint8_t* clamped;
    T* depths;
    T* xy;
    T* inv_cov;
    T* masses;
    uint32_t* tiles_touched;
    T aa; // filter_kernel_SD * 2 * tan_fovx / width
    Formulation form;
};

// vol_marcher_forward.cu:98-176.  Gaussian i of the scene, written to slot o
// of the per-frame arrays (o = i for one frame; the view's offset + i in a batch).
template <class T>
__device__ __forceinline__ void vm_preprocess_one(const VmPre<T>& p, const CameraT<T>& cam, uint32_t i, uint32_t o)
{
    p.tiles_touched[o] = 0;
    p.rects[2 * o] = 0;
    p.rects[2 * o + 1] = 0;
    p.xy[2 * o] = T(0);
    p.xy[2 * o + 1] = T(0);
    p.depths[o] = T(0);
    p.masses[o] = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        p.rgb[3 * o + k] = T(0);
        p.clamped[3 * o + k] = 0;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k)
        p.inv_cov[6 * o + k] = T(0);
    const V3<T> mu = { p.centroids[3 * i], p.centroids[3 * i + 1], p.centroids[3 * i + 2] };
    if (view_z(cam.view, mu) < T(0.2f))
        return;
    const T w = p.weights[i];
    const V3<T> sc = mul3(V3<T> { p.scales[3 * i], p.scales[3 * i + 1], p.scales[3 * i + 2] }, cam.cov_scale_multiplier);
    const T* q = p.rotations + 4 * size_t(i);
    const M3<T> R = quat_to_mat3(q[0], q[1], q[2], q[3]);
    const V3<T> campos = { cam.campos[0], cam.campos[1], cam.campos[2] };
    const T dist = len3(sub3(campos, mu));
    const S3<T> cov3 = compute_cov(sc, R);
    const T fks = dist * p.aa;
    const T fks2 = fks * fks;
    S3<T> filtered = cov3;
    filtered.v[0] = filtered.v[0] + fks2;
    filtered.v[3] = filtered.v[3] + fks2;
    filtered.v[5] = filtered.v[5] + fks2;
    const T mass = weight_to_mass(p.form, w, sc, affine_transform_and_cut(cov3, upper3(cam.view)));
    if (mass <= T(0))
        return;
    const Gaussian2d<T> g = splat_project(p.form, w, mu, sc, R, cam, T(kFilterSD * kFilterSD));
    const auto iso = [](T wt, T var, T isoline) {
        const T sv = T(-2) * dgmr_fm::log_f(isoline / wt);
        if (sv <= T(0))
            return T(0);
        return dgmr_fm::sqrt_f(sv * var);
    };
    const int ex = dgmr_fm::to_int_rz(dgmr_fm::ceil_f(iso(g.weight, g.cov.v[0], T(1.f / 255.f))));
    const int ey = dgmr_fm::to_int_rz(dgmr_fm::ceil_f(iso(g.weight, g.cov.v[2], T(1.f / 255.f))));
    p.rects[2 * o] = ex;
    p.rects[2 * o + 1] = ey;
    const TileRect r = get_rect(float(g.centroid.x), float(g.centroid.y), ex, ey, cam.gx, cam.gy);
    const unsigned touched = (r.x1 - r.x0) * (r.y1 - r.y0);
    if (touched == 0)
        return;
    p.tiles_touched[o] = touched;
    p.xy[2 * o] = g.centroid.x;
    p.xy[2 * o + 1] = g.centroid.y;
    const S3<T> inv = inverse_sym3(filtered);
    const T smax = max_f(sc.x, max_f(sc.y, sc.z));
    const T depth = dist - (smax * T(kRelevanceSigma)) / T(2);
    p.depths[o] = depth;
    const V3<T> dir = { (mu.x - campos.x) / dist, (mu.y - campos.y) / dist, (mu.z - campos.z) / dist };
    uint8_t mask[3];
    const V3<T> col = sh_to_colour(p.sh, i, p.sh_stride, p.sh_degree, dir, mask);
    p.rgb[3 * o] = col.x;
    p.rgb[3 * o + 1] = col.y;
    p.rgb[3 * o + 2] = col.z;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        p.clamped[3 * o + k] = mask[k];
#pragma unroll
    for (int k = 0; k < 6; ++k)
        p.inv_cov[6 * o + k] = inv.v[k];
    p.masses[o] = mass;
}

template <class T>
__global__ void __launch_bounds__(128) k_vm_preprocess(VmPre<T> p, CameraT<T> cam)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < p.N)
        vm_preprocess_one(p, cam, i, i);
}

// Ray through the pixel centre (vol_marcher_forward.cu:308-315)
template <class T>
__device__ __forceinline__ V3<T> pixel_dir(const CameraT<T>& cam, unsigned px, unsigned py)
{
    const T pxc = T(px) + T(0.5);
    const T pyc = T(py) + T(0.5);
    const T nx = (pxc * T(2)) / T(float(cam.W)) - T(1);
    const T ny = (pyc * T(2)) / T(float(cam.H)) - T(1);
    const T* m = cam.inv_proj;
    const T z = T(0), o = T(1);
    T vx = ((m[0] * nx + m[4] * ny) + m[8] * z) + m[12] * o;
    T vy = ((m[1] * nx + m[5] * ny) + m[9] * z) + m[13] * o;
    T vz = ((m[2] * nx + m[6] * ny) + m[10] * z) + m[14] * o;
    const T vw = ((m[3] * nx + m[7] * ny) + m[11] * z) + m[15] * o;
    vx = vx / vw;
    vy = vy / vw;
    vz = vz / vw;
    const V3<T> d = { vx - cam.campos[0], vy - cam.campos[1], vz - cam.campos[2] };
    const T il = T(1) / dgmr_fm::sqrt_f(dot3(d, d));
    return mul3(d, il);
}

template <class T>
struct VmMarch {
    const int32_t* ranges;
    const int32_t* list;
    const T* centroids;
    const T* inv_cov;
    const T* masses;
    const T* rgb;
    const T* depths;
    T* fb;
    T* remaining_T;
    const T* grad_fb; // backward only
    double* acc; // backward only: [N,13] (kVmAcc)
    uint32_t* stats;
    ConstSamplesT<T> cs;
    int mode; // dgmr_render_mode (forward)
    int debug_bin;
    T max_depth;
    unsigned long long* work; // forward, optional: (ray, Gaussian, large step) bin fills
    // optional step store: the forward writes, the backward reads, for the first
    // store_steps large steps of every ray, its kSmallSteps sample borders
    // ([step][ray][kSmallSteps]) and its section count ([step][ray])
    T* store_borders;
    int32_t* store_sections;
    uint32_t store_steps;
};

// the step store inside one buffer: the borders first, then the section counts
template <class T>
inline void carve_step_store(void* base, uint32_t n_rays, uint32_t steps, T** borders, int32_t** sections)
{
    char* p = static_cast<char*>(base);
    *borders = reinterpret_cast<T*>(p);
    *sections = reinterpret_cast<int32_t*>(p + align_up(size_t(steps) * n_rays * kSmallSteps * sizeof(T)));
}

inline size_t step_store_bytes(uint32_t n_rays, uint32_t steps, size_t elem)
{
    return align_up(size_t(steps) * n_rays * kSmallSteps * elem) + align_up(size_t(steps) * n_rays * sizeof(int32_t));
}

// Which Gaussians of the tile list a ray can use.  Both passes of every large
// step only act on a Gaussian that passes its gate -- pass 1's (mass on the
// ray in (1/255, 1000], positive variance, finite centre) or pass 2's
// (gaussian_on_ray) -- and the gates depend on the ray alone, not on the
// step.  So a first pass over the tile records, per ray and per batch of list
// entries, a mask of the entries that pass either gate, and the large steps
// only intersect those.  Pass 1's depth break also only needs them: the list
// is in depth order, so the first entry with depth > end of the section set
// that is skipped here would be followed by a masked entry with a depth at
// least as large, checked against the same end.  The results are identical;
// the per-step cost drops from the tile's list to the ray's own Gaussians.
template <class T>
__device__ __forceinline__ bool ray_can_use(const Gauss1d<T>& g, T mass)
{
    const T mor = g.weight * mass;
    const bool pass1 = !(mor <= T(1.0f / 255.f) || mor > T(1000)) && !(g.C <= T(0)) && !dgmr_fm::isnan_f(g.centre);
    T sd, mor2;
    const bool pass2 = gaussian_on_ray(g, mass, &sd, &mor2);
    return pass1 || pass2;
}

} // namespace dgmr

#include "dgmr_march_warp.cuh"

namespace dgmr {

template <class T>
struct VmBwdGauss {
    uint32_t N;
    const T* centroids;
    const T* sh;
    int sh_stride, sh_degree;
    const T* weights;
    const T* scales;
    const T* rotations;
    const uint8_t* clamped;
    const int32_t* tiles_touched;
    const double* acc;
    T* g_sh;
    T* g_weights;
    T* g_centroids; // the march's contribution plus the chain rule's
    T* g_scales;
    T* g_rotations;
    T aa;
    Formulation form;
};

// vol_marcher_backward.cu:321-384, for Gaussian i of the scene seen in slot o
// (o = i for one frame).  kAdd = false writes the gradient rows (a single
// frame); kAdd = true adds this view's rows to them (a batch, whose views of
// one scene are added in view order after the rows are zeroed).  Each term
// added is the value a single frame writes, so a batch's gradient is the sum,
// in view order, of the single-view gradients.
template <class T, bool kAdd>
__device__ __forceinline__ void vm_bwd_gaussian_one(const VmBwdGauss<T>& p, const CameraT<T>& cam, T aa, uint32_t i, uint32_t o)
{
    const double* a = p.acc + size_t(o) * kVmAcc;
    const V3<T> g_march = { T(a[10]), T(a[11]), T(a[12]) }; // the march's own centroid gradient
    const auto put_centroid = [&](V3<T> g) {
        if (kAdd) {
            p.g_centroids[3 * i] += g.x;
            p.g_centroids[3 * i + 1] += g.y;
            p.g_centroids[3 * i + 2] += g.z;
        } else {
            p.g_centroids[3 * i] = g.x;
            p.g_centroids[3 * i + 1] = g.y;
            p.g_centroids[3 * i + 2] = g.z;
        }
    };
    if (!kAdd) {
        for (int k = 0; k < p.sh_stride * 3; ++k)
            p.g_sh[size_t(i) * p.sh_stride * 3 + k] = T(0);
        p.g_weights[i] = T(0);
#pragma unroll
        for (int k = 0; k < 3; ++k)
            p.g_scales[3 * i + k] = T(0);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            p.g_rotations[4 * i + k] = T(0);
    }
    if (p.tiles_touched[o] == 0) {
        put_centroid(g_march);
        return;
    }
    const V3<T> mu = { p.centroids[3 * i], p.centroids[3 * i + 1], p.centroids[3 * i + 2] };
    if (view_z(cam.view, mu) < T(0.2)) {
        put_centroid(g_march);
        return;
    }
    const T w = p.weights[i];
    // the reference does not apply cov_scale_multiplier in the backward (vol_marcher_backward.cu:342)
    const V3<T> sc = { p.scales[3 * i], p.scales[3 * i + 1], p.scales[3 * i + 2] };
    const T* q = p.rotations + 4 * size_t(i);
    const M3<T> R = quat_to_mat3(q[0], q[1], q[2], q[3]);
    const V3<T> campos = { cam.campos[0], cam.campos[1], cam.campos[2] };
    const V3<T> delta = sub3(mu, campos);
    const T dist = len3(delta);
    const S3<T> cov3 = compute_cov(sc, R);
    const T fks = dist * aa;
    S3<T> filtered = cov3;
    filtered.v[0] = filtered.v[0] + fks * fks;
    filtered.v[3] = filtered.v[3] + fks * fks;
    filtered.v[5] = filtered.v[5] + fks * fks;
    const M3<T> W3 = upper3(cam.view);
    const S2<T> cov2d = affine_transform_and_cut(cov3, W3);
    const T mass = weight_to_mass(p.form, w, sc, cov2d);
    if (mass <= T(0)) {
        put_centroid(g_march);
        return;
    }
    const V3<T> dir = { delta.x / dist, delta.y / dist, delta.z / dist };
    const V3<T> g_dir = grad_sh_to_colour(p.sh, i, p.sh_stride, p.sh_degree, dir, V3<T> { T(a[1]), T(a[2]), T(a[3]) }, p.clamped + 3 * size_t(o), T(1),
        p.g_sh, kAdd);
    V3<T> g_mu = mul3(g_dir, T(1) / dist);
    T g_dist = -dot3(g_dir, delta) / (dist * dist);
    S3<T> g_inv;
#pragma unroll
    for (int k = 0; k < 6; ++k)
        g_inv.v[k] = T(a[4 + k]);
    const S3<T> g_filtered = grad_inverse_sym3(filtered, g_inv);
    // adjoint of weight_to_mass (math.h:298-320)
    const T g_mass = T(a[0]);
    T g_w = T(0);
    S2<T> g_cov2d = { { T(0), T(0), T(0) } };
    V3<T> g_s = { T(0), T(0), T(0) };
    if (p.form == Formulation::Opacity) {
        const T dcov = det2(cov2d);
        const T i2 = integrate_exponential_cov2(cov2d);
        g_w = g_mass * i2;
        const T g_i2 = g_mass * w;
        const T g_det = (dcov > T(0)) ? g_i2 * two_pi<T>() / (T(2) * dgmr_fm::sqrt_f(dcov)) : T(0);
        g_cov2d = { { g_det * cov2d.v[2], g_det * T(-2) * cov2d.v[1], g_det * cov2d.v[0] } };
    } else if (p.form == Formulation::Mass) {
        g_w = g_mass;
    } else if (p.form == Formulation::Density) {
        g_w = g_mass * integrate_exponential3(sc);
        const T k = (g_mass * w) * two_pi_pow_1_5<T>();
        g_s = { k * sc.y * sc.z, k * sc.x * sc.z, k * sc.x * sc.y };
    } else {
        const V2<T> l2 = p.form == Formulation::Ots ? larger2(sc) : smaller2(sc);
        g_w = g_mass * integrate_exponential2(l2);
        const T k = (g_mass * w) * two_pi<T>();
        const V2<T> g_l2 = { k * l2.y, k * l2.x };
        g_s = p.form == Formulation::Ots ? grad_larger2(sc, g_l2) : grad_smaller2(sc, g_l2);
    }
    S3<T> g_cov3 = g_filtered;
    const T g_fks2 = (g_filtered.v[0] + g_filtered.v[3]) + g_filtered.v[5];
    g_dist = g_dist + (g_fks2 * T(2) * fks) * aa;
    grad_affine_transform_and_cut(cov3, W3, g_cov2d, &g_cov3, static_cast<M3<T>*>(nullptr));
    T g_q[4] = { T(0), T(0), T(0), T(0) };
    grad_compute_cov(sc, q[0], q[1], q[2], q[3], g_cov3, &g_s, g_q);
    g_mu = add3(g_mu, mul3(delta, g_dist / dist));
    if (kAdd) {
        p.g_weights[i] += g_w;
        p.g_scales[3 * i] += g_s.x;
        p.g_scales[3 * i + 1] += g_s.y;
        p.g_scales[3 * i + 2] += g_s.z;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            p.g_rotations[4 * i + k] += g_q[k];
    } else {
        p.g_weights[i] = g_w;
        p.g_scales[3 * i] = g_s.x;
        p.g_scales[3 * i + 1] = g_s.y;
        p.g_scales[3 * i + 2] = g_s.z;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            p.g_rotations[4 * i + k] = g_q[k];
    }
    put_centroid(V3<T> { g_march.x + g_mu.x, g_march.y + g_mu.y, g_march.z + g_mu.z });
}

template <class T>
__global__ void __launch_bounds__(128) k_vm_bwd_gaussians(VmBwdGauss<T> p, CameraT<T> cam)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < p.N)
        vm_bwd_gaussian_one<T, false>(p, cam, p.aa, i, i);
}

// Heaviest-tile-first order of the march's blocks, in the workspace past the
// layout (none -- natural order -- if the workspace has no room for it).
template <class T>
inline const uint32_t* march_order(const int32_t* ranges, const CameraT<T>& cam, void* workspace, size_t layout_bytes, size_t workspace_bytes,
    cudaStream_t s)
{
    const uint32_t n_tiles = cam.gx * cam.gy;
    const size_t off = align_up(layout_bytes);
    if (!workspace || workspace_bytes < off + size_t(n_tiles) * sizeof(uint32_t))
        return nullptr;
    uint32_t* order = reinterpret_cast<uint32_t*>(static_cast<char*>(workspace) + off);
    k_tile_order<<<1, 1024, 0, s>>>(ranges, n_tiles, order);
    note_launch();
    return order;
}

template <class T>
__host__ __device__ inline T aa_multiplier(const CameraT<T>& cam)
{
    return ((T(kFilterSD) * cam.tan_fovx) * T(2)) / T(float(cam.W));
}

template <class T>
dgmr_status vm_preprocess(const dgmr_scene* scene, const dgmr_camera* camera, dgmr_vm_cache* c, void* workspace, size_t workspace_bytes,
    dgmr_frame_stats* stats, cudaStream_t s)
{
    const uint32_t N = uint32_t(scene->n_gaussians);
    const VmLayout<T> Lw = vm_layout<T>(N, frame_tiles(camera), 0, workspace);
    if (workspace_bytes < Lw.pre_bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<T> cam = make_camera<T>(*camera);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : Lw.stats;
    cudaMemsetAsync(st_dev, 0, 16, s);
    if (N == 0)
        return launch_status();
    VmPre<T> p { N, static_cast<const T*>(scene->centroids), static_cast<const T*>(scene->sh), scene->sh_stride, scene->sh_degree,
        static_cast<const T*>(scene->weights), static_cast<const T*>(scene->scales), static_cast<const T*>(scene->rotations), c->rects, static_cast<T*>(c->rgb),
        c->rgb_sh_clamped, static_cast<T*>(c->depths), static_cast<T*>(c->points_xy_image), static_cast<T*>(c->inverse_filtered_cov3d),
        static_cast<T*>(c->filtered_masses), reinterpret_cast<uint32_t*>(c->tiles_touched), aa_multiplier(cam),
        scene_formulation(scene, Formulation::Opacity) };
    k_vm_preprocess<T><<<(N + 127) / 128, 128, 0, s>>>(p, cam);
    note_launch();
    inclusive_scan_u32(reinterpret_cast<uint32_t*>(c->tiles_touched), reinterpret_cast<uint32_t*>(c->point_offsets), N, Lw.pre_scan_tmp, s);
    k_pair_count<<<1, 1, 0, s>>>(reinterpret_cast<uint32_t*>(c->point_offsets), N, 0xffffffffu, st_dev, Lw.pre_scan_tmp);
    note_launch();
    return launch_status();
}

template <class T>
dgmr_status vm_render(const dgmr_scene* scene, const dgmr_camera* camera, dgmr_vm_cache* c, int64_t cap64, void* workspace, size_t workspace_bytes,
    dgmr_frame_stats* stats, cudaStream_t s, const dgmr_render_options* options, void* store = nullptr, uint32_t store_steps = 0)
{
    const uint32_t N = uint32_t(scene->n_gaussians), cap = uint32_t(cap64);
    const VmLayout<T> L = vm_layout<T>(N, frame_tiles(camera), cap, workspace);
    if (workspace_bytes < L.bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<T> cam = make_camera<T>(*camera);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    cudaMemsetAsync(st_dev, 0, 16, s);
    BinningBuffers bin = L.bin;
    if (N > 0)
        k_depth_keys<T><<<(N + 255) / 256, 256, 0, s>>>(static_cast<const T*>(c->depths), N, bin.depth_key, bin.perm);
    if (N > 0)
        note_launch();
    const int par = run_binning<T>(N, cam.gx, cam.gy, reinterpret_cast<uint32_t*>(c->tiles_touched), reinterpret_cast<uint32_t*>(c->point_offsets), c->rects,
        static_cast<T*>(c->points_xy_image), cap, bin, c->i_ranges, st_dev, num_sms(), s, true);
    if (cap > 0)
        cudaMemcpyAsync(c->b_point_list, bin.pair_val[par], size_t(cap) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    VmMarch<T> a {};
    a.ranges = c->i_ranges;
    a.list = c->b_point_list;
    a.centroids = static_cast<const T*>(scene->centroids);
    a.inv_cov = static_cast<const T*>(c->inverse_filtered_cov3d);
    a.masses = static_cast<const T*>(c->filtered_masses);
    a.rgb = static_cast<const T*>(c->rgb);
    a.depths = static_cast<const T*>(c->depths);
    a.fb = static_cast<T*>(c->framebuffer);
    a.remaining_T = static_cast<T*>(c->remaining_transparency);
    a.stats = st_dev;
    a.cs = const_samples<T>();
    a.mode = options ? options->render_mode : DGMR_RENDER_FULL;
    a.debug_bin = options ? options->debug_bin : -1;
    a.max_depth = options ? T(options->max_depth) : T(20);
    a.work = options ? options->work_counter : nullptr;
    if (store && store_steps > 0) {
        carve_step_store<T>(store, uint32_t(camera->width) * uint32_t(camera->height), store_steps, &a.store_borders, &a.store_sections);
        a.store_steps = store_steps;
    }
    const uint32_t* order = march_order(c->i_ranges, cam, workspace, L.bytes, workspace_bytes, s);
    k_vm_march_warp<T, VmSingleFrame<T>><<<cam.gx * cam.gy * (kTilePixels / kRayWarps), kRayWarps * 32, 0, s>>>(a, VmSingleFrame<T> { cam }, order);
    note_launch();
    return launch_status();
}

template <class T>
dgmr_status vm_backward(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_vm_cache* c, const void* grad_fb, void* g_sh, void* g_weights,
    void* g_centroids, void* g_scales, void* g_rotations, void* workspace, size_t workspace_bytes, dgmr_frame_stats* stats, cudaStream_t s,
    const void* store = nullptr, uint32_t store_steps = 0)
{
    const uint32_t N = uint32_t(scene->n_gaussians);
    const VmLayout<T> L = vm_layout<T>(N, frame_tiles(camera), 0, workspace);
    if (workspace_bytes < L.bytes)
        return DGMR_ERR_WORKSPACE;
    const CameraT<T> cam = make_camera<T>(*camera);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    if (N == 0)
        return DGMR_OK;
    cudaMemsetAsync(L.acc, 0, size_t(N) * kVmAcc * sizeof(double), s);
    VmMarch<T> a {};
    a.ranges = c->i_ranges;
    a.list = c->b_point_list;
    a.centroids = static_cast<const T*>(scene->centroids);
    a.inv_cov = static_cast<const T*>(c->inverse_filtered_cov3d);
    a.masses = static_cast<const T*>(c->filtered_masses);
    a.rgb = static_cast<const T*>(c->rgb);
    a.depths = static_cast<const T*>(c->depths);
    a.fb = static_cast<T*>(c->framebuffer);
    a.remaining_T = static_cast<T*>(c->remaining_transparency);
    a.grad_fb = static_cast<const T*>(grad_fb);
    a.acc = L.acc;
    a.stats = st_dev;
    a.cs = const_samples<T>();
    if (store && store_steps > 0) {
        carve_step_store<T>(const_cast<void*>(store), uint32_t(camera->width) * uint32_t(camera->height), store_steps, &a.store_borders,
            &a.store_sections);
        a.store_steps = store_steps;
    }
    const uint32_t* order = march_order(c->i_ranges, cam, workspace, L.bytes, workspace_bytes, s);
    k_vm_march_warp_bwd<T, VmSingleFrame<T>><<<cam.gx * cam.gy * (kTilePixels / kRayWarps), kRayWarps * 32, 0, s>>>(a, VmSingleFrame<T> { cam }, order);
    note_launch();
    VmBwdGauss<T> p { N, static_cast<const T*>(scene->centroids), static_cast<const T*>(scene->sh), scene->sh_stride, scene->sh_degree,
        static_cast<const T*>(scene->weights), static_cast<const T*>(scene->scales), static_cast<const T*>(scene->rotations), c->rgb_sh_clamped,
        c->tiles_touched, L.acc, static_cast<T*>(g_sh), static_cast<T*>(g_weights), static_cast<T*>(g_centroids), static_cast<T*>(g_scales),
        static_cast<T*>(g_rotations), aa_multiplier(cam), scene_formulation(scene, Formulation::Opacity) };
    k_vm_bwd_gaussians<T><<<(N + 127) / 128, 128, 0, s>>>(p, cam);
    note_launch(2);
    return launch_status();
}

// The per-pixel and per-tile arrays are always needed; the per-Gaussian ones
// only when there are Gaussians (an empty tensor may have no address).
inline bool cache_ok(const dgmr_vm_cache* c, bool need_list, int32_t n_gaussians)
{
    if (!c || !c->framebuffer || !c->i_ranges || !c->remaining_transparency || (need_list && !c->b_point_list))
        return false;
    return n_gaussians == 0
        || (c->rects && c->rgb && c->rgb_sh_clamped && c->depths && c->points_xy_image && c->inverse_filtered_cov3d && c->filtered_masses
            && c->tiles_touched && c->point_offsets);
}

// ---------------------------------------------------------------------------
// Batched volume marching (no reference counterpart: the reference marches
// one view per call, vol_marcher_forward.cu:42-503).  Many views of one or
// several scenes (float32) go through ONE launch sequence over the view table
// of dgmr_batch.cuh: one preprocess over every (view, Gaussian) slot, the
// splat renderer's batched binning, one march over the tiles of all views
// (heaviest first) and, for the backward, one backward march plus one pass
// over every scene Gaussian that adds its views in view order.  Each view's
// point list is the one it gets alone (the binning keeps every view's
// (depth, index) order), and the march of a ray reads only its own view's
// list, camera and planes, so each image is the same, bit for bit, as a
// dgmr_vm_forward_render of that view.

// The batch's frames for the march kernels.
struct VmBatchFrames {
    BatchTable tab;
    __device__ __forceinline__ unsigned view(unsigned t) const { return BatchTable::owner(tab.tile_off, tab.n_views, t); }
    __device__ __forceinline__ const CameraT<float>& cam(unsigned v) const { return tab.views[v].cam; }
    __device__ __forceinline__ unsigned tile_base(unsigned v) const { return tab.tile_off[v]; }
    __device__ __forceinline__ size_t px_base(unsigned v) const { return tab.views[v].px_off; }
    __device__ __forceinline__ size_t rays() const { return tab.px_total; }
    __device__ __forceinline__ float* fb(unsigned v, const VmMarch<float>&) const { return tab.views[v].fb; }
    __device__ __forceinline__ float* remaining_T(unsigned v, const VmMarch<float>&) const { return tab.final_T + tab.views[v].px_off; }
    __device__ __forceinline__ const float* grad_fb(unsigned v, const VmMarch<float>&) const { return tab.views[v].grad_fb; }
};

// Frame workspace: statistics, the per-slot arrays (the single frame's cache,
// plus a copy of each slot's centroid so the march reads every list entry by
// its slot), the backward's accumulators, ranges, remaining transmittance of
// every pixel, the march order and the binning's Gaussian-sized buffers.
// Pair workspace: the binning's pair buffers and sort scratch.
struct VmBatchLayout {
    uint32_t* stats;
    int32_t* rects;
    float* rgb;
    uint8_t* clamped;
    float* depths;
    float* xy;
    float* inv_cov;
    float* masses;
    uint32_t* tiles_touched;
    uint32_t* point_offsets;
    float* centroids;
    double* acc;
    int32_t* ranges;
    float* remaining_T;
    uint32_t* tile_order;
    BinningBuffers bin;
    size_t bytes;
    size_t pair_bytes;
};

inline VmBatchLayout vm_batch_layout(uint32_t G, uint32_t n_tiles, size_t n_px, uint32_t cap, void* base, void* pair_base)
{
    VmBatchLayout L;
    Carver c;
    c.base = static_cast<char*>(base);
    L.stats = c.take<uint32_t>(4);
    L.rects = c.take<int32_t>(size_t(G) * 2);
    L.rgb = c.take<float>(size_t(G) * 3);
    L.clamped = c.take<uint8_t>(size_t(G) * 3);
    L.depths = c.take<float>(G);
    L.xy = c.take<float>(size_t(G) * 2);
    L.inv_cov = c.take<float>(size_t(G) * 6);
    L.masses = c.take<float>(G);
    L.tiles_touched = c.take<uint32_t>(G);
    L.point_offsets = c.take<uint32_t>(G);
    L.centroids = c.take<float>(size_t(G) * 3);
    L.acc = c.take<double>(size_t(G) * kVmAcc);
    L.ranges = c.take<int32_t>(size_t(n_tiles) * 2);
    L.remaining_T = c.take<float>(n_px);
    L.tile_order = c.take<uint32_t>(n_tiles);
    carve_binning_gaussians(c, L.bin, G, n_tiles);
    L.bytes = c.off;
    Carver pc;
    pc.base = static_cast<char*>(pair_base);
    carve_binning_pairs(pc, L.bin, G, cap);
    L.pair_bytes = pc.off;
    return L;
}

// One thread per (view, Gaussian) slot: the single frame's preprocess with the
// view's camera, then the slot's depth key, identity permutation and centroid.
__global__ void __launch_bounds__(128) k_vm_batch_preprocess(VmPre<float> out, float* __restrict__ slot_centroids, uint32_t* __restrict__ depth_key,
    uint32_t* __restrict__ perm, const __grid_constant__ BatchTable tab)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= tab.G)
        return;
    const uint32_t v = BatchTable::owner(tab.g_off, tab.n_views, g);
    const BatchView& bv = tab.views[v];
    const BatchScene& sc = tab.scenes[bv.scene];
    const uint32_t i = g - tab.g_off[v];
    VmPre<float> p = out;
    p.N = sc.n;
    p.centroids = sc.centroids;
    p.sh = sc.sh;
    p.sh_stride = sc.sh_stride;
    p.sh_degree = sc.sh_degree;
    p.weights = sc.weights;
    p.scales = sc.scales;
    p.rotations = sc.rotations;
    p.aa = aa_multiplier(bv.cam);
    p.form = sc.form;
    vm_preprocess_one(p, bv.cam, i, g);
    depth_key[g] = __float_as_uint(p.depths[g]);
    perm[g] = g;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        slot_centroids[3 * size_t(g) + k] = sc.centroids[3 * size_t(i) + k];
}

// per scene Gaussian: zero its gradient rows, then add the chain rule of every
// view of its scene that has an image gradient, in view order
__global__ void __launch_bounds__(128) k_vm_batch_bwd_gaussians(VmBwdGauss<float> state, const __grid_constant__ BatchTable tab)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= tab.scene_off[tab.n_scenes])
        return;
    const uint32_t s = BatchTable::owner(tab.scene_off, tab.n_scenes, k);
    const BatchScene& sc = tab.scenes[s];
    const uint32_t i = k - tab.scene_off[s];
    if (!sc.g_sh) // a scene entry without gradient outputs
        return;
    VmBwdGauss<float> p = state;
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
    for (int c = 0; c < p.sh_stride * 3; ++c)
        p.g_sh[size_t(i) * p.sh_stride * 3 + c] = 0.f;
    p.g_weights[i] = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        p.g_centroids[3 * i + c] = 0.f;
        p.g_scales[3 * i + c] = 0.f;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
        p.g_rotations[4 * i + c] = 0.f;
    for (uint32_t q = sc.view_begin; q < sc.view_end; ++q) {
        const uint32_t v = tab.view_by_scene[q];
        if (tab.views[v].grad_fb)
            vm_bwd_gaussian_one<float, true>(p, tab.views[v].cam, aa_multiplier(tab.views[v].cam), i, tab.g_off[v] + i);
    }
}

struct VmBatchPlan {
    BatchTable tab;
    VmBatchLayout L;
};

// Validates the batch and builds its table and layout.  grads may be null
// (forward); the bases may be null (size query).
dgmr_status make_vm_batch(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, const dgmr_scene_grads* grads,
    int64_t pair_capacity, void* frame_ws, void* pair_ws, VmBatchPlan& plan)
{
    if (pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff))
        return DGMR_ERR_BAD_ARG;
    BatchTable& t = plan.tab;
    const dgmr_status st = build_batch_table(scenes, n_scenes, views, n_views, grads, Formulation::Opacity, t);
    if (st != DGMR_OK)
        return st;
    plan.L = vm_batch_layout(t.G, t.n_tiles, t.px_total, uint32_t(pair_capacity), frame_ws, pair_ws);
    t.final_T = plan.L.remaining_T;
    t.n_contrib = nullptr;
    return DGMR_OK;
}

dgmr_status vm_batch_check_ws(const VmBatchPlan& plan, void* frame_ws, size_t frame_bytes, void* pair_ws, size_t pair_bytes, int64_t pair_capacity,
    bool need_pairs = true)
{
    if (!frame_ws || (need_pairs && pair_capacity > 0 && !pair_ws))
        return DGMR_ERR_BAD_ARG;
    if (frame_bytes < plan.L.bytes || (need_pairs && pair_bytes < plan.L.pair_bytes))
        return DGMR_ERR_WORKSPACE;
    return DGMR_OK;
}

void vm_batch_preprocess(const VmBatchPlan& plan, uint32_t* st_dev, cudaStream_t s)
{
    const VmBatchLayout& L = plan.L;
    const uint32_t G = plan.tab.G;
    cudaMemsetAsync(st_dev, 0, 16, s);
    if (G == 0)
        return;
    VmPre<float> p { G, nullptr, nullptr, 1, 0, nullptr, nullptr, nullptr, L.rects, L.rgb, L.clamped, L.depths, L.xy, L.inv_cov, L.masses,
        L.tiles_touched, 0.f, Formulation::Opacity };
    k_vm_batch_preprocess<<<(G + 127) / 128, 128, 0, s>>>(p, L.centroids, L.bin.depth_key, L.bin.perm, plan.tab);
    note_launch();
    inclusive_scan_u32(L.tiles_touched, L.point_offsets, G, L.bin.scan_tmp, s);
}

// the march's entries: every list entry is a slot of the batch
VmMarch<float> vm_batch_march(const VmBatchLayout& L, const uint32_t* list, uint32_t* st_dev)
{
    VmMarch<float> a {};
    a.ranges = L.ranges;
    a.list = reinterpret_cast<const int32_t*>(list);
    a.centroids = L.centroids;
    a.inv_cov = L.inv_cov;
    a.masses = L.masses;
    a.rgb = L.rgb;
    a.depths = L.depths;
    a.stats = st_dev;
    a.cs = const_samples<float>();
    a.mode = DGMR_RENDER_FULL;
    a.debug_bin = -1;
    a.max_depth = 20.f;
    return a;
}

} // namespace dgmr

using namespace dgmr;

extern "C" {

size_t dgmr_vm_workspace_size(int32_t n_gaussians, int32_t width, int32_t height, int64_t pair_capacity, int32_t dtype)
{
    if (n_gaussians < 0 || width <= 0 || height <= 0 || pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff))
        return 0;
    const uint32_t n_tiles = ((uint32_t(width) + kTile - 1) / kTile) * ((uint32_t(height) + kTile - 1) / kTile);
    const size_t masks = size_t(n_tiles) * sizeof(uint32_t); // march order
    if (dtype == DGMR_F64)
        return align_up(vm_layout<double>(uint32_t(n_gaussians), n_tiles, uint32_t(pair_capacity), nullptr).bytes) + masks;
    return align_up(vm_layout<float>(uint32_t(n_gaussians), n_tiles, uint32_t(pair_capacity), nullptr).bytes) + masks;
}

dgmr_status dgmr_vm_forward_preprocess(const dgmr_scene* scene, const dgmr_camera* camera, dgmr_vm_cache* cache, void* workspace, size_t workspace_bytes,
    dgmr_frame_stats* stats, dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, -1);
    if (st != DGMR_OK)
        return st;
    if (!cache_ok(cache, false, scene->n_gaussians) || !workspace)
        return DGMR_ERR_BAD_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (scene->dtype == DGMR_F64)
        return vm_preprocess<double>(scene, camera, cache, workspace, workspace_bytes, stats, s);
    return vm_preprocess<float>(scene, camera, cache, workspace, workspace_bytes, stats, s);
}

dgmr_status dgmr_vm_forward_render_options(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_render_options* options,
    dgmr_vm_cache* cache, int64_t pair_capacity, void* workspace, size_t workspace_bytes, dgmr_frame_stats* stats, dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, -1);
    if (st != DGMR_OK)
        return st;
    if (!cache_ok(cache, pair_capacity > 0, scene->n_gaussians) || !workspace || pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff))
        return DGMR_ERR_BAD_ARG;
    if (options && options->render_mode != DGMR_RENDER_FULL && options->render_mode != DGMR_RENDER_BINS && options->render_mode != DGMR_RENDER_DEPTH)
        return DGMR_ERR_BAD_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (scene->dtype == DGMR_F64)
        return vm_render<double>(scene, camera, cache, pair_capacity, workspace, workspace_bytes, stats, s, options);
    return vm_render<float>(scene, camera, cache, pair_capacity, workspace, workspace_bytes, stats, s, options);
}

dgmr_status dgmr_vm_forward_render(const dgmr_scene* scene, const dgmr_camera* camera, dgmr_vm_cache* cache, int64_t pair_capacity, void* workspace,
    size_t workspace_bytes, dgmr_frame_stats* stats, dgmr_stream stream)
{
    return dgmr_vm_forward_render_options(scene, camera, nullptr, cache, pair_capacity, workspace, workspace_bytes, stats, stream);
}

dgmr_status dgmr_vm_backward(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_vm_cache* cache, const void* grad_framebuffer, void* grad_sh,
    void* grad_weights, void* grad_centroids, void* grad_scales, void* grad_rotations, void* workspace, size_t workspace_bytes, dgmr_frame_stats* stats,
    dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, -1);
    if (st != DGMR_OK)
        return st;
    const bool grads_ok = scene->n_gaussians == 0 || (grad_sh && grad_weights && grad_centroids && grad_scales && grad_rotations);
    if (!cache_ok(cache, false, scene->n_gaussians) || !workspace || !grad_framebuffer || !grads_ok)
        return DGMR_ERR_BAD_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (scene->dtype == DGMR_F64)
        return vm_backward<double>(scene, camera, cache, grad_framebuffer, grad_sh, grad_weights, grad_centroids, grad_scales, grad_rotations, workspace,
            workspace_bytes, stats, s);
    return vm_backward<float>(scene, camera, cache, grad_framebuffer, grad_sh, grad_weights, grad_centroids, grad_scales, grad_rotations, workspace,
        workspace_bytes, stats, s);
}

size_t dgmr_vm_step_store_size(int32_t width, int32_t height, int32_t store_steps, int32_t dtype)
{
    if (width <= 0 || height <= 0 || store_steps < 0 || store_steps > int32_t(kMaxLargeSteps))
        return 0;
    return step_store_bytes(uint32_t(width) * uint32_t(height), uint32_t(store_steps), dtype == DGMR_F64 ? sizeof(double) : sizeof(float));
}

dgmr_status dgmr_vm_forward_render_stored(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_render_options* options, dgmr_vm_cache* cache,
    int64_t pair_capacity, void* workspace, size_t workspace_bytes, void* step_store, size_t step_store_bytes_given, int32_t store_steps,
    dgmr_frame_stats* stats, dgmr_stream stream)
{
    dgmr_status st = check_scene(scene, camera, -1);
    if (st != DGMR_OK)
        return st;
    if (!cache_ok(cache, pair_capacity > 0, scene->n_gaussians) || !workspace || pair_capacity < 0 || pair_capacity > int64_t(0x7fffffff))
        return DGMR_ERR_BAD_ARG;
    if (options && options->render_mode != DGMR_RENDER_FULL && options->render_mode != DGMR_RENDER_BINS && options->render_mode != DGMR_RENDER_DEPTH)
        return DGMR_ERR_BAD_ARG;
    if (store_steps < 0 || (store_steps > 0 && !step_store))
        return DGMR_ERR_BAD_ARG;
    if (store_steps > 0 && step_store_bytes_given < dgmr_vm_step_store_size(camera->width, camera->height, store_steps, scene->dtype))
        return DGMR_ERR_WORKSPACE;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (scene->dtype == DGMR_F64)
        return vm_render<double>(scene, camera, cache, pair_capacity, workspace, workspace_bytes, stats, s, options, step_store, uint32_t(store_steps));
    return vm_render<float>(scene, camera, cache, pair_capacity, workspace, workspace_bytes, stats, s, options, step_store, uint32_t(store_steps));
}

dgmr_status dgmr_vm_backward_stored(const dgmr_scene* scene, const dgmr_camera* camera, const dgmr_vm_cache* cache, const void* grad_framebuffer,
    void* grad_sh, void* grad_weights, void* grad_centroids, void* grad_scales, void* grad_rotations, void* workspace, size_t workspace_bytes,
    const void* step_store, size_t step_store_bytes_given, int32_t store_steps, dgmr_frame_stats* stats, dgmr_stream stream)
{
    if (!scene || !camera || store_steps < 0 || (store_steps > 0 && !step_store))
        return DGMR_ERR_BAD_ARG;
    if (store_steps > 0 && step_store_bytes_given < dgmr_vm_step_store_size(camera->width, camera->height, store_steps, scene->dtype))
        return DGMR_ERR_WORKSPACE;
    dgmr_status st = check_scene(scene, camera, -1);
    if (st != DGMR_OK)
        return st;
    const bool grads_ok = scene->n_gaussians == 0 || (grad_sh && grad_weights && grad_centroids && grad_scales && grad_rotations);
    if (!cache_ok(cache, false, scene->n_gaussians) || !workspace || !grad_framebuffer || !grads_ok)
        return DGMR_ERR_BAD_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (scene->dtype == DGMR_F64)
        return vm_backward<double>(scene, camera, cache, grad_framebuffer, grad_sh, grad_weights, grad_centroids, grad_scales, grad_rotations, workspace,
            workspace_bytes, stats, s, step_store, uint32_t(store_steps));
    return vm_backward<float>(scene, camera, cache, grad_framebuffer, grad_sh, grad_weights, grad_centroids, grad_scales, grad_rotations, workspace,
        workspace_bytes, stats, s, step_store, uint32_t(store_steps));
}

dgmr_status dgmr_vm_batch_workspace_size(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, int64_t pair_capacity,
    size_t* frame_workspace_bytes, size_t* pair_workspace_bytes)
{
    if (!frame_workspace_bytes || !pair_workspace_bytes)
        return DGMR_ERR_BAD_ARG;
    static thread_local VmBatchPlan plan;
    const dgmr_status st = make_vm_batch(scenes, n_scenes, views, n_views, nullptr, pair_capacity, nullptr, nullptr, plan);
    if (st != DGMR_OK)
        return st;
    *frame_workspace_bytes = plan.L.bytes;
    *pair_workspace_bytes = plan.L.pair_bytes;
    return DGMR_OK;
}

dgmr_status dgmr_vm_batch_preprocess(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, void* frame_workspace,
    size_t frame_workspace_bytes, dgmr_frame_stats* stats, dgmr_stream stream)
{
    static thread_local VmBatchPlan plan;
    dgmr_status st = make_vm_batch(scenes, n_scenes, views, n_views, nullptr, 0, frame_workspace, nullptr, plan);
    if (st != DGMR_OK)
        return st;
    st = vm_batch_check_ws(plan, frame_workspace, frame_workspace_bytes, nullptr, 0, 0, false);
    if (st != DGMR_OK)
        return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : plan.L.stats;
    vm_batch_preprocess(plan, st_dev, s);
    if (plan.tab.G > 0) {
        k_pair_count<<<1, 1, 0, s>>>(plan.L.point_offsets, plan.tab.G, 0xffffffffu, st_dev, plan.L.bin.n_sort);
        note_launch();
    }
    return launch_status();
}

dgmr_status dgmr_vm_batch_forward(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views, void* frame_workspace,
    size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes, int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream)
{
    static thread_local VmBatchPlan plan;
    dgmr_status st = make_vm_batch(scenes, n_scenes, views, n_views, nullptr, pair_capacity, frame_workspace, pair_workspace, plan);
    if (st != DGMR_OK)
        return st;
    st = vm_batch_check_ws(plan, frame_workspace, frame_workspace_bytes, pair_workspace, pair_workspace_bytes, pair_capacity);
    if (st != DGMR_OK)
        return st;
    for (int v = 0; v < n_views; ++v)
        if (!views[v].framebuffer)
            return DGMR_ERR_BAD_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    VmBatchLayout& L = plan.L;
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    const uint32_t G = plan.tab.G, cap = uint32_t(pair_capacity), n_tiles = plan.tab.n_tiles;
    vm_batch_preprocess(plan, st_dev, s);
    const int par = run_binning_grids<float>(G, n_tiles, plan.tab.n_stiles, plan.tab, L.tiles_touched, L.point_offsets, L.rects, L.xy, cap, L.bin, L.ranges,
        st_dev, num_sms(), s, true);
    k_tile_order<<<1, 1024, 0, s>>>(L.ranges, n_tiles, L.tile_order);
    const VmMarch<float> a = vm_batch_march(L, L.bin.pair_val[par], st_dev);
    k_vm_march_warp<float, VmBatchFrames><<<n_tiles * (kTilePixels / kRayWarps), kRayWarps * 32, 0, s>>>(a, VmBatchFrames { plan.tab }, L.tile_order);
    note_launch(2);
    return launch_status();
}

dgmr_status dgmr_vm_batch_backward(const dgmr_scene* scenes, int32_t n_scenes, const dgmr_batch_view* views, int32_t n_views,
    const dgmr_scene_grads* grads, void* frame_workspace, size_t frame_workspace_bytes, void* pair_workspace, size_t pair_workspace_bytes,
    int64_t pair_capacity, dgmr_frame_stats* stats, dgmr_stream stream)
{
    if (!grads)
        return DGMR_ERR_BAD_ARG;
    static thread_local VmBatchPlan plan;
    dgmr_status st = make_vm_batch(scenes, n_scenes, views, n_views, grads, pair_capacity, frame_workspace, pair_workspace, plan);
    if (st != DGMR_OK)
        return st;
    st = vm_batch_check_ws(plan, frame_workspace, frame_workspace_bytes, pair_workspace, pair_workspace_bytes, pair_capacity);
    if (st != DGMR_OK)
        return st;
    for (int v = 0; v < n_views; ++v)
        if (!views[v].framebuffer)
            return DGMR_ERR_BAD_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    VmBatchLayout& L = plan.L;
    uint32_t* st_dev = stats ? reinterpret_cast<uint32_t*>(stats) : L.stats;
    const uint32_t G = plan.tab.G, n_tiles = plan.tab.n_tiles;
    const uint32_t n_scene_gaussians = plan.tab.scene_off[n_scenes];
    if (n_scene_gaussians == 0)
        return DGMR_OK;
    cudaMemsetAsync(L.acc, 0, size_t(G) * kVmAcc * sizeof(double), s);
    VmMarch<float> a = vm_batch_march(L, L.bin.pair_val[tile_sort_parity(plan.tab.n_stiles)], st_dev);
    a.acc = L.acc;
    k_vm_march_warp_bwd<float, VmBatchFrames><<<n_tiles * (kTilePixels / kRayWarps), kRayWarps * 32, 0, s>>>(a, VmBatchFrames { plan.tab }, L.tile_order);
    VmBwdGauss<float> state { 0, nullptr, nullptr, 1, 0, nullptr, nullptr, nullptr, L.clamped, reinterpret_cast<const int32_t*>(L.tiles_touched), L.acc,
        nullptr, nullptr, nullptr, nullptr, nullptr, 0.f, Formulation::Opacity };
    k_vm_batch_bwd_gaussians<<<(n_scene_gaussians + 127) / 128, 128, 0, s>>>(state, plan.tab);
    note_launch(2);
    return launch_status();
}

dgmr_status dgmr_vm_set_const_samples(int32_t n_sections, const double* sections)
{
    if (n_sections < 0 || n_sections > 4 || (n_sections > 0 && !sections))
        return DGMR_ERR_BAD_ARG;
    g_const_samples.n = n_sections;
    for (int i = 0; i < n_sections; ++i)
        for (int j = 0; j < 3; ++j)
            g_const_samples.s[i][j] = sections[3 * i + j];
    return DGMR_OK;
}

const char* dgmr_status_string(dgmr_status status)
{
    switch (status) {
    case DGMR_OK:
        return "ok";
    case DGMR_ERR_BAD_ARG:
        return "invalid argument";
    case DGMR_ERR_WORKSPACE:
        return "workspace too small";
    case DGMR_ERR_CUDA:
        return "CUDA launch error";
    case DGMR_ERR_STATIC_SCRATCH:
        return "frame exceeds the 64 MiB static scratch of the no-allocation entry point";
    case DGMR_ERR_PAIR_OVERFLOW:
        return "pair capacity too small for the frame (rendered incompletely)";
    }
    return "unknown status";
}

const char* dgmr_version(void) { return "dgmr_b200 0.1 sm_100a"; }

uint64_t dgmr_launch_count(void) { return launch_counter().load(); }

} // extern "C"
