// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the dgmr rendering path.
//
// Used by tests/ (parity checks), by bench.py's cpu_baseline / --impl
// reference legs (timed CPU path) and by __graft_entry__.smoke() (checker).
// The product never links or calls this library.
//
// Restates, on the CPU and in plain loops:
//   splat forward       src/dgmr/splat_forward.cu:30-338 (preprocess :70-118,
//                       scan :120-143, duplicateWithKeys :145-191, stable radix
//                       sort over bits [0, 32+msb) :193-211, identifyTileRanges
//                       :213-240, blend :242-335)
//   vol_marcher forward src/dgmr/vol_marcher_forward.cu:42-503
//   vol_marcher backward src/dgmr/vol_marcher_backward.cu:53-386
//   splat backward      no reference kernel; assembled from the projection
//                       adjoint grad/math.h:333-527, the SH adjoint
//                       grad/math.h:203-282 and a reverse-order adjoint of the
//                       blend at splat_forward.cu:299-321 (alpha = min(0.99, .)).
// Built with -ffp-contract=off so float results match the device kernels.
#include <algorithm>
#include <cstdlib>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#include <parallel/algorithm>
#endif

#include "dgmr_oracle_marching.h"
#include "dgmr_oracle_volume_fit.h"

using namespace orc;

namespace {

constexpr unsigned TILE = 16;
constexpr unsigned N_LARGE = 16; // vol_marcher.h:61
constexpr unsigned N_SMALL = 128; // vol_marcher.h:62
constexpr unsigned N_STEPS_PER_G = 32; // vol_marcher.h:63
constexpr float RELEVANCE_SIGMA = 3.f; // vol_marcher.h:65
constexpr float FILTER_SD = 0.55f; // vol_marcher.h:60
constexpr unsigned MAX_LARGE_STEPS = 4096; // guard: a march that makes no progress stops here

// Gradient-check mode (the reference's DGMR_TORCH_GRAD_CHECK_CONST_SAMPLES,
// vol_marcher_forward.cu:343-350): every large step puts these fixed sections
// instead of collecting them from the Gaussians, so sample positions do not
// move with the parameters.
struct ConstSamples {
    int n = 0;
    double s[4][3];
};
ConstSamples g_const_samples;

// The marcher's debug render mode (vol_marcher.h:48-56): 0 Full, 1 Bins, 2 Depth.
struct RenderMode {
    int mode = 0;
    int bin = -1;
    double max_depth = 20.0;
};
RenderMode g_render_mode;

// The formulation of the following calls (types.h:26-32): 0 = each renderer's
// reference default (splat and vol_raster Ots, vol_marcher Opacity), else 1 + value.
int g_formulation = 0;
inline Formulation form_or(Formulation renderer_default) { return g_formulation == 0 ? renderer_default : Formulation(g_formulation - 1); }

template <class T>
struct SceneIn {
    int N;
    const T* centroids;
    const T* sh;
    int sh_stride;
    int sh_degree;
    const T* weights;
    const T* scales;
    const T* rotations;
    const T* view;
    const T* proj;
    const T* campos;
    const T* bg;
    int W, H;
    T tan_fovx, tan_fovy;
    T cov_scale_multiplier;
};

template <class T>
inline V3<T> load3(const T* p, size_t i) { return { p[3 * i], p[3 * i + 1], p[3 * i + 2] }; }

template <class T>
void load_sh16(const SceneIn<T>& s, unsigned i, T pad, V3<T> out[16])
{
    for (int j = 0; j < 16; ++j)
        out[j] = sh_coef(s.sh, i, s.sh_stride, j, pad);
}

// ------------------------------------------------------------------ binning
// Keys are (tile << 32 | bits(float depth)), emitted per Gaussian in row-major
// rect order at the inclusive-scan offsets, then stably sorted.
struct Binning {
    std::vector<uint64_t> keys;
    std::vector<uint32_t> vals;
    std::vector<int32_t> ranges; // [T][2]
};

template <class T>
Binning bin_gaussians(int N, const int32_t* rects, const T* xy, const T* depths, const int32_t* tiles_touched, const int32_t* offsets, unsigned gx,
    unsigned gy)
{
    Binning b;
    const int64_t P = N > 0 ? offsets[N - 1] : 0;
    b.keys.resize(size_t(P));
    b.vals.resize(size_t(P));
    b.ranges.assign(size_t(gx) * gy * 2, 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        if (tiles_touched[i] == 0)
            continue;
        uint32_t off = (i == 0) ? 0 : uint32_t(offsets[i - 1]);
        const URect r = get_rect(float(xy[2 * i]), float(xy[2 * i + 1]), rects[2 * i], rects[2 * i + 1], gx, gy);
        const float df = float(depths[i]);
        uint32_t dbits;
        std::memcpy(&dbits, &df, 4);
        for (unsigned y = r.y0; y < r.y1; ++y)
            for (unsigned x = r.x0; x < r.x1; ++x) {
                b.keys[off] = (uint64_t(y * gx + x) << 32) | dbits;
                b.vals[off] = uint32_t(i);
                ++off;
            }
    }
    std::vector<uint32_t> order(static_cast<size_t>(P));
    for (int64_t k = 0; k < P; ++k)
        order[size_t(k)] = uint32_t(k);
    const auto less = [&](uint32_t a, uint32_t c) { return b.keys[a] < b.keys[c]; };
#ifdef _OPENMP
    __gnu_parallel::stable_sort(order.begin(), order.end(), less);
#else
    std::stable_sort(order.begin(), order.end(), less);
#endif
    std::vector<uint64_t> k2(static_cast<size_t>(P));
    std::vector<uint32_t> v2(static_cast<size_t>(P));
    for (int64_t k = 0; k < P; ++k) {
        k2[size_t(k)] = b.keys[order[size_t(k)]];
        v2[size_t(k)] = b.vals[order[size_t(k)]];
    }
    b.keys.swap(k2);
    b.vals.swap(v2);
    for (int64_t k = 0; k < P; ++k) {
        const uint32_t cur = uint32_t(b.keys[size_t(k)] >> 32);
        if (k == 0)
            b.ranges[2 * cur] = 0;
        else {
            const uint32_t prev = uint32_t(b.keys[size_t(k - 1)] >> 32);
            if (cur != prev) {
                b.ranges[2 * prev + 1] = int32_t(k);
                b.ranges[2 * cur] = int32_t(k);
            }
        }
        if (k == P - 1)
            b.ranges[2 * cur + 1] = int32_t(P);
    }
    return b;
}

void inclusive_scan(int N, const int32_t* in, int32_t* out)
{
    uint32_t acc = 0;
    for (int i = 0; i < N; ++i) {
        acc += uint32_t(in[i]);
        out[i] = int32_t(acc);
    }
}

// ------------------------------------------------------------- splat forward
struct SplatOut {
    float* fb; // [3,H,W]
    int32_t* rects; // [N,2]
    float* rgb; // [N,3]
    uint8_t* clamped; // [N,3]
    float* depths; // [N]
    float* xy; // [N,2]
    float* conic_opacity; // [N,4]
    int32_t* tiles_touched; // [N]
    int32_t* point_offsets; // [N]
    int32_t* i_ranges; // [T,2]
    float* final_T; // [H,W] (optional)
    int32_t* n_contrib; // [H,W] (optional)
};

template <class T>
void splat_preprocess(const SceneIn<T>& s, T* rgb, uint8_t* clamped, T* depths, T* xy, T* conic_opacity, int32_t* rects, int32_t* tiles_touched)
{
    const unsigned W = unsigned(s.W), H = unsigned(s.H);
    const unsigned gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    Camera<T> cam;
    cam.view = s.view;
    cam.proj = s.proj;
    cam.focal_y = T(float(H)) / (T(2.0f) * s.tan_fovy);
    cam.focal_x = T(float(W)) / (T(2.0f) * s.tan_fovx);
    cam.tan_fovx = s.tan_fovx;
    cam.tan_fovy = s.tan_fovy;
    cam.W = W;
    cam.H = H;
    const V3<T> campos = load3(s.campos, 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s.N; ++i) {
        tiles_touched[i] = 0;
        rects[2 * i] = rects[2 * i + 1] = 0;
        xy[2 * i] = xy[2 * i + 1] = T(0);
        depths[i] = T(0);
        for (int c = 0; c < 3; ++c) {
            rgb[3 * i + c] = T(0);
            clamped[3 * i + c] = 0;
        }
        for (int c = 0; c < 4; ++c)
            conic_opacity[4 * i + c] = T(0);
        const V3<T> mu = load3(s.centroids, size_t(i));
        if (mat4_mul_point(s.view, mu).z < T(0.2)) // splat_forward.cu:86
            continue;
        const T w = s.weights[i];
        const V3<T> sc = mul(load3(s.scales, size_t(i)), s.cov_scale_multiplier);
        const Gaussian2d<T> g = splat(form_or(Formulation::Ots), w, mu, sc, s.rotations + 4 * size_t(i), cam, T(0.3f));
        const int ex = ofm::to_int_rz(ofm::ceil_f(T(3.f) * ofm::sqrt_f(g.cov.v[0])));
        const int ey = ofm::to_int_rz(ofm::ceil_f(T(3.f) * ofm::sqrt_f(g.cov.v[2])));
        rects[2 * i] = ex;
        rects[2 * i + 1] = ey;
        const URect r = get_rect(float(g.centroid.x), float(g.centroid.y), ex, ey, gx, gy);
        const unsigned touched = (r.x1 - r.x0) * (r.y1 - r.y0);
        if (touched == 0)
            continue;
        tiles_touched[i] = int32_t(touched);
        xy[2 * i] = g.centroid.x;
        xy[2 * i + 1] = g.centroid.y;
        depths[i] = length(sub(campos, mu));
        const V3<T> v = sub(mu, campos);
        const V3<T> dir = mul(v, T(1) / ofm::sqrt_f(dot(v, v)));
        V3<T> sh16[16];
        load_sh16(s, unsigned(i), T(0), sh16);
        bool cl[3];
        const V3<T> col = sh_to_colour(sh16, s.sh_degree, dir, cl);
        rgb[3 * i] = col.x;
        rgb[3 * i + 1] = col.y;
        rgb[3 * i + 2] = col.z;
        for (int c = 0; c < 3; ++c)
            clamped[3 * i + c] = cl[c] ? 1 : 0;
        const S2<T> con = inverse2(g.cov);
        conic_opacity[4 * i] = con.v[0];
        conic_opacity[4 * i + 1] = con.v[1];
        conic_opacity[4 * i + 2] = con.v[2];
        conic_opacity[4 * i + 3] = g.weight;
    }
}

// alpha of one (pixel, splat) pair, splat_forward.cu:302-309.  The quadratic
// form d'Qd is evaluated as dx * (a dx + 2b dy) + (c dy) dy with two fused
// multiply-adds, in this order (the device blend uses the same sequence).
template <class T>
inline T splat_alpha(const T* co, const T* xy, T px, T py, T* g_out = nullptr, T* dx_out = nullptr, T* dy_out = nullptr)
{
    const T dx = px - xy[0];
    const T dy = py - xy[1];
    const T q = std::fma(std::fma(co[0], dx, (T(2) * co[1]) * dy), dx, (co[2] * dy) * dy);
    const T g = ofm::exp_f(T(-0.5f) * q);
    if (std::is_same<T, float>::value && audit().on.load(std::memory_order_relaxed)) {
        const T gl = std::exp(T(-0.5f) * q);
        const T al = min_f(T(0.99f), co[3] * g);
        audit_note(AUDIT_ALPHA, !(al < T(1.0f / 255.0f)), !(min_f(T(0.99f), co[3] * gl) < T(1.0f / 255.0f)), double(al), double(T(1.0f / 255.0f)));
    }
    if (g_out) {
        *g_out = g;
        *dx_out = dx;
        *dy_out = dy;
    }
    return min_f(T(0.99f), co[3] * g);
}

template <class T>
void splat_blend(const SceneIn<T>& s, const T* rgb, const T* xy, const T* conic_opacity, const int32_t* ranges, const uint32_t* list, T* fb, T* final_T,
    int32_t* n_contrib)
{
    const unsigned W = unsigned(s.W), H = unsigned(s.H);
    const unsigned gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    const V3<T> bg = load3(s.bg, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int tile = 0; tile < int(gx * gy); ++tile) {
        const unsigned tx = unsigned(tile) % gx, ty = unsigned(tile) / gx;
        const int32_t b = ranges[2 * tile], e = ranges[2 * tile + 1];
        for (unsigned ly = 0; ly < TILE; ++ly)
            for (unsigned lx = 0; lx < TILE; ++lx) {
                const unsigned px = tx * TILE + lx, py = ty * TILE + ly;
                if (px >= W || py >= H)
                    continue;
                T Tr = T(1);
                V3<T> C = { 0, 0, 0 };
                int32_t last = 0;
                for (int32_t k = b; k < e; ++k) {
                    const uint32_t id = list[k];
                    const T alpha = splat_alpha(conic_opacity + 4 * size_t(id), xy + 2 * size_t(id), T(float(px)), T(float(py)));
                    if (alpha < T(1.0f / 255.0f))
                        continue;
                    const T test_T = Tr * (T(1) - alpha);
                    if (test_T < T(0.0001f))
                        break;
                    // C += rgb * alpha * T, as one product and three fused multiply-adds
                    const T wgt = alpha * Tr;
                    C.x = std::fma(rgb[3 * id], wgt, C.x);
                    C.y = std::fma(rgb[3 * id + 1], wgt, C.y);
                    C.z = std::fma(rgb[3 * id + 2], wgt, C.z);
                    Tr = test_T;
                    last = k - b + 1;
                }
                const size_t pix = size_t(py) * W + px;
                fb[pix] = C.x + Tr * bg.x;
                fb[size_t(W) * H + pix] = C.y + Tr * bg.y;
                fb[2 * size_t(W) * H + pix] = C.z + Tr * bg.z;
                if (final_T)
                    final_T[pix] = Tr;
                if (n_contrib)
                    n_contrib[pix] = last;
            }
    }
}

// ------------------------------------------------------------- vol_marcher
template <class T>
struct VmCache {
    T* fb; // [3,H,W]
    int32_t* rects; // [N,2]
    T* rgb; // [N,3]
    uint8_t* clamped; // [N,3]
    T* depths; // [N]
    T* xy; // [N,2]
    T* inv_cov; // [N,6]
    T* masses; // [N]
    int32_t* tiles_touched; // [N]
    int32_t* point_offsets; // [N]
    int32_t* i_ranges; // [T,2]
    T* remaining_T; // [H,W]
};

template <class T>
T vm_aa_multiplier(const SceneIn<T>& s)
{
    return ((T(FILTER_SD) * s.tan_fovx) * T(2)) / T(float(unsigned(s.W)));
}

// vol_marcher_forward.cu:98-176
template <class T>
void vm_preprocess(const SceneIn<T>& s, VmCache<T>& c)
{
    const unsigned W = unsigned(s.W), H = unsigned(s.H);
    const unsigned gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    Camera<T> cam;
    cam.view = s.view;
    cam.proj = s.proj;
    cam.focal_y = T(float(H)) / (T(2.0f) * s.tan_fovy);
    cam.focal_x = T(float(W)) / (T(2.0f) * s.tan_fovx);
    cam.tan_fovx = s.tan_fovx;
    cam.tan_fovy = s.tan_fovy;
    cam.W = W;
    cam.H = H;
    const T aa = vm_aa_multiplier(s);
    const V3<T> campos = load3(s.campos, 0);
    const M3<T> W3 = mat3_of(s.view);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s.N; ++i) {
        c.tiles_touched[i] = 0;
        c.rects[2 * i] = c.rects[2 * i + 1] = 0;
        c.xy[2 * i] = c.xy[2 * i + 1] = T(0);
        c.depths[i] = T(0);
        c.masses[i] = T(0);
        for (int k = 0; k < 3; ++k) {
            c.rgb[3 * i + k] = T(0);
            c.clamped[3 * i + k] = 0;
        }
        for (int k = 0; k < 6; ++k)
            c.inv_cov[6 * i + k] = T(0);
        const V3<T> mu = load3(s.centroids, size_t(i));
        if (mat4_mul_point(s.view, mu).z < T(0.2f))
            continue;
        const T w = s.weights[i];
        const V3<T> sc = mul(load3(s.scales, size_t(i)), s.cov_scale_multiplier);
        const T* q = s.rotations + 4 * size_t(i);
        const T dist = length(sub(campos, mu));
        const S3<T> cov3 = compute_cov(sc, q);
        const T fks = dist * aa;
        const T fks2 = fks * fks;
        S3<T> filtered = cov3;
        filtered.v[0] = filtered.v[0] + fks2;
        filtered.v[3] = filtered.v[3] + fks2;
        filtered.v[5] = filtered.v[5] + fks2;
        const T mass = weight_to_mass(form_or(Formulation::Opacity), w, sc, affine_transform_and_cut(cov3, W3));
        if (mass <= T(0))
            continue;
        const Gaussian2d<T> g = splat(form_or(Formulation::Opacity), w, mu, sc, q, cam, T(FILTER_SD * FILTER_SD));
        const auto iso = [](T wt, T var, T isoline) {
            const T sv = T(-2) * ofm::log_f(isoline / wt);
            if (sv <= T(0))
                return T(0);
            return ofm::sqrt_f(sv * var);
        };
        const int ex = ofm::to_int_rz(ofm::ceil_f(iso(g.weight, g.cov.v[0], T(1.f / 255.f))));
        const int ey = ofm::to_int_rz(ofm::ceil_f(iso(g.weight, g.cov.v[2], T(1.f / 255.f))));
        if (std::is_same<T, float>::value && audit().on.load(std::memory_order_relaxed)) {
            const auto iso_l = [](T wt, T var, T isoline) {
                const T sv = T(-2) * std::log(isoline / wt);
                return sv <= T(0) ? T(0) : ofm::sqrt_f(sv * var);
            };
            const int exl = ofm::to_int_rz(ofm::ceil_f(iso_l(g.weight, g.cov.v[0], T(1.f / 255.f))));
            const int eyl = ofm::to_int_rz(ofm::ceil_f(iso_l(g.weight, g.cov.v[2], T(1.f / 255.f))));
            const T rx = iso(g.weight, g.cov.v[0], T(1.f / 255.f)), ry = iso(g.weight, g.cov.v[2], T(1.f / 255.f));
            audit_note(AUDIT_RECT, true, ex == exl, double(rx), std::round(double(rx)));
            audit_note(AUDIT_RECT, true, ey == eyl, double(ry), std::round(double(ry)));
        }
        c.rects[2 * i] = ex;
        c.rects[2 * i + 1] = ey;
        const URect r = get_rect(float(g.centroid.x), float(g.centroid.y), ex, ey, gx, gy);
        const unsigned touched = (r.x1 - r.x0) * (r.y1 - r.y0);
        if (touched == 0)
            continue;
        c.tiles_touched[i] = int32_t(touched);
        c.xy[2 * i] = g.centroid.x;
        c.xy[2 * i + 1] = g.centroid.y;
        const S3<T> inv = inverse_sym3(filtered);
        const T smax = max_f(sc.x, max_f(sc.y, sc.z));
        c.depths[i] = dist - (smax * T(RELEVANCE_SIGMA)) / T(2);
        const V3<T> dir = { (mu.x - campos.x) / dist, (mu.y - campos.y) / dist, (mu.z - campos.z) / dist };
        V3<T> sh16[16];
        load_sh16(s, unsigned(i), T(0), sh16);
        bool cl[3];
        const V3<T> col = sh_to_colour(sh16, s.sh_degree, dir, cl);
        c.rgb[3 * i] = col.x;
        c.rgb[3 * i + 1] = col.y;
        c.rgb[3 * i + 2] = col.z;
        for (int k = 0; k < 3; ++k)
            c.clamped[3 * i + k] = cl[k] ? 1 : 0;
        for (int k = 0; k < 6; ++k)
            c.inv_cov[6 * i + k] = inv.v[k];
        c.masses[i] = mass;
    }
}

// glm::inverse of a 4x4 (column-major), evaluated in double by cofactors
template <class T>
void inverse4(const T* m_in, T* out)
{
    double m[16], inv[16];
    for (int i = 0; i < 16; ++i)
        m[i] = double(m_in[i]);
    inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
    inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
    inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
    inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
    inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
    inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
    inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
    inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
    inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
    inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
    inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
    inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
    inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
    inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
    inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
    inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
    const double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
    for (int i = 0; i < 16; ++i)
        out[i] = T(inv[i] / det);
}

// Ray through the pixel centre: NDC z = 0 unprojected (vol_marcher_forward.cu:308-315)
template <class T>
Ray<T> pixel_ray(const T* inv_proj, V3<T> campos, unsigned px, unsigned py, unsigned W, unsigned H)
{
    const T pxc = T(px) + T(0.5);
    const T pyc = T(py) + T(0.5);
    const T nx = (pxc * T(2)) / T(float(W)) - T(1);
    const T ny = (pyc * T(2)) / T(float(H)) - T(1);
    V4<T> v = mat4_mul_vec4(inv_proj, V4<T> { nx, ny, T(0), T(1) });
    v.x = v.x / v.w;
    v.y = v.y / v.w;
    v.z = v.z / v.w;
    const V3<T> dvec = { v.x - campos.x, v.y - campos.y, v.z - campos.z };
    const T il = T(1) / ofm::sqrt_f(dot(dvec, dvec));
    Ray<T> r;
    r.o = campos;
    r.d = mul(dvec, il);
    return r;
}

// pass 1 of a large step: collect sample sections (vol_marcher_forward.cu:351-403)
template <class T>
void collect_sections(DensityArray<N_LARGE, T>& sections, const Ray<T>& ray, const int32_t* list, int32_t b, int32_t e, const T* centroids, const T* inv_cov,
    const T* masses, const T* depths)
{
    if (g_const_samples.n > 0) {
        for (int i = 0; i < g_const_samples.n; ++i)
            sections.put({ T(g_const_samples.s[i][0]), T(g_const_samples.s[i][1]), T(g_const_samples.s[i][2]) });
        return;
    }
    for (int32_t k = b; k < e; ++k) {
        const uint32_t id = uint32_t(list[k]);
        const V3<T> mu = load3(centroids, id);
        S3<T> Q;
        for (int j = 0; j < 6; ++j)
            Q.v[j] = inv_cov[6 * size_t(id) + j];
        const Gauss1d<T> g = intersect_with_ray_inv_C(mu, Q, ray);
        const T sd = ofm::sqrt_f(g.C);
        if (sections.end() < depths[id])
            break;
        const T mor = g.weight * masses[id];
        if (std::is_same<T, float>::value && audit().on.load(std::memory_order_relaxed)) {
            const T mor_l = intersect_weight_libm(mu, Q, ray) * masses[id];
            audit_note(AUDIT_SECTION_MASS, !(mor <= T(1.0f / 255.f) || mor > T(1000)), !(mor_l <= T(1.0f / 255.f) || mor_l > T(1000)), double(mor),
                double(T(1.0f / 255.f)));
        }
        if (mor <= T(1.0f / 255.f) || mor > T(1000))
            continue;
        if (g.C <= T(0))
            continue;
        if (ofm::isnan_f(g.centre))
            continue;
        const T start = g.centre - sd * T(RELEVANCE_SIGMA);
        const T end = g.centre + sd * T(RELEVANCE_SIGMA);
        const T delta_t = ((sd * T(RELEVANCE_SIGMA)) * T(2)) / T(float(N_STEPS_PER_G - 1));
        sections.put({ start, end, delta_t });
    }
}

template <class T>
void fill_bins(const Ray<T>& ray, const int32_t* list, int32_t b, int32_t e, const T* centroids, const T* inv_cov, const T* masses, const T* rgb,
    const T* borders, Bin4<T>* bins)
{
    for (int32_t k = b; k < e; ++k) {
        const uint32_t id = uint32_t(list[k]);
        S3<T> Q;
        for (int j = 0; j < 6; ++j)
            Q.v[j] = inv_cov[6 * size_t(id) + j];
        sample_gaussian<T, N_SMALL - 1>(masses[id], load3(rgb, id), load3(centroids, id), Q, ray, borders, bins);
    }
}

// the per-pixel march (vol_marcher_forward.cu:295-501)
template <class T>
void vm_march(const SceneIn<T>& s, const int32_t* list, VmCache<T>& c, int32_t* status)
{
    const unsigned W = unsigned(s.W), H = unsigned(s.H);
    const unsigned gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    T inv_proj[16];
    inverse4(s.proj, inv_proj);
    const V3<T> campos = load3(s.campos, 0);
    const V3<T> bg = load3(s.bg, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int tile = 0; tile < int(gx * gy); ++tile) {
        const unsigned tx = unsigned(tile) % gx, ty = unsigned(tile) / gx;
        const int32_t b = c.i_ranges[2 * tile], e = c.i_ranges[2 * tile + 1];
        std::vector<Bin4<T>> bins(N_SMALL - 1);
        for (unsigned ly = 0; ly < TILE; ++ly)
            for (unsigned lx = 0; lx < TILE; ++lx) {
                const unsigned px = tx * TILE + lx, py = ty * TILE + ly;
                if (px >= W || py >= H)
                    continue;
                const Ray<T> ray = pixel_ray(inv_proj, campos, px, py, W, H);
                T start = T(0);
                V3<T> colour = { 0, 0, 0 };
                T Tr = T(1);
                T distance = T(0);
                for (unsigned step = 0;; ++step) {
                    if (step >= MAX_LARGE_STEPS) {
#pragma omp atomic write
                        *status = 1;
                        break;
                    }
                    DensityArray<N_LARGE, T> sections(start);
                    collect_sections(sections, ray, list, b, e, s.centroids, c.inv_cov, c.masses, c.depths);
                    T borders[N_SMALL];
                    sample<N_SMALL>(sections, borders);
                    std::fill(bins.begin(), bins.end(), Bin4<T> { 0, 0, 0, 0 });
                    fill_bins(ray, list, b, e, s.centroids, c.inv_cov, c.masses, c.rgb, borders, bins.data());
                    if (g_render_mode.mode == 1) { // vol_marcher_forward.cu:453-465
                        const Bin4<T>& bk = bins[std::min(unsigned(g_render_mode.bin), N_SMALL - 2)];
                        const T mass = ((bk.r + bk.g) + bk.b) + bk.m;
                        const T md = T(g_render_mode.max_depth);
                        colour = { mass * md, mass * md, mass * md };
                        if (mass == T(0))
                            colour = { T(0), T(1), T(0) };
                        if (ofm::isnan_f(mass))
                            colour = { T(1), T(0), T(0.5) };
                        if (mass < T(0))
                            colour = { T(1), T(0), T(0) };
                        Tr = T(0);
                    } else if (g_render_mode.mode == 2) { // vol_marcher_forward.cu:466-481
                        for (unsigned k = 0; k < N_SMALL - 1; ++k)
                            Tr = Tr * ofm::exp_f(-bins[k].m);
                        distance = max_f(sections.end(), distance);
                        const T dd = distance / T(g_render_mode.max_depth);
                        colour = { dd, dd, dd };
                    } else {
                        integrate_bins<T, N_SMALL - 1>(colour, Tr, bins.data());
                    }
                    if (sections.size() == 0 || Tr < T(1.f / 255.f))
                        break;
                    start = borders[N_SMALL - 1];
                }
                const size_t pix = size_t(py) * W + px;
                c.fb[pix] = colour.x + Tr * bg.x;
                c.fb[size_t(W) * H + pix] = colour.y + Tr * bg.y;
                c.fb[2 * size_t(W) * H + pix] = colour.z + Tr * bg.z;
                c.remaining_T[pix] = Tr;
            }
    }
}

// ---------------------------------------------------------- vol_marcher bwd
template <class T>
struct VmGrads {
    T* sh; // [N, sh_stride, 3]
    T* weights; // [N]
    T* centroids; // [N,3]
    T* scales; // [N,3]
    T* rotations; // [N,4]
};

// adjoint of a symmetric 3x3 inverse: packed grad of M = P^-1 -> packed grad of P
template <class T>
S3<T> grad_inverse_sym3(const S3<T>& P, const S3<T>& g_M)
{
    const S3<T> M = inverse_sym3(P);
    T Mf[3][3], Gf[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            Mf[i][j] = sym3(M, i, j);
            Gf[i][j] = (i == j) ? sym3(g_M, i, j) : sym3(g_M, i, j) / T(2);
        }
    T MG[3][3], H[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            MG[i][j] = (Mf[i][0] * Gf[0][j] + Mf[i][1] * Gf[1][j]) + Mf[i][2] * Gf[2][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            H[i][j] = -((MG[i][0] * Mf[0][j] + MG[i][1] * Mf[1][j]) + MG[i][2] * Mf[2][j]);
    S3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j)
            r.v[sym3_idx<T>(i, j)] = (i == j) ? H[i][j] : T(2) * H[i][j];
    return r;
}

// adjoint of cut(A S A^T) w.r.t. S (packed) and A (full, rows 0-1)
template <class T>
void grad_affine_transform_and_cut(const S3<T>& S, const M3<T>& A, const S2<T>& g, S3<T>* g_S, M3<T>* g_A)
{
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            const int p = sym3_idx<T>(i, j);
            T v;
            if (i == j)
                v = g.v[0] * A.m[0][i] * A.m[0][i] + g.v[1] * A.m[0][i] * A.m[1][i] + g.v[2] * A.m[1][i] * A.m[1][i];
            else
                v = g.v[0] * T(2) * A.m[0][i] * A.m[0][j] + g.v[1] * (A.m[0][i] * A.m[1][j] + A.m[0][j] * A.m[1][i])
                    + g.v[2] * T(2) * A.m[1][i] * A.m[1][j];
            g_S->v[p] = g_S->v[p] + v;
        }
    if (g_A) {
        // c00 = a0 S a0^T, c01 = a0 S a1^T, c11 = a1 S a1^T
        T Sa0[3], Sa1[3];
        for (int i = 0; i < 3; ++i) {
            Sa0[i] = (sym3(S, i, 0) * A.m[0][0] + sym3(S, i, 1) * A.m[0][1]) + sym3(S, i, 2) * A.m[0][2];
            Sa1[i] = (sym3(S, i, 0) * A.m[1][0] + sym3(S, i, 1) * A.m[1][1]) + sym3(S, i, 2) * A.m[1][2];
        }
        for (int k = 0; k < 3; ++k) {
            g_A->m[0][k] = g_A->m[0][k] + g.v[0] * T(2) * Sa0[k] + g.v[1] * Sa1[k];
            g_A->m[1][k] = g_A->m[1][k] + g.v[1] * Sa0[k] + g.v[2] * T(2) * Sa1[k];
        }
    }
}

// adjoint of compute_cov w.r.t. scales and the (w,x,y,z) quaternion
template <class T>
void grad_compute_cov(V3<T> s, const T* q, const S3<T>& g, V3<T>* g_s, T* g_q)
{
    const M3<T> R = quat_to_mat3<T>(q);
    M3<T> M;
    for (int r = 0; r < 3; ++r) {
        M.m[r][0] = R.m[r][0] * s.x;
        M.m[r][1] = R.m[r][1] * s.y;
        M.m[r][2] = R.m[r][2] * s.z;
    }
    T G[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            G[i][j] = (i == j) ? sym3(g, i, j) : sym3(g, i, j) / T(2);
    // dL/dM = 2 G M
    T gM[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            gM[i][j] = T(2) * ((G[i][0] * M.m[0][j] + G[i][1] * M.m[1][j]) + G[i][2] * M.m[2][j]);
    T gR[3][3];
    const T sv[3] = { s.x, s.y, s.z };
    T gs[3] = { 0, 0, 0 };
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            gR[r][c] = gM[r][c] * sv[c];
            gs[c] = gs[c] + gM[r][c] * R.m[r][c];
        }
    g_s->x = g_s->x + gs[0];
    g_s->y = g_s->y + gs[1];
    g_s->z = g_s->z + gs[2];
    const T w = q[0], x = q[1], y = q[2], z = q[3];
    T gw = 0, gx = 0, gy = 0, gz = 0;
    // R00 = 1-2(yy+zz)
    gy += gR[0][0] * (T(-4) * y);
    gz += gR[0][0] * (T(-4) * z);
    // R10 = 2(xy+wz)
    gw += gR[1][0] * (T(2) * z);
    gx += gR[1][0] * (T(2) * y);
    gy += gR[1][0] * (T(2) * x);
    gz += gR[1][0] * (T(2) * w);
    // R20 = 2(xz-wy)
    gw += gR[2][0] * (T(-2) * y);
    gx += gR[2][0] * (T(2) * z);
    gy += gR[2][0] * (T(-2) * w);
    gz += gR[2][0] * (T(2) * x);
    // R01 = 2(xy-wz)
    gw += gR[0][1] * (T(-2) * z);
    gx += gR[0][1] * (T(2) * y);
    gy += gR[0][1] * (T(2) * x);
    gz += gR[0][1] * (T(-2) * w);
    // R11 = 1-2(xx+zz)
    gx += gR[1][1] * (T(-4) * x);
    gz += gR[1][1] * (T(-4) * z);
    // R21 = 2(yz+wx)
    gw += gR[2][1] * (T(2) * x);
    gx += gR[2][1] * (T(2) * w);
    gy += gR[2][1] * (T(2) * z);
    gz += gR[2][1] * (T(2) * y);
    // R02 = 2(xz+wy)
    gw += gR[0][2] * (T(2) * y);
    gx += gR[0][2] * (T(2) * z);
    gy += gR[0][2] * (T(2) * w);
    gz += gR[0][2] * (T(2) * x);
    // R12 = 2(yz-wx)
    gw += gR[1][2] * (T(-2) * x);
    gx += gR[1][2] * (T(-2) * w);
    gy += gR[1][2] * (T(2) * z);
    gz += gR[1][2] * (T(2) * y);
    // R22 = 1-2(xx+yy)
    gx += gR[2][2] * (T(-4) * x);
    gy += gR[2][2] * (T(-4) * y);
    g_q[0] += gw;
    g_q[1] += gx;
    g_q[2] += gy;
    g_q[3] += gz;
}

template <class T>
void vm_backward_impl(const SceneIn<T>& s, const VmCache<T>& c, const int32_t* list, const T* grad_fb, VmGrads<T>& out, int32_t* status)
{
    const unsigned W = unsigned(s.W), H = unsigned(s.H);
    const unsigned gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    const int N = s.N;
    T inv_proj[16];
    inverse4(s.proj, inv_proj);
    const V3<T> campos = load3(s.campos, 0);
    const V3<T> bg = load3(s.bg, 0);

    // per-Gaussian accumulators: mass, rgb[3], centroid[3], inv_cov[6]; summed in double
    int n_threads = 1;
#ifdef _OPENMP
    n_threads = omp_get_max_threads();
#endif
    std::vector<double> acc(size_t(n_threads) * size_t(N) * 13, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int tile = 0; tile < int(gx * gy); ++tile) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* my = acc.data() + size_t(tid) * size_t(N) * 13;
        const unsigned tx = unsigned(tile) % gx, ty = unsigned(tile) / gx;
        const int32_t b = c.i_ranges[2 * tile], e = c.i_ranges[2 * tile + 1];
        std::vector<Bin4<T>> bins(N_SMALL - 1), gbins(N_SMALL - 1);
        for (unsigned ly = 0; ly < TILE; ++ly)
            for (unsigned lx = 0; lx < TILE; ++lx) {
                const unsigned px = tx * TILE + lx, py = ty * TILE + ly;
                if (px >= W || py >= H)
                    continue;
                const size_t pix = size_t(py) * W + px;
                const Ray<T> ray = pixel_ray(inv_proj, campos, px, py, W, H);
                const T final_T = c.remaining_T[pix];
                const V3<T> final_colour = { c.fb[pix], c.fb[size_t(W) * H + pix], c.fb[2 * size_t(W) * H + pix] };
                V3<T> colour = { final_colour.x - final_T * bg.x, final_colour.y - final_T * bg.y, final_colour.z - final_T * bg.z };
                const V3<T> g_colour = { grad_fb[pix], grad_fb[size_t(W) * H + pix], grad_fb[2 * size_t(W) * H + pix] };
                const T g_T = dot(g_colour, bg);
                T start = T(0);
                T Tr = T(1);
                for (unsigned step = 0;; ++step) {
                    if (step >= MAX_LARGE_STEPS) {
#pragma omp atomic write
                        *status = 1;
                        break;
                    }
                    DensityArray<N_LARGE, T> sections(start);
                    collect_sections(sections, ray, list, b, e, s.centroids, c.inv_cov, c.masses, c.depths);
                    T borders[N_SMALL];
                    sample<N_SMALL>(sections, borders);
                    std::fill(bins.begin(), bins.end(), Bin4<T> { 0, 0, 0, 0 });
                    fill_bins(ray, list, b, e, s.centroids, c.inv_cov, c.masses, c.rgb, borders, bins.data());
                    grad_integrate_bins<T, N_SMALL - 1>(colour, Tr, final_T, bins.data(), g_colour, g_T, gbins.data());
                    for (int32_t k = b; k < e; ++k) {
                        const uint32_t id = uint32_t(list[k]);
                        S3<T> Q;
                        for (int j = 0; j < 6; ++j)
                            Q.v[j] = c.inv_cov[6 * size_t(id) + j];
                        T gm = 0;
                        V3<T> grgb = { 0, 0, 0 }, gpos = { 0, 0, 0 };
                        S3<T> gQ = { { 0, 0, 0, 0, 0, 0 } };
                        grad_sample_gaussian<T, N_SMALL - 1>(c.masses[id], load3(c.rgb, id), load3(s.centroids, id), Q, ray, borders, gbins.data(), &gm, &grgb,
                            &gpos, &gQ);
                        double* a = my + size_t(id) * 13;
                        a[0] += double(gm);
                        a[1] += double(grgb.x);
                        a[2] += double(grgb.y);
                        a[3] += double(grgb.z);
                        a[4] += double(gpos.x);
                        a[5] += double(gpos.y);
                        a[6] += double(gpos.z);
                        for (int j = 0; j < 6; ++j)
                            a[7 + j] += double(gQ.v[j]);
                    }
                    if (sections.size() == 0 || Tr < T(1.f / 255.f))
                        break;
                    start = borders[N_SMALL - 1];
                }
            }
    }
    std::vector<double> tot(size_t(N) * 13, 0.0);
    for (int t = 0; t < n_threads; ++t)
        for (size_t k = 0; k < tot.size(); ++k)
            tot[k] += acc[size_t(t) * size_t(N) * 13 + k];

    // per-Gaussian chain rule (vol_marcher_backward.cu:321-384)
    const T aa = vm_aa_multiplier(s);
    const M3<T> W3 = mat3_of(s.view);
    for (int i = 0; i < N; ++i) {
        for (int k = 0; k < s.sh_stride * 3; ++k)
            out.sh[size_t(i) * s.sh_stride * 3 + k] = T(0);
        out.weights[i] = T(0);
        for (int k = 0; k < 3; ++k) {
            out.centroids[3 * i + k] = T(tot[size_t(i) * 13 + 4 + k]);
            out.scales[3 * i + k] = T(0);
        }
        for (int k = 0; k < 4; ++k)
            out.rotations[4 * i + k] = T(0);
        if (c.tiles_touched[i] == 0)
            continue;
        const V3<T> mu = load3(s.centroids, size_t(i));
        if (mat4_mul_point(s.view, mu).z < T(0.2))
            continue;
        const T w = s.weights[i];
        const V3<T> sc = load3(s.scales, size_t(i)); // the reference does not apply cov_scale_multiplier here
        const T* q = s.rotations + 4 * size_t(i);
        const V3<T> delta = sub(mu, campos);
        const T dist = length(delta);
        const S3<T> cov3 = compute_cov(sc, q);
        const T fks = dist * aa;
        S3<T> filtered = cov3;
        filtered.v[0] = filtered.v[0] + fks * fks;
        filtered.v[3] = filtered.v[3] + fks * fks;
        filtered.v[5] = filtered.v[5] + fks * fks;
        const S2<T> cov2d = affine_transform_and_cut(cov3, W3);
        const T mass = weight_to_mass(form_or(Formulation::Opacity), w, sc, cov2d);
        if (mass <= T(0))
            continue;
        const V3<T> dir = { delta.x / dist, delta.y / dist, delta.z / dist };
        V3<T> sh16[16];
        load_sh16(s, unsigned(i), T(1), sh16);
        const V3<T> g_rgb = { T(tot[size_t(i) * 13 + 1]), T(tot[size_t(i) * 13 + 2]), T(tot[size_t(i) * 13 + 3]) };
        const bool cl[3] = { c.clamped[3 * i] != 0, c.clamped[3 * i + 1] != 0, c.clamped[3 * i + 2] != 0 };
        V3<T> g_sh16[16];
        const V3<T> g_dir = grad_sh_to_colour(sh16, s.sh_degree, dir, g_rgb, cl, g_sh16);
        for (int j = 0; j < s.sh_stride && j < 16; ++j) {
            out.sh[(size_t(i) * s.sh_stride + j) * 3] = g_sh16[j].x;
            out.sh[(size_t(i) * s.sh_stride + j) * 3 + 1] = g_sh16[j].y;
            out.sh[(size_t(i) * s.sh_stride + j) * 3 + 2] = g_sh16[j].z;
        }
        // direction = delta / dist
        V3<T> g_mu = mul(g_dir, T(1) / dist);
        T g_dist = -dot(g_dir, delta) / (dist * dist);
        S3<T> g_invcov;
        for (int j = 0; j < 6; ++j)
            g_invcov.v[j] = T(tot[size_t(i) * 13 + 7 + j]);
        const S3<T> g_filtered = grad_inverse_sym3(filtered, g_invcov);
        const T g_mass = T(tot[size_t(i) * 13]);
        // adjoint of weight_to_mass (math.h:298-320)
        const Formulation f = form_or(Formulation::Opacity);
        T g_w = T(0);
        S2<T> g_cov2d = { { 0, 0, 0 } };
        V3<T> g_s = { 0, 0, 0 };
        if (f == Formulation::Opacity) { // mass = w * 2 pi sqrt(det cov2d)
            const T dcov = det2(cov2d);
            const T i2 = integrate_exponential_cov2(cov2d);
            g_w = g_mass * i2;
            const T g_i2 = g_mass * w;
            const T g_det = (dcov > T(0)) ? g_i2 * two_pi<T>() / (T(2) * ofm::sqrt_f(dcov)) : T(0);
            g_cov2d = { { g_det * cov2d.v[2], g_det * T(-2) * cov2d.v[1], g_det * cov2d.v[0] } };
        } else if (f == Formulation::Mass) {
            g_w = g_mass;
        } else if (f == Formulation::Density) {
            g_w = g_mass * integrate_exponential3(sc);
            const T k = (g_mass * w) * two_pi_pow_1_5<T>();
            g_s = { k * sc.y * sc.z, k * sc.x * sc.z, k * sc.x * sc.y };
        } else {
            const V2<T> l2 = f == Formulation::Ots ? larger2(sc) : smaller2(sc);
            g_w = g_mass * integrate_exponential2(l2);
            const T k = (g_mass * w) * two_pi<T>();
            const V2<T> g_l2 = { k * l2.y, k * l2.x };
            g_s = f == Formulation::Ots ? grad_larger2(sc, g_l2) : grad_smaller2(sc, g_l2);
        }
        S3<T> g_cov3 = g_filtered;
        const T g_fks2 = (g_filtered.v[0] + g_filtered.v[3]) + g_filtered.v[5];
        g_dist = g_dist + (g_fks2 * T(2) * fks) * aa;
        grad_affine_transform_and_cut(cov3, W3, g_cov2d, &g_cov3, static_cast<M3<T>*>(nullptr));
        T g_q[4] = { 0, 0, 0, 0 };
        grad_compute_cov(sc, q, g_cov3, &g_s, g_q);
        g_mu = add(g_mu, mul(delta, g_dist / dist));
        out.weights[i] = g_w;
        for (int k = 0; k < 3; ++k)
            out.scales[3 * i + k] = g_s[k];
        for (int k = 0; k < 4; ++k)
            out.rotations[4 * i + k] = g_q[k];
        out.centroids[3 * i] += g_mu.x;
        out.centroids[3 * i + 1] += g_mu.y;
        out.centroids[3 * i + 2] += g_mu.z;
    }
}

// --------------------------------------------------------------- splat bwd
// Adjoint of splat (grad/math.h:333-527 restated, with the derivative of the
// fov clamp limits w.r.t. t.z included) for one Gaussian, every formulation.
template <class T>
void grad_splat(Formulation f, T weight, V3<T> mu, V3<T> s, const T* q, const Camera<T>& cam, T filter, T g_w2, V2<T> g_xy, S2<T> g_cov, T* g_weight,
    V3<T>* g_mu, V3<T>* g_s, T* g_q)
{
    const V4<T> tu4 = mat4_mul_point(cam.view, mu);
    const T lim_x = (T(1.3) * cam.tan_fovx) * tu4.z;
    const T lim_y = (T(1.3) * cam.tan_fovy) * tu4.z;
    const V3<T> t = { clamp_f(tu4.x, -lim_x, lim_x), clamp_f(tu4.y, -lim_y, lim_y), tu4.z };
    const T l = length(t);
    const M3<T> SJ = make_jakobian(t, l, cam.focal_x, cam.focal_y);
    const M3<T> W = mat3_of(cam.view);
    const M3<T> Tm = matmul(SJ, W);
    const S3<T> cov3 = compute_cov(s, q);
    const S2<T> c = affine_transform_and_cut(cov3, Tm);
    S2<T> cov2 = c;
    cov2.v[0] = cov2.v[0] + filter;
    cov2.v[2] = cov2.v[2] + filter;
    const T detSJ = det3(SJ);
    T g_detSJ = T(0);
    if (f == Formulation::Opacity) {
        // weight2d = w sqrt(max(eps, det c / det(c + filter)))
        const T dcv = det2(c), dn = det2(cov2);
        const T r = dcv / dn;
        const T factor = ofm::sqrt_f(max_f(T(0.000025), r));
        *g_weight = *g_weight + g_w2 * factor;
        if (T(0.000025) < r) {
            const T g_r = (g_w2 * weight) / (T(2) * factor);
            const T g_dc = g_r / dn;
            const T g_dn = -g_r * dcv / (dn * dn);
            g_cov.v[0] = (g_cov.v[0] + g_dc * c.v[2]) + g_dn * cov2.v[2];
            g_cov.v[1] = (g_cov.v[1] - g_dc * T(2) * c.v[1]) - g_dn * T(2) * cov2.v[1];
            g_cov.v[2] = (g_cov.v[2] + g_dc * c.v[0]) + g_dn * cov2.v[0];
        }
    } else {
        // weight2d = w detSJ A(s) / i2(cov2)
        T A = T(1);
        if (f == Formulation::Density)
            A = integrate_exponential3(s);
        else if (f == Formulation::Ots)
            A = integrate_exponential2(larger2(s));
        else if (f == Formulation::Ols)
            A = integrate_exponential2(smaller2(s));
        const T dc = det2(cov2);
        const T i2 = integrate_exponential_cov2(cov2);
        *g_weight = *g_weight + g_w2 * detSJ * A / i2;
        g_detSJ = g_w2 * weight * A / i2;
        const T g_A = g_w2 * weight * detSJ / i2;
        const T g_i2 = -g_w2 * weight * detSJ * A / (i2 * i2);
        const T g_dc = (dc > T(0)) ? g_i2 * two_pi<T>() / (T(2) * ofm::sqrt_f(dc)) : T(0);
        g_cov.v[0] = g_cov.v[0] + g_dc * cov2.v[2];
        g_cov.v[1] = g_cov.v[1] - g_dc * T(2) * cov2.v[1];
        g_cov.v[2] = g_cov.v[2] + g_dc * cov2.v[0];
        if (f == Formulation::Density) {
            const T k = g_A * two_pi_pow_1_5<T>();
            *g_s = add(*g_s, V3<T> { k * s.y * s.z, k * s.x * s.z, k * s.x * s.y });
        } else if (f == Formulation::Ots || f == Formulation::Ols) {
            const V2<T> l2 = f == Formulation::Ots ? larger2(s) : smaller2(s);
            const V2<T> g_l2 = { g_A * two_pi<T>() * l2.y, g_A * two_pi<T>() * l2.x };
            *g_s = add(*g_s, f == Formulation::Ots ? grad_larger2(s, g_l2) : grad_smaller2(s, g_l2));
        }
    }
    M3<T> g_SJ = cofactor3(SJ);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            g_SJ.m[i][j] = g_SJ.m[i][j] * g_detSJ;
    S3<T> g_cov3 = { { 0, 0, 0, 0, 0, 0 } };
    M3<T> g_Tm = { { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } } };
    grad_affine_transform_and_cut(cov3, Tm, g_cov, &g_cov3, &g_Tm);
    // Tm = SJ W -> g_SJ += g_Tm W^T
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            g_SJ.m[i][j] = g_SJ.m[i][j] + (g_Tm.m[i][0] * W.m[j][0] + g_Tm.m[i][1] * W.m[j][1]) + g_Tm.m[i][2] * W.m[j][2];
    const T fx = cam.focal_x, fy = cam.focal_y;
    const T tz2 = t.z * t.z, tz3 = tz2 * t.z;
    V3<T> g_t;
    g_t.x = g_SJ.m[0][2] * (-fx / tz2) + g_SJ.m[2][0] / l;
    g_t.y = g_SJ.m[1][2] * (-fy / tz2) + g_SJ.m[2][1] / l;
    g_t.z = g_SJ.m[0][0] * (-fx / tz2) + g_SJ.m[1][1] * (-fy / tz2) + g_SJ.m[0][2] * (T(2) * fx * t.x / tz3) + g_SJ.m[1][2] * (T(2) * fy * t.y / tz3)
        + g_SJ.m[2][2] / l;
    const T g_l = -(g_SJ.m[2][0] * t.x + g_SJ.m[2][1] * t.y + g_SJ.m[2][2] * t.z) / (l * l);
    g_t = add(g_t, mul(t, g_l / l));
    // clamp: t.x = clamp(tu.x, -lim(tz), lim(tz))
    V3<T> g_tu = { 0, 0, g_t.z };
    if (tu4.x < -lim_x) {
        g_tu.z = g_tu.z - g_t.x * (T(1.3) * cam.tan_fovx);
    } else if (tu4.x > lim_x) {
        g_tu.z = g_tu.z + g_t.x * (T(1.3) * cam.tan_fovx);
    } else {
        g_tu.x = g_t.x;
    }
    if (tu4.y < -lim_y) {
        g_tu.z = g_tu.z - g_t.y * (T(1.3) * cam.tan_fovy);
    } else if (tu4.y > lim_y) {
        g_tu.z = g_tu.z + g_t.y * (T(1.3) * cam.tan_fovy);
    } else {
        g_tu.y = g_t.y;
    }
    V3<T> gm = { 0, 0, 0 };
    for (int c = 0; c < 3; ++c)
        gm[c] = (W.m[0][c] * g_tu.x + W.m[1][c] * g_tu.y) + W.m[2][c] * g_tu.z;
    // screen centroid via the projection
    const V4<T> pp = mat4_mul_point(cam.proj, mu);
    const T d = pp.w + T(0.0000001);
    const T g_px = g_xy.x * T(0.5) * T(int(cam.W));
    const T g_py = g_xy.y * T(0.5) * T(int(cam.H));
    const T g_ppx = g_px / d, g_ppy = g_py / d;
    const T g_ppw = -(g_px * pp.x + g_py * pp.y) / (d * d);
    for (int c = 0; c < 3; ++c)
        gm[c] = gm[c] + (cam.proj[c * 4 + 0] * g_ppx + cam.proj[c * 4 + 1] * g_ppy) + cam.proj[c * 4 + 3] * g_ppw;
    *g_mu = add(*g_mu, gm);
    grad_compute_cov(s, q, g_cov3, g_s, g_q);
}

template <class T>
struct SplatGrads {
    T* sh; // [N, sh_stride, 3]
    T* weights; // [N]
    T* centroids; // [N,3]
    T* scales; // [N,3]
    T* rotations; // [N,4]
};

template <class T>
void splat_backward_impl(const SceneIn<T>& s, const T* rgb, const uint8_t* clamped, const T* xy, const T* conic_opacity, const int32_t* tiles_touched,
    const int32_t* ranges, const uint32_t* list, const T* final_T, const int32_t* n_contrib, const T* grad_fb, SplatGrads<T>& out)
{
    const unsigned W = unsigned(s.W), H = unsigned(s.H);
    const unsigned gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    const int N = s.N;
    const V3<T> bg = load3(s.bg, 0);
    int n_threads = 1;
#ifdef _OPENMP
    n_threads = omp_get_max_threads();
#endif
    // xy[2], conic[3], opacity, rgb[3]
    std::vector<double> acc(size_t(n_threads) * size_t(N) * 9, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int tile = 0; tile < int(gx * gy); ++tile) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* my = acc.data() + size_t(tid) * size_t(N) * 9;
        const unsigned tx = unsigned(tile) % gx, ty = unsigned(tile) / gx;
        const int32_t b = ranges[2 * tile];
        for (unsigned ly = 0; ly < TILE; ++ly)
            for (unsigned lx = 0; lx < TILE; ++lx) {
                const unsigned px = tx * TILE + lx, py = ty * TILE + ly;
                if (px >= W || py >= H)
                    continue;
                const size_t pix = size_t(py) * W + px;
                const V3<T> gout = { grad_fb[pix], grad_fb[size_t(W) * H + pix], grad_fb[2 * size_t(W) * H + pix] };
                const T Tf = final_T[pix];
                T Tr = Tf;
                V3<T> accum = { 0, 0, 0 };
                const T bg_dot = dot(bg, gout);
                for (int32_t k = b + n_contrib[pix] - 1; k >= b; --k) {
                    const uint32_t id = list[k];
                    const T* co = conic_opacity + 4 * size_t(id);
                    T g, dx, dy;
                    const T alpha = splat_alpha(co, xy + 2 * size_t(id), T(float(px)), T(float(py)), &g, &dx, &dy);
                    if (alpha < T(1.0f / 255.0f))
                        continue;
                    // T before this splat, and the background term's 1 / (1 - alpha): one reciprocal
                    const T inv = T(1) / (T(1) - alpha);
                    Tr = Tr * inv;
                    const V3<T> c = load3(rgb, id);
                    double* a = my + size_t(id) * 9;
                    a[6] += double(alpha * Tr * gout.x);
                    a[7] += double(alpha * Tr * gout.y);
                    a[8] += double(alpha * Tr * gout.z);
                    const T g_alpha = Tr * ((c.x - accum.x) * gout.x + (c.y - accum.y) * gout.y + (c.z - accum.z) * gout.z) - (Tf * bg_dot) * inv;
                    accum = { alpha * c.x + (T(1) - alpha) * accum.x, alpha * c.y + (T(1) - alpha) * accum.y, alpha * c.z + (T(1) - alpha) * accum.z };
                    const T og = co[3] * g;
                    if (!(og < T(0.99f)))
                        continue; // alpha clamped at 0.99: no gradient
                    a[5] += double(g_alpha * g);
                    const T g_g = g_alpha * co[3];
                    const T g_q = T(-0.5) * g * g_g;
                    a[2] += double(g_q * dx * dx);
                    a[3] += double(g_q * T(2) * dx * dy);
                    a[4] += double(g_q * dy * dy);
                    // d = pix - xy
                    a[0] -= double(g_q * (T(2) * co[0] * dx + T(2) * co[1] * dy));
                    a[1] -= double(g_q * (T(2) * co[2] * dy + T(2) * co[1] * dx));
                }
            }
    }
    std::vector<double> tot(size_t(N) * 9, 0.0);
    for (int t = 0; t < n_threads; ++t)
        for (size_t k = 0; k < tot.size(); ++k)
            tot[k] += acc[size_t(t) * size_t(N) * 9 + k];

    Camera<T> cam;
    cam.view = s.view;
    cam.proj = s.proj;
    cam.focal_y = T(float(H)) / (T(2.0f) * s.tan_fovy);
    cam.focal_x = T(float(W)) / (T(2.0f) * s.tan_fovx);
    cam.tan_fovx = s.tan_fovx;
    cam.tan_fovy = s.tan_fovy;
    cam.W = W;
    cam.H = H;
    const V3<T> campos = load3(s.campos, 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        for (int k = 0; k < s.sh_stride * 3; ++k)
            out.sh[size_t(i) * s.sh_stride * 3 + k] = T(0);
        out.weights[i] = T(0);
        for (int k = 0; k < 3; ++k) {
            out.centroids[3 * i + k] = T(0);
            out.scales[3 * i + k] = T(0);
        }
        for (int k = 0; k < 4; ++k)
            out.rotations[4 * i + k] = T(0);
        if (tiles_touched[i] == 0)
            continue;
        const double* a = tot.data() + size_t(i) * 9;
        const V3<T> mu = load3(s.centroids, size_t(i));
        const V3<T> sc = mul(load3(s.scales, size_t(i)), s.cov_scale_multiplier);
        const T* q = s.rotations + 4 * size_t(i);
        // conic = inverse(cov2f): packed conic grad -> packed cov grad
        const Gaussian2d<T> g2 = splat(Formulation::Ots, s.weights[i], mu, sc, q, cam, T(0.3f));
        const S2<T> M = inverse2(g2.cov);
        const T G[2][2] = { { T(a[2]), T(a[3]) / T(2) }, { T(a[3]) / T(2), T(a[4]) } };
        const T Mf[2][2] = { { M.v[0], M.v[1] }, { M.v[1], M.v[2] } };
        T MG[2][2], Hm[2][2];
        for (int r = 0; r < 2; ++r)
            for (int cc = 0; cc < 2; ++cc)
                MG[r][cc] = Mf[r][0] * G[0][cc] + Mf[r][1] * G[1][cc];
        for (int r = 0; r < 2; ++r)
            for (int cc = 0; cc < 2; ++cc)
                Hm[r][cc] = -(MG[r][0] * Mf[0][cc] + MG[r][1] * Mf[1][cc]);
        const S2<T> g_cov = { { Hm[0][0], T(2) * Hm[0][1], Hm[1][1] } };
        T g_weight = 0;
        V3<T> g_mu = { 0, 0, 0 }, g_s = { 0, 0, 0 };
        T g_q[4] = { 0, 0, 0, 0 };
        grad_splat(form_or(Formulation::Ots), s.weights[i], mu, sc, q, cam, T(0.3f), T(a[5]), V2<T> { T(a[0]), T(a[1]) }, g_cov, &g_weight, &g_mu, &g_s,
            g_q);
        // colour
        const V3<T> v = sub(mu, campos);
        const T vl = ofm::sqrt_f(dot(v, v));
        const V3<T> dir = mul(v, T(1) / vl);
        V3<T> sh16[16];
        load_sh16(s, unsigned(i), T(0), sh16);
        const bool cl[3] = { clamped[3 * i] != 0, clamped[3 * i + 1] != 0, clamped[3 * i + 2] != 0 };
        V3<T> g_sh16[16];
        const V3<T> g_dir = grad_sh_to_colour(sh16, s.sh_degree, dir, V3<T> { T(a[6]), T(a[7]), T(a[8]) }, cl, g_sh16);
        // dir = v / |v|
        const T gd = dot(g_dir, dir);
        g_mu = add(g_mu, mul(sub(g_dir, mul(dir, gd)), T(1) / vl));
        for (int j = 0; j < s.sh_stride && j < 16; ++j) {
            out.sh[(size_t(i) * s.sh_stride + j) * 3] = g_sh16[j].x;
            out.sh[(size_t(i) * s.sh_stride + j) * 3 + 1] = g_sh16[j].y;
            out.sh[(size_t(i) * s.sh_stride + j) * 3 + 2] = g_sh16[j].z;
        }
        out.weights[i] = g_weight;
        out.centroids[3 * i] = g_mu.x;
        out.centroids[3 * i + 1] = g_mu.y;
        out.centroids[3 * i + 2] = g_mu.z;
        for (int k = 0; k < 3; ++k)
            out.scales[3 * i + k] = g_s[k] * s.cov_scale_multiplier;
        for (int k = 0; k < 4; ++k)
            out.rotations[4 * i + k] = g_q[k];
    }
}

template <class T>
SceneIn<T> make_scene(int N, const T* centroids, const T* sh, int sh_stride, int sh_degree, const T* weights, const T* scales, const T* rotations,
    const T* view, const T* proj, const T* campos, const T* bg, int W, int H, T tanfx, T tanfy, T cov_mult)
{
    SceneIn<T> s;
    s.N = N;
    s.centroids = centroids;
    s.sh = sh;
    s.sh_stride = sh_stride;
    s.sh_degree = sh_degree;
    s.weights = weights;
    s.scales = scales;
    s.rotations = rotations;
    s.view = view;
    s.proj = proj;
    s.campos = campos;
    s.bg = bg;
    s.W = W;
    s.H = H;
    s.tan_fovx = tanfx;
    s.tan_fovy = tanfy;
    s.cov_scale_multiplier = cov_mult;
    return s;
}

// ------------------------------------------------------------- vol_raster
// src/dgmr/vol_raster_forward.cu:39-520 (float only, as in the reference)
constexpr unsigned VR_BINS = 32; // vol_raster_forward.h:61
constexpr unsigned VR_STEPS_PER_BIN = 256; // vol_raster_forward.h:62
constexpr float VR_TRANSMISSION = 0.005f; // vol_raster_forward.h:63
constexpr float VR_RELEVANCE_SIGMA = 3.f; // vol_raster_forward.h:64

struct VrCache {
    float *rgb, *depths, *xy, *inv_cov, *masses;
    uint8_t* clamped;
    int32_t *rects, *tiles_touched;
};

// vol_raster_forward.cu:86-136
void vr_preprocess(const SceneIn<float>& s, VrCache& c)
{
    const unsigned W = unsigned(s.W), H = unsigned(s.H);
    const unsigned gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    Camera<float> cam;
    cam.view = s.view;
    cam.proj = s.proj;
    cam.focal_y = float(H) / (2.0f * s.tan_fovy);
    cam.focal_x = float(W) / (2.0f * s.tan_fovx);
    cam.tan_fovx = s.tan_fovx;
    cam.tan_fovy = s.tan_fovy;
    cam.W = W;
    cam.H = H;
    const float aa = vm_aa_multiplier(s);
    const V3<float> campos = load3(s.campos, 0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s.N; ++i) {
        c.tiles_touched[i] = 0;
        c.rects[2 * i] = c.rects[2 * i + 1] = 0;
        c.xy[2 * i] = c.xy[2 * i + 1] = 0.f;
        c.depths[i] = 0.f;
        c.masses[i] = 0.f;
        for (int k = 0; k < 3; ++k) {
            c.rgb[3 * i + k] = 0.f;
            c.clamped[3 * i + k] = 0;
        }
        for (int k = 0; k < 6; ++k)
            c.inv_cov[6 * i + k] = 0.f;
        const V3<float> mu = load3(s.centroids, size_t(i));
        if (mat4_mul_point(s.view, mu).z < 0.2f)
            continue;
        const float w = s.weights[i];
        const V3<float> sc = mul(load3(s.scales, size_t(i)), s.cov_scale_multiplier);
        const float* q = s.rotations + 4 * size_t(i);
        const Gaussian2d<float> g = splat(form_or(Formulation::Ots), w, mu, sc, q, cam, 0.3f);
        const S3<float> cov3 = compute_cov(sc, q);
        const float fks = length(sub(mu, campos)) * aa;
        const float fks2 = fks * fks;
        S3<float> filtered = cov3;
        filtered.v[0] = filtered.v[0] + fks2;
        filtered.v[3] = filtered.v[3] + fks2;
        filtered.v[5] = filtered.v[5] + fks2;
        // weight_to_mass<Ots> of the scales plus the squared filter size (vol_raster_forward.cu:106)
        c.masses[i] = weight_to_mass(form_or(Formulation::Ots), w, V3<float> { sc.x + fks2, sc.y + fks2, sc.z + fks2 }, g.cov);
        const int ex = ofm::to_int_rz(ofm::ceil_f(3.f * ofm::sqrt_f(g.cov.v[0])));
        const int ey = ofm::to_int_rz(ofm::ceil_f(3.f * ofm::sqrt_f(g.cov.v[2])));
        c.rects[2 * i] = ex;
        c.rects[2 * i + 1] = ey;
        const URect r = get_rect(g.centroid.x, g.centroid.y, ex, ey, gx, gy);
        const unsigned touched = (r.x1 - r.x0) * (r.y1 - r.y0);
        if (touched == 0)
            continue;
        c.tiles_touched[i] = int32_t(touched);
        c.xy[2 * i] = g.centroid.x;
        c.xy[2 * i + 1] = g.centroid.y;
        c.depths[i] = length(sub(campos, mu));
        const V3<float> v = sub(mu, campos);
        const V3<float> dir = mul(v, 1.f / ofm::sqrt_f(dot(v, v)));
        V3<float> sh16[16];
        load_sh16(s, unsigned(i), 0.f, sh16);
        bool cl[3];
        const V3<float> col = sh_to_colour(sh16, s.sh_degree, dir, cl);
        c.rgb[3 * i] = col.x;
        c.rgb[3 * i + 1] = col.y;
        c.rgb[3 * i + 2] = col.z;
        for (int k = 0; k < 3; ++k)
            c.clamped[3 * i + k] = cl[k] ? 1 : 0;
        const S3<float> inv = inverse_sym3(filtered);
        for (int k = 0; k < 6; ++k)
            c.inv_cov[6 * i + k] = inv.v[k];
    }
}

// exp(-(x - c)^2 / (2 var)), the unnormalised 1-D Gaussian
inline float eval_exponential_1d(float c, float var, float x)
{
    const float dx = x - c;
    return ofm::exp_f((-0.5f * (dx * dx)) / var);
}

// Ray through the pixel corner at NDC z = -1 (vol_raster_forward.cu:263-268)
Ray<float> vr_pixel_ray(const float* inv_proj, V3<float> campos, unsigned px, unsigned py, unsigned W, unsigned H)
{
    const float nx = float(px * 2u) / float(W) - 1.f;
    const float ny = float(py * 2u) / float(H) - 1.f;
    V4<float> v = mat4_mul_vec4(inv_proj, V4<float> { nx, ny, -1.f, 1.f });
    v.x = v.x / v.w;
    v.y = v.y / v.w;
    v.z = v.z / v.w;
    const V3<float> dvec = { v.x - campos.x, v.y - campos.y, v.z - campos.z };
    const float il = 1.f / ofm::sqrt_f(dot(dvec, dvec));
    Ray<float> r;
    r.o = campos;
    r.d = mul(dvec, il);
    return r;
}

// vol_raster_forward.cu:253-517: bin sizing, rasterisation into bins, piecewise-linear blend
void vr_render(const SceneIn<float>& s, const VrCache& c, const int32_t* ranges, const uint32_t* list, float* fb)
{
    const unsigned W = unsigned(s.W), H = unsigned(s.H);
    const unsigned gx = (W + TILE - 1) / TILE, gy = (H + TILE - 1) / TILE;
    float inv_proj[16];
    inverse4(s.proj, inv_proj);
    const V3<float> campos = load3(s.campos, 0);
    const V3<float> bg = load3(s.bg, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int tile = 0; tile < int(gx * gy); ++tile) {
        const unsigned tx = unsigned(tile) % gx, ty = unsigned(tile) / gx;
        const int32_t b = ranges[2 * tile], e = ranges[2 * tile + 1];
        for (unsigned ly = 0; ly < TILE; ++ly)
            for (unsigned lx = 0; lx < TILE; ++lx) {
                const unsigned px = tx * TILE + lx, py = ty * TILE + ly;
                if (px >= W || py >= H)
                    continue;
                const Ray<float> ray = vr_pixel_ray(inv_proj, campos, px, py, W, H);
                oracle_vf::DepthBins<VR_BINS> sizer;
                sizer.reset(VR_RELEVANCE_SIGMA, VR_TRANSMISSION);
                for (int32_t k = b; k < e; ++k) { // pass A: bin sizes
                    const uint32_t id = list[k];
                    S3<float> Q;
                    for (int j = 0; j < 6; ++j)
                        Q.v[j] = c.inv_cov[6 * size_t(id) + j];
                    const Gauss1d<float> g = intersect_with_ray_inv_C(load3(s.centroids, id), Q, ray);
                    const float mor = g.weight * c.masses[id];
                    if (mor < 0.001f || mor > 1000.f)
                        continue;
                    if (g.C + 0.f <= 0.f)
                        continue;
                    sizer.add(mor, g.centre, ofm::sqrt_f(g.C + 0.f));
                    if (sizer.saturated())
                        break;
                }
                sizer.close();
                float bin_mass[VR_BINS][4] = {};
                float bin_eval[VR_BINS + 1][4] = {};
                for (int32_t k = b; k < e; ++k) { // pass B: masses and border values per bin
                    const uint32_t id = list[k];
                    S3<float> Q;
                    for (int j = 0; j < 6; ++j)
                        Q.v[j] = c.inv_cov[6 * size_t(id) + j];
                    const Gauss1d<float> g = intersect_with_ray_inv_C(load3(s.centroids, id), Q, ray);
                    const float centre = g.centre;
                    const float variance = g.C + 0.f;
                    const float sd = ofm::sqrt_f(variance);
                    const float inv_sd = 1.f / sd;
                    const float weight = g.weight * c.masses[id];
                    if (variance <= 0.f || ofm::isnan_f(variance) || ofm::isnan_f(weight) || weight > 100000.f)
                        continue;
                    if (weight * integrate_normalised_inv_SD(centre, inv_sd, 0.f, sizer.upper(VR_BINS - 1)) <= 0.001f)
                        continue;
                    const V3<float> rgb = load3(c.rgb, id);
                    float cdf_start = cdf_inv_SD(centre, inv_sd, 0.f);
                    for (unsigned q = 0; q < VR_BINS; ++q) {
                        const float cdf_end = cdf_inv_SD(centre, inv_sd, sizer.upper(q));
                        const float mass = (cdf_end - cdf_start) * weight;
                        cdf_start = cdf_end;
                        if (mass < 0.0001f)
                            continue;
                        bin_mass[q][0] = bin_mass[q][0] + rgb.x * mass;
                        bin_mass[q][1] = bin_mass[q][1] + rgb.y * mass;
                        bin_mass[q][2] = bin_mass[q][2] + rgb.z * mass;
                        bin_mass[q][3] = bin_mass[q][3] + mass;
                        const float ev = weight * eval_exponential_1d(centre, variance, sizer.lower(q));
                        bin_eval[q][0] = bin_eval[q][0] + rgb.x * ev;
                        bin_eval[q][1] = bin_eval[q][1] + rgb.y * ev;
                        bin_eval[q][2] = bin_eval[q][2] + rgb.z * ev;
                        bin_eval[q][3] = bin_eval[q][3] + ev;
                    }
                    const float ev = weight * eval_exponential_1d(centre, variance, sizer.upper(VR_BINS - 1));
                    bin_eval[VR_BINS][0] = bin_eval[VR_BINS][0] + rgb.x * ev;
                    bin_eval[VR_BINS][1] = bin_eval[VR_BINS][1] + rgb.y * ev;
                    bin_eval[VR_BINS][2] = bin_eval[VR_BINS][2] + rgb.z * ev;
                    bin_eval[VR_BINS][3] = bin_eval[VR_BINS][3] + ev;
                }
                // blend (RenderMode::Full).  The split of a bin's mass between its halves
                // evaluates to 0.5 for every bin and channel (vol_raster_forward.cu:473).
                float res[3] = { 0.f, 0.f, 0.f };
                float transparency = 1.f;
                for (unsigned q = 0; q < VR_BINS; ++q) {
                    const float t_right = sizer.upper(q) - sizer.lower(q);
                    if (t_right <= 0.f)
                        continue;
                    oracle_vf::BinChannel ch[4];
                    for (int k = 0; k < 4; ++k)
                        ch[k] = oracle_vf::fit_channel(0.5f, bin_mass[q][k], bin_eval[q][k], bin_eval[q + 1][k], t_right);
                    oracle_vf::integrate_bin(ch, t_right, VR_STEPS_PER_BIN, res, transparency);
                }
                // final colour C + T * background with T = 1 in this mode (vol_raster_forward.cu:509-513)
                const size_t pix = size_t(py) * W + px;
                fb[pix] = res[0] + 1.f * bg.x;
                fb[size_t(W) * H + pix] = res[1] + 1.f * bg.y;
                fb[2 * size_t(W) * H + pix] = res[2] + 1.f * bg.z;
            }
    }
}

} // namespace

// ======================================================================= C ABI
#define SCENE_ARGS(T)                                                                                                                         \
    int N, const T *centroids, const T *sh, int sh_stride, int sh_degree, const T *weights, const T *scales, const T *rotations, const T *view, \
        const T *proj, const T *campos, const T *bg, int W, int H, T tanfx, T tanfy, T cov_mult
#define SCENE_PASS N, centroids, sh, sh_stride, sh_degree, weights, scales, rotations, view, proj, campos, bg, W, H, tanfx, tanfy, cov_mult

extern "C" {

int orc_num_threads()
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

uint32_t orc_higher_msb(uint32_t n) { return higher_msb(n); }

// the formulation of the following calls: 0 = each renderer's default, else 1 + types.h value
void orc_set_formulation(int f) { g_formulation = (f >= 0 && f <= 5) ? f : 0; }

// the marcher's debug render mode for the following vol_marcher forwards (0 Full, 1 Bins, 2 Depth)
void orc_set_render_mode(int mode, int bin, double max_depth)
{
    g_render_mode.mode = mode;
    g_render_mode.bin = bin;
    g_render_mode.max_depth = max_depth;
}

// n fixed (start, end, delta_t) sections for the marcher's gradient-check mode; n = 0 turns it off
void orc_set_const_samples(int n, const double* sections)
{
    g_const_samples.n = n < 0 ? 0 : (n > 4 ? 4 : n);
    for (int i = 0; i < g_const_samples.n; ++i)
        for (int j = 0; j < 3; ++j)
            g_const_samples.s[i][j] = sections[3 * i + j];
}

// Splat forward.  Returns P (the number of (tile, Gaussian) pairs).  Sorted
// keys/values are written only if P <= pair_capacity.
int64_t orc_splat_forward_f32(SCENE_ARGS(float), float* fb, int32_t* rects, float* rgb, uint8_t* clamped, float* depths, float* xy, float* conic_opacity,
    int32_t* tiles_touched, int32_t* point_offsets, int32_t* i_ranges, uint64_t* keys, uint32_t* vals, int64_t pair_capacity, float* final_T,
    int32_t* n_contrib)
{
    const SceneIn<float> s = make_scene<float>(SCENE_PASS);
    const unsigned gx = (unsigned(W) + TILE - 1) / TILE, gy = (unsigned(H) + TILE - 1) / TILE;
    splat_preprocess(s, rgb, clamped, depths, xy, conic_opacity, rects, tiles_touched);
    inclusive_scan(N, tiles_touched, point_offsets);
    const Binning b = bin_gaussians(N, rects, xy, depths, tiles_touched, point_offsets, gx, gy);
    std::memcpy(i_ranges, b.ranges.data(), b.ranges.size() * 4);
    const int64_t P = int64_t(b.keys.size());
    if (P <= pair_capacity && keys && vals) {
        std::memcpy(keys, b.keys.data(), size_t(P) * 8);
        std::memcpy(vals, b.vals.data(), size_t(P) * 4);
    }
    splat_blend(s, rgb, xy, conic_opacity, b.ranges.data(), b.vals.data(), fb, final_T, n_contrib);
    return P;
}

// Splat backward from the forward's per-Gaussian cache, sorted list, final
// transmittance and contributor counts.
void orc_splat_backward_f32(SCENE_ARGS(float), const float* rgb, const uint8_t* clamped, const float* xy, const float* conic_opacity,
    const int32_t* tiles_touched, const int32_t* i_ranges, const uint32_t* list, const float* final_T, const int32_t* n_contrib, const float* grad_fb,
    float* g_sh, float* g_weights, float* g_centroids, float* g_scales, float* g_rotations)
{
    const SceneIn<float> s = make_scene<float>(SCENE_PASS);
    SplatGrads<float> g { g_sh, g_weights, g_centroids, g_scales, g_rotations };
    splat_backward_impl(s, rgb, clamped, xy, conic_opacity, tiles_touched, i_ranges, list, final_T, n_contrib, grad_fb, g);
}

// Double-precision splat forward+backward for finite-difference checks:
// renders, then back-propagates grad_fb through the same sorted list.
void orc_splat_render_f64(SCENE_ARGS(double), double* fb, const double* grad_fb, double* g_sh, double* g_weights, double* g_centroids, double* g_scales,
    double* g_rotations)
{
    const SceneIn<double> s = make_scene<double>(SCENE_PASS);
    const unsigned gx = (unsigned(W) + TILE - 1) / TILE, gy = (unsigned(H) + TILE - 1) / TILE;
    std::vector<double> rgb(size_t(N) * 3), depths(static_cast<size_t>(N)), xy(size_t(N) * 2), co(size_t(N) * 4), fT(size_t(W) * H);
    std::vector<uint8_t> cl(size_t(N) * 3);
    std::vector<int32_t> rects(size_t(N) * 2), tt(static_cast<size_t>(N)), off(static_cast<size_t>(N)), nc(size_t(W) * H);
    splat_preprocess(s, rgb.data(), cl.data(), depths.data(), xy.data(), co.data(), rects.data(), tt.data());
    inclusive_scan(N, tt.data(), off.data());
    const Binning b = bin_gaussians(N, rects.data(), xy.data(), depths.data(), tt.data(), off.data(), gx, gy);
    splat_blend(s, rgb.data(), xy.data(), co.data(), b.ranges.data(), b.vals.data(), fb, fT.data(), nc.data());
    if (grad_fb) {
        SplatGrads<double> g { g_sh, g_weights, g_centroids, g_scales, g_rotations };
        splat_backward_impl(s, rgb.data(), cl.data(), xy.data(), co.data(), tt.data(), b.ranges.data(), b.vals.data(), fT.data(), nc.data(), grad_fb, g);
    }
}

#define VM_CACHE_ARGS(T)                                                                                                                     \
    T *fb, int32_t *rects, T *rgb, uint8_t *clamped, T *depths, T *xy, T *inv_cov, T *masses, int32_t *tiles_touched, int32_t *point_offsets, \
        int32_t *i_ranges, T *remaining_T

// vol_marcher forward, phase 1 (per-Gaussian preprocess + scan).  Returns P.
#define DEF_VM(T, SUFFIX)                                                                                                                               \
    int64_t orc_vm_preprocess_##SUFFIX(SCENE_ARGS(T), VM_CACHE_ARGS(T))                                                                                 \
    {                                                                                                                                                    \
        const SceneIn<T> s = make_scene<T>(SCENE_PASS);                                                                                                  \
        VmCache<T> c { fb, rects, rgb, clamped, depths, xy, inv_cov, masses, tiles_touched, point_offsets, i_ranges, remaining_T };                      \
        vm_preprocess(s, c);                                                                                                                             \
        inclusive_scan(N, tiles_touched, point_offsets);                                                                                                 \
        return N > 0 ? int64_t(uint32_t(point_offsets[N - 1])) : 0;                                                                                      \
    }                                                                                                                                                    \
    /* phase 2: binning + march; list has P entries.  Returns 0, or 1 if a march hit the step limit. */                                                \
    int32_t orc_vm_render_##SUFFIX(SCENE_ARGS(T), VM_CACHE_ARGS(T), int32_t* b_point_list, uint64_t* keys)                                               \
    {                                                                                                                                                    \
        const SceneIn<T> s = make_scene<T>(SCENE_PASS);                                                                                                  \
        VmCache<T> c { fb, rects, rgb, clamped, depths, xy, inv_cov, masses, tiles_touched, point_offsets, i_ranges, remaining_T };                      \
        const unsigned gx = (unsigned(W) + TILE - 1) / TILE, gy = (unsigned(H) + TILE - 1) / TILE;                                                       \
        const Binning b = bin_gaussians(N, rects, xy, depths, tiles_touched, point_offsets, gx, gy);                                                     \
        std::memcpy(i_ranges, b.ranges.data(), b.ranges.size() * 4);                                                                                     \
        std::memcpy(b_point_list, b.vals.data(), b.vals.size() * 4);                                                                                     \
        if (keys)                                                                                                                                        \
            std::memcpy(keys, b.keys.data(), b.keys.size() * 8);                                                                                         \
        for (size_t k = 0; k < size_t(W) * H; ++k) {                                                                                                     \
            remaining_T[k] = T(1);                                                                                                                       \
            fb[k] = fb[size_t(W) * H + k] = fb[2 * size_t(W) * H + k] = T(0);                                                                            \
        }                                                                                                                                                \
        int32_t status = 0;                                                                                                                              \
        vm_march(s, b_point_list, c, &status);                                                                                                           \
        return status;                                                                                                                                   \
    }                                                                                                                                                    \
    int32_t orc_vm_backward_##SUFFIX(SCENE_ARGS(T), VM_CACHE_ARGS(T), const int32_t* b_point_list, const T* grad_fb, T* g_sh, T* g_weights,              \
        T* g_centroids, T* g_scales, T* g_rotations)                                                                                                     \
    {                                                                                                                                                    \
        const SceneIn<T> s = make_scene<T>(SCENE_PASS);                                                                                                  \
        VmCache<T> c { fb, rects, rgb, clamped, depths, xy, inv_cov, masses, tiles_touched, point_offsets, i_ranges, remaining_T };                      \
        VmGrads<T> g { g_sh, g_weights, g_centroids, g_scales, g_rotations };                                                                            \
        int32_t status = 0;                                                                                                                              \
        vm_backward_impl(s, c, b_point_list, grad_fb, g, &status);                                                                                       \
        return status;                                                                                                                                   \
    }

DEF_VM(float, f32)
DEF_VM(double, f64)

// ------------------------------------------------- known-answer test hooks
// vol_raster forward (float).  Returns P; the sorted point list is written
// when P <= pair_capacity.
int64_t orc_vr_forward_f32(SCENE_ARGS(float), float* fb, int32_t* rects, float* rgb, uint8_t* clamped, float* depths, float* xy, float* inv_cov,
    float* masses, int32_t* tiles_touched, int32_t* point_offsets, int32_t* i_ranges, uint32_t* point_list, int64_t pair_capacity)
{
    const SceneIn<float> s = make_scene<float>(SCENE_PASS);
    const unsigned gx = (unsigned(W) + TILE - 1) / TILE, gy = (unsigned(H) + TILE - 1) / TILE;
    VrCache c { rgb, depths, xy, inv_cov, masses, clamped, rects, tiles_touched };
    vr_preprocess(s, c);
    inclusive_scan(N, tiles_touched, point_offsets);
    const Binning b = bin_gaussians(N, rects, xy, depths, tiles_touched, point_offsets, gx, gy);
    std::memcpy(i_ranges, b.ranges.data(), b.ranges.size() * 4);
    const int64_t P = int64_t(b.vals.size());
    if (P <= pair_capacity && point_list)
        std::memcpy(point_list, b.vals.data(), size_t(P) * 4);
    if (P == 0) {
        // no pair: the framebuffer is the background (the reference returns before writing it)
        for (size_t k = 0; k < size_t(W) * size_t(H); ++k)
            for (int ch = 0; ch < 3; ++ch)
                fb[size_t(ch) * size_t(W) * size_t(H) + k] = bg[ch];
        return 0;
    }
    vr_render(s, c, b.ranges.data(), b.vals.data(), fb);
    return P;
}

} // extern "C"

namespace {
template <unsigned CAP, class T>
int da_puts(T start, const T* ops, int n_ops, T* out_sections, T* out_end)
{
    DensityArray<CAP, T> a(start);
    for (int i = 0; i < n_ops; ++i)
        a.put({ ops[3 * i], ops[3 * i + 1], ops[3 * i + 2] });
    for (unsigned i = 0; i < a.size(); ++i) {
        out_sections[3 * i] = a[i].start;
        out_sections[3 * i + 1] = a[i].end;
        out_sections[3 * i + 2] = a[i].delta_t;
    }
    *out_end = a.end();
    return int(a.size());
}

template <class T>
int da_dispatch(int cap, T start, const T* ops, int n_ops, T* out, T* end)
{
    switch (cap) {
    case 4:
        return da_puts<4, T>(start, ops, n_ops, out, end);
    case 8:
        return da_puts<8, T>(start, ops, n_ops, out, end);
    case 16:
        return da_puts<16, T>(start, ops, n_ops, out, end);
    }
    return -1;
}

template <unsigned CAP, class T>
void da_sample(T start, const T* ops, int n_ops, int n_samples, T* out)
{
    DensityArray<CAP, T> a(start);
    for (int i = 0; i < n_ops; ++i)
        a.put({ ops[3 * i], ops[3 * i + 1], ops[3 * i + 2] });
    if (n_samples == 16)
        sample<16>(a, out);
    else if (n_samples == 128)
        sample<128>(a, out);
}

// unittests/marching_steps.cpp:939-1002: std::srand(0), iters x puts random
// puts into a DensityArray<8>, validity after every put and the stored delta_t
// at `probes` random points against the true minimum.  Returns #failures.
template <class T>
int da_randomised(int iters, int puts, int probes)
{
    std::srand(0);
    const auto r = []() { return T(std::rand()) / T(RAND_MAX); };
    int failures = 0;
    for (int i = 0; i < iters; ++i) {
        const T smallest = r();
        DensityArray<8, T> arr(smallest);
        std::vector<Section<T>> entries;
        for (int j = 0; j < puts; ++j) {
            const T start = r() * 10.0f;
            const T end = start + r();
            entries.push_back({ start, end, r() });
            arr.put(entries.back());
            if (arr.size()) {
                failures += !(arr[0].start >= smallest);
                failures += !(arr[0].start < arr[0].end);
            }
            for (unsigned k = 1; k < arr.size(); ++k) {
                failures += !(arr[k - 1].start != arr[k].start || arr[k - 1].end != arr[k].end || arr[k - 1].delta_t != arr[k].delta_t);
                failures += !(arr[k].start < arr[k].end);
                failures += !(arr[k - 1].end <= arr[k].start);
            }
            if (arr.size() == 0)
                continue;
            for (int l = 0; l < probes; ++l) {
                const T t = r() * (arr[arr.size() - 1].end - smallest - 0.00001f) + smallest;
                T real = T(1) / T(0);
                for (const auto& e : entries)
                    if (e.start <= t && t < e.end)
                        real = min_f(real, e.delta_t);
                T comp = T(1) / T(0);
                for (unsigned k = 0; k < arr.size(); ++k)
                    if (arr[k].start <= t && t < arr[k].end) {
                        comp = arr[k].delta_t;
                        break;
                    }
                failures += !(real == comp);
            }
        }
    }
    return failures;
}
} // namespace

extern "C" {

int orc_density_array_f32(int capacity, float start, const float* ops, int n_ops, float* out_sections, float* out_end)
{
    return da_dispatch<float>(capacity, start, ops, n_ops, out_sections, out_end);
}
int orc_density_array_f64(int capacity, double start, const double* ops, int n_ops, double* out_sections, double* out_end)
{
    return da_dispatch<double>(capacity, start, ops, n_ops, out_sections, out_end);
}
void orc_density_combine_f32(const float* a, const float* b, float* out9)
{
    Section<float> p[3];
    DensityArray<4, float>::combine({ a[0], a[1], a[2] }, { b[0], b[1], b[2] }, p);
    for (int i = 0; i < 3; ++i) {
        out9[3 * i] = p[i].start;
        out9[3 * i + 1] = p[i].end;
        out9[3 * i + 2] = p[i].delta_t;
    }
}
void orc_density_combine_f64(const double* a, const double* b, double* out9)
{
    Section<double> p[3];
    DensityArray<4, double>::combine({ a[0], a[1], a[2] }, { b[0], b[1], b[2] }, p);
    for (int i = 0; i < 3; ++i) {
        out9[3 * i] = p[i].start;
        out9[3 * i + 1] = p[i].end;
        out9[3 * i + 2] = p[i].delta_t;
    }
}
void orc_density_sample_f32(int capacity, float start, const float* ops, int n_ops, int n_samples, float* out)
{
    if (capacity == 4)
        da_sample<4, float>(start, ops, n_ops, n_samples, out);
    else
        da_sample<16, float>(start, ops, n_ops, n_samples, out);
}
void orc_density_sample_f64(int capacity, double start, const double* ops, int n_ops, int n_samples, double* out)
{
    if (capacity == 4)
        da_sample<4, double>(start, ops, n_ops, n_samples, out);
    else
        da_sample<16, double>(start, ops, n_ops, n_samples, out);
}
int orc_density_randomised_f32(int iters, int puts, int probes) { return da_randomised<float>(iters, puts, probes); }
int orc_density_randomised_f64(int iters, int puts, int probes) { return da_randomised<double>(iters, puts, probes); }

// elementary functions, for error-bound tests against libm
void orc_fmath_f32(int which, const float* x, float* y, int n)
{
    for (int i = 0; i < n; ++i)
        switch (which) { // 0-2: the shared fixed-sequence routines; 3-5: the host libm
        case 0: y[i] = ofm::exp_f(x[i]); break;
        case 1: y[i] = ofm::log_f(x[i]); break;
        case 2: y[i] = ofm::erf_f(x[i]); break;
        case 3: y[i] = std::exp(x[i]); break;
        case 4: y[i] = std::log(x[i]); break;
        default: y[i] = std::erf(x[i]); break;
        }
}

// math.h:112-155 larger2 / smaller2 (the Ots / Ols mass formulations), for
// the reference's known answers (unittests/math.cpp:96-117): which = 0 larger2,
// 1 smaller2; n vec3 in v, n vec2 out.
void orc_pick2_f32(int which, const float* v, float* out, int n)
{
    for (int i = 0; i < n; ++i) {
        const V3<float> a { v[3 * i], v[3 * i + 1], v[3 * i + 2] };
        const V2<float> r = which == 0 ? larger2(a) : smaller2(a);
        out[2 * i] = r.x;
        out[2 * i + 1] = r.y;
    }
}

// Decision audit: on = 1 resets the counters and starts counting, 0 stops;
// out10 = (seen, flipped, near threshold) of alpha, section-mass and rect
// decisions, then the marcher's bin fills.
void orc_audit(int on, long* out10)
{
    DecisionAudit& a = audit();
    if (on) {
        for (int k = 0; k < AUDIT_KINDS; ++k) {
            a.seen[k] = 0;
            a.flipped[k] = 0;
            a.near[k] = 0;
        }
        a.fills = 0;
    }
    a.on = on;
    if (out10) {
        for (int k = 0; k < AUDIT_KINDS; ++k) {
            out10[3 * k] = a.seen[k].load();
            out10[3 * k + 1] = a.flipped[k].load();
            out10[3 * k + 2] = a.near[k].load();
        }
        out10[9] = a.fills.load();
    }
}

} // extern "C"
