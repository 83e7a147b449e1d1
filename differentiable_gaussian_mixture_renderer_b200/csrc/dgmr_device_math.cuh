// Per-Gaussian and per-ray device math of the rendering path.
//
// Follows the reference's device headers (src/dgmr/math.h, grad/math.h,
// util.h, constants.h) and the cuda_stroke primitives they call, restated
// from the mathematics.  Every expression is written with a fixed evaluation
// order and this translation unit is compiled with -fmad=false, IEEE division
// and square root, so tile rectangles, sort keys and blended colours are
// reproducible bit for bit by a CPU build that follows the same order.
#pragma once

#include <cstdint>

#include "dgmr_fmath.h"

namespace dgmr {

using dgmr_fm::clamp_f;
using dgmr_fm::max_f;
using dgmr_fm::min_f;

constexpr unsigned kTile = 16; // constants.h:45-46
constexpr unsigned kTilePixels = kTile * kTile;

template <class T>
struct V3 {
    T x, y, z;
};
template <class T>
struct V2 {
    T x, y;
};
template <class T>
struct V4 {
    T x, y, z, w;
};
template <class T>
struct M3 {
    T m[3][3];
};
template <class T>
struct S2 {
    T v[3]; // 00 01 11
};
template <class T>
struct S3 {
    T v[6]; // 00 01 02 11 12 22
};

template <class T>
__device__ __forceinline__ V3<T> sub3(V3<T> a, V3<T> b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
template <class T>
__device__ __forceinline__ V3<T> add3(V3<T> a, V3<T> b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
template <class T>
__device__ __forceinline__ V3<T> mul3(V3<T> a, T s) { return { a.x * s, a.y * s, a.z * s }; }
template <class T>
__device__ __forceinline__ T dot3(V3<T> a, V3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T>
__device__ __forceinline__ T len3(V3<T> a) { return dgmr_fm::sqrt_f(dot3(a, a)); }

// packed index of element (i, j) of a symmetric 3x3: 00 01 02 11 12 22
__host__ __device__ __forceinline__ constexpr int sym3_index(int i, int j)
{
    return (i < j ? i : j) * (5 - (i < j ? i : j)) / 2 + (i < j ? j : i);
}

template <class T>
__device__ __forceinline__ T sym3(const S3<T>& s, int i, int j) { return s.v[sym3_index(i, j)]; }

// camera data passed by value to the kernels; matrices in glm layout [c*4+r]
template <class T>
struct CameraT {
    T view[16];
    T proj[16];
    T inv_proj[16];
    T campos[3];
    T bg[3];
    T focal_x, focal_y, tan_fovx, tan_fovy;
    T cov_scale_multiplier;
    unsigned W, H, gx, gy;
};

template <class T>
__device__ __forceinline__ V4<T> mat4_point(const T* m, V3<T> p)
{
    V4<T> r;
    r.x = ((m[0] * p.x + m[4] * p.y) + m[8] * p.z) + m[12];
    r.y = ((m[1] * p.x + m[5] * p.y) + m[9] * p.z) + m[13];
    r.z = ((m[2] * p.x + m[6] * p.y) + m[10] * p.z) + m[14];
    r.w = ((m[3] * p.x + m[7] * p.y) + m[11] * p.z) + m[15];
    return r;
}

template <class T>
__device__ __forceinline__ T view_z(const T* m, V3<T> p) { return ((m[2] * p.x + m[6] * p.y) + m[10] * p.z) + m[14]; }

template <class T>
__device__ __forceinline__ M3<T> upper3(const T* m)
{
    M3<T> r;
#pragma unroll
    for (int rr = 0; rr < 3; ++rr)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            r.m[rr][c] = m[c * 4 + rr];
    return r;
}

template <class T>
__device__ __forceinline__ M3<T> matmul3(const M3<T>& a, const M3<T>& b)
{
    M3<T> r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r.m[i][j] = (a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j]) + a.m[i][2] * b.m[2][j];
    return r;
}

template <class T>
__device__ __forceinline__ T det3(const M3<T>& a)
{
    const auto& m = a.m;
    return (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]))
        + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

template <class T>
__device__ __forceinline__ M3<T> cofactor3(const M3<T>& a)
{
    const auto& m = a.m;
    M3<T> c;
    c.m[0][0] = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    c.m[0][1] = -(m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    c.m[0][2] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    c.m[1][0] = -(m[0][1] * m[2][2] - m[0][2] * m[2][1]);
    c.m[1][1] = m[0][0] * m[2][2] - m[0][2] * m[2][0];
    c.m[1][2] = -(m[0][0] * m[2][1] - m[0][1] * m[2][0]);
    c.m[2][0] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    c.m[2][1] = -(m[0][0] * m[1][2] - m[0][2] * m[1][0]);
    c.m[2][2] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
    return c;
}

// glm::toMat3 of a (w,x,y,z) quaternion without normalisation
template <class T>
__device__ __forceinline__ M3<T> quat_to_mat3(T w, T x, T y, T z)
{
    const T xx = x * x, yy = y * y, zz = z * z;
    const T xz = x * z, xy = x * y, yz = y * z;
    const T wx = w * x, wy = w * y, wz = w * z;
    M3<T> r;
    r.m[0][0] = T(1) - T(2) * (yy + zz);
    r.m[1][0] = T(2) * (xy + wz);
    r.m[2][0] = T(2) * (xz - wy);
    r.m[0][1] = T(2) * (xy - wz);
    r.m[1][1] = T(1) - T(2) * (xx + zz);
    r.m[2][1] = T(2) * (yz + wx);
    r.m[0][2] = T(2) * (xz + wy);
    r.m[1][2] = T(2) * (yz - wx);
    r.m[2][2] = T(1) - T(2) * (xx + yy);
    return r;
}

// math.h:170-175
template <class T>
__device__ __forceinline__ S3<T> compute_cov(V3<T> s, const M3<T>& R)
{
    M3<T> M;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        M.m[r][0] = R.m[r][0] * s.x;
        M.m[r][1] = R.m[r][1] * s.y;
        M.m[r][2] = R.m[r][2] * s.z;
    }
    S3<T> c;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
            c.v[sym3_index(i, j)] = (M.m[i][0] * M.m[j][0] + M.m[i][1] * M.m[j][1]) + M.m[i][2] * M.m[j][2];
    return c;
}

// math.h:65-73
template <class T>
__device__ __forceinline__ S2<T> affine_transform_and_cut(const S3<T>& S, const M3<T>& A)
{
    T in0[3], in1[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        in0[i] = (sym3(S, i, 0) * A.m[0][0] + sym3(S, i, 1) * A.m[0][1]) + sym3(S, i, 2) * A.m[0][2];
        in1[i] = (sym3(S, i, 0) * A.m[1][0] + sym3(S, i, 1) * A.m[1][1]) + sym3(S, i, 2) * A.m[1][2];
    }
    S2<T> r;
    r.v[0] = (A.m[0][0] * in0[0] + A.m[0][1] * in0[1]) + A.m[0][2] * in0[2];
    r.v[1] = (A.m[0][0] * in1[0] + A.m[0][1] * in1[1]) + A.m[0][2] * in1[2];
    r.v[2] = (A.m[1][0] * in1[0] + A.m[1][1] * in1[1]) + A.m[1][2] * in1[2];
    return r;
}

template <class T>
__device__ __forceinline__ T det2(const S2<T>& c) { return c.v[0] * c.v[2] - c.v[1] * c.v[1]; }

template <class T>
__device__ __forceinline__ S2<T> inverse2(const S2<T>& c)
{
    const T d = det2(c);
    return S2<T> { { c.v[2] / d, -c.v[1] / d, c.v[0] / d } };
}

template <class T>
__device__ __forceinline__ T det_sym3(const S3<T>& s)
{
    const T a = s.v[0], b = s.v[1], c = s.v[2], d = s.v[3], e = s.v[4], f = s.v[5];
    return (a * (d * f - e * e) - b * (b * f - e * c)) + c * (b * e - d * c);
}

template <class T>
__device__ __forceinline__ S3<T> inverse_sym3(const S3<T>& s)
{
    const T a = s.v[0], b = s.v[1], c = s.v[2], d = s.v[3], e = s.v[4], f = s.v[5];
    const T A = d * f - e * e;
    const T B = c * e - b * f;
    const T C = b * e - c * d;
    const T det = (a * A + b * B) + c * C;
    return S3<T> { { A / det, B / det, C / det, (a * f - c * c) / det, (b * c - a * e) / det, (a * d - b * b) / det } };
}

template <class T>
__device__ __forceinline__ constexpr T two_pi() { return T(6.283185307179586476925286766559); }
template <class T>
__device__ __forceinline__ constexpr T two_pi_pow_1_5() { return T(15.749609945722419); }

template <class T>
__device__ __forceinline__ T integrate_exponential_cov2(const S2<T>& c) { return two_pi<T>() * dgmr_fm::sqrt_f(det2(c)); }

// math.h:76-87: integral of the unnormalised Gaussian with these standard deviations
template <class T>
__device__ __forceinline__ T integrate_exponential2(V2<T> s) { return (two_pi<T>() * s.x) * s.y; }
template <class T>
__device__ __forceinline__ T integrate_exponential3(V3<T> s) { return ((two_pi_pow_1_5<T>() * s.x) * s.y) * s.z; }

// math.h:112-133
template <class T>
__device__ __forceinline__ V2<T> larger2(V3<T> v)
{
    if (v.x < v.y) {
        if (v.x < v.z)
            return { v.y, v.z };
    } else {
        if (v.y < v.z)
            return { v.x, v.z };
    }
    return { v.x, v.y };
}
template <class T>
__device__ __forceinline__ V3<T> grad_larger2(V3<T> v, V2<T> g)
{
    if (v.x < v.y) {
        if (v.x < v.z)
            return { T(0), g.x, g.y };
    } else {
        if (v.y < v.z)
            return { g.x, T(0), g.y };
    }
    return { g.x, g.y, T(0) };
}

// math.h:136-155
template <class T>
__device__ __forceinline__ V2<T> smaller2(V3<T> v)
{
    if (v.x > v.y) {
        if (v.x > v.z)
            return { v.y, v.z };
    } else {
        if (v.y > v.z)
            return { v.x, v.z };
    }
    return { v.x, v.y };
}
template <class T>
__device__ __forceinline__ V3<T> grad_smaller2(V3<T> v, V2<T> g)
{
    if (v.x > v.y) {
        if (v.x > v.z)
            return { T(0), g.x, g.y };
    } else {
        if (v.y > v.z)
            return { g.x, T(0), g.y };
    }
    return { g.x, g.y, T(0) };
}

// math.h:157-168
template <class T>
__device__ __forceinline__ M3<T> make_jakobian(V3<T> t, T l, T fx, T fy)
{
    M3<T> J;
    J.m[0][0] = fx / t.z;
    J.m[0][1] = T(0);
    J.m[0][2] = -(fx * t.x) / (t.z * t.z);
    J.m[1][0] = T(0);
    J.m[1][1] = fy / t.z;
    J.m[1][2] = -(fy * t.y) / (t.z * t.z);
    J.m[2][0] = t.x / l;
    J.m[2][1] = t.y / l;
    J.m[2][2] = t.z / l;
    return J;
}

template <class T>
struct Gaussian2d {
    T weight;
    V2<T> centroid;
    S2<T> cov;
};

// types.h:26-32.  Which formulation a renderer uses is a compile-time choice in
// the reference (splat and vol_raster: Ots, splat_forward.h:58 and
// vol_raster_forward.h:66; vol_marcher: Opacity, vol_marcher.h:66); here it
// is a per-call value with those defaults.
enum class Formulation : int { Opacity = 0, Mass = 1, Density = 2, Ots = 3, Ols = 4 };

// math.h:322-410: the screen-space Gaussian of one 3-D Gaussian, with the
// 1.3 tan(fov) clamp of t (:334-340) and the formulation's weight
template <class T>
__device__ __forceinline__ Gaussian2d<T> splat_project(Formulation f, T weight, V3<T> mu, V3<T> s, const M3<T>& R, const CameraT<T>& cam, T filter)
{
    const V4<T> tu = mat4_point(cam.view, mu);
    const T lim_x = (T(1.3) * cam.tan_fovx) * tu.z;
    const T lim_y = (T(1.3) * cam.tan_fovy) * tu.z;
    const V3<T> t = { clamp_f(tu.x, -lim_x, lim_x), clamp_f(tu.y, -lim_y, lim_y), tu.z };
    const T l = len3(t);
    const M3<T> SJ = make_jakobian(t, l, cam.focal_x, cam.focal_y);
    const M3<T> Tm = matmul3(SJ, upper3(cam.view));
    Gaussian2d<T> g;
    {
        const V4<T> pp = mat4_point(cam.proj, mu);
        const T d = pp.w + T(0.0000001);
        const T px = pp.x / d, py = pp.y / d;
        g.centroid.x = ((px + T(1)) * T(int(cam.W)) - T(1)) * T(0.5);
        g.centroid.y = ((py + T(1)) * T(int(cam.H)) - T(1)) * T(0.5);
    }
    const S3<T> cov3 = compute_cov(s, R);
    g.cov = affine_transform_and_cut(cov3, Tm);
    if (f == Formulation::Opacity) {
        S2<T> nc = g.cov;
        nc.v[0] = nc.v[0] + filter;
        nc.v[2] = nc.v[2] + filter;
        const T factor = dgmr_fm::sqrt_f(max_f(T(0.000025), det2(g.cov) / det2(nc)));
        g.cov = nc;
        g.weight = weight * factor;
        return g;
    }
    g.cov.v[0] = g.cov.v[0] + filter;
    g.cov.v[2] = g.cov.v[2] + filter;
    const T detSJ = det3(SJ);
    if (f == Formulation::Mass) {
        g.weight = (weight * detSJ) * (T(1) / integrate_exponential_cov2(g.cov));
    } else if (f == Formulation::Density) {
        g.weight = ((weight * detSJ) * integrate_exponential3(s)) / integrate_exponential_cov2(g.cov);
    } else {
        const T i2p = integrate_exponential2(f == Formulation::Ots ? larger2(s) : smaller2(s));
        g.weight = ((weight * detSJ) * i2p) / integrate_exponential_cov2(g.cov);
    }
    return g;
}

// math.h:298-320: mass of a Gaussian from its weight
template <class T>
__device__ __forceinline__ T weight_to_mass(Formulation f, T weight, V3<T> s, const S2<T>& cov2d)
{
    switch (f) {
    case Formulation::Opacity:
        return weight * integrate_exponential_cov2(cov2d);
    case Formulation::Mass:
        return weight;
    case Formulation::Density:
        return weight * integrate_exponential3(s);
    case Formulation::Ots:
        return weight * integrate_exponential2(larger2(s));
    case Formulation::Ols:
        return weight * integrate_exponential2(smaller2(s));
    }
    return T(0);
}

// SH constants, constants.h:26-43
#define DGMR_SH_C0 0.28209479177387814
#define DGMR_SH_C1 0.4886025119029199
#define DGMR_SH_C2_0 1.0925484305920792
#define DGMR_SH_C2_1 -1.0925484305920792
#define DGMR_SH_C2_2 0.31539156525252005
#define DGMR_SH_C2_3 -1.0925484305920792
#define DGMR_SH_C2_4 0.5462742152960396
#define DGMR_SH_C3_0 -0.5900435899266435
#define DGMR_SH_C3_1 2.890611442640554
#define DGMR_SH_C3_2 -0.4570457994644658
#define DGMR_SH_C3_3 0.3731763325901154
#define DGMR_SH_C3_4 -0.4570457994644658
#define DGMR_SH_C3_5 1.445305721320277
#define DGMR_SH_C3_6 -0.5900435899266435

template <class T>
__device__ __forceinline__ V3<T> sh_load(const T* sh, uint32_t i, int stride, int j, T pad)
{
    if (j >= stride)
        return { pad, pad, pad };
    const T* p = sh + (size_t(i) * stride + j) * 3;
    return { p[0], p[1], p[2] };
}

// math.h:233-271; writes the "not clamped" mask (result >= 0) like glm::greaterThanEqual
template <class T>
__device__ __forceinline__ V3<T> sh_to_colour(const T* sh, uint32_t i, int stride, int deg, V3<T> dir, uint8_t* mask)
{
    V3<T> r = mul3(sh_load(sh, i, stride, 0, T(0)), T(DGMR_SH_C0));
    if (deg > 0) {
        const T x = dir.x, y = dir.y, z = dir.z;
        r = sub3(add3(sub3(r, mul3(sh_load(sh, i, stride, 1, T(0)), T(DGMR_SH_C1) * y)), mul3(sh_load(sh, i, stride, 2, T(0)), T(DGMR_SH_C1) * z)),
            mul3(sh_load(sh, i, stride, 3, T(0)), T(DGMR_SH_C1) * x));
        if (deg > 1) {
            const T xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            V3<T> acc = mul3(sh_load(sh, i, stride, 4, T(0)), T(DGMR_SH_C2_0) * xy);
            acc = add3(acc, mul3(sh_load(sh, i, stride, 5, T(0)), T(DGMR_SH_C2_1) * yz));
            acc = add3(acc, mul3(sh_load(sh, i, stride, 6, T(0)), T(DGMR_SH_C2_2) * ((T(2) * zz - xx) - yy)));
            acc = add3(acc, mul3(sh_load(sh, i, stride, 7, T(0)), T(DGMR_SH_C2_3) * xz));
            acc = add3(acc, mul3(sh_load(sh, i, stride, 8, T(0)), T(DGMR_SH_C2_4) * (xx - yy)));
            r = add3(r, acc);
            if (deg > 2) {
                V3<T> a3 = mul3(sh_load(sh, i, stride, 9, T(0)), (T(DGMR_SH_C3_0) * y) * (T(3) * xx - yy));
                a3 = add3(a3, mul3(sh_load(sh, i, stride, 10, T(0)), (T(DGMR_SH_C3_1) * xy) * z));
                a3 = add3(a3, mul3(sh_load(sh, i, stride, 11, T(0)), (T(DGMR_SH_C3_2) * y) * ((T(4) * zz - xx) - yy)));
                a3 = add3(a3, mul3(sh_load(sh, i, stride, 12, T(0)), (T(DGMR_SH_C3_3) * z) * ((T(2) * zz - T(3) * xx) - T(3) * yy)));
                a3 = add3(a3, mul3(sh_load(sh, i, stride, 13, T(0)), (T(DGMR_SH_C3_4) * x) * ((T(4) * zz - xx) - yy)));
                a3 = add3(a3, mul3(sh_load(sh, i, stride, 14, T(0)), (T(DGMR_SH_C3_5) * z) * (xx - yy)));
                a3 = add3(a3, mul3(sh_load(sh, i, stride, 15, T(0)), (T(DGMR_SH_C3_6) * x) * (xx - T(3) * yy)));
                r = add3(r, a3);
            }
        }
    }
    r = add3(r, V3<T> { T(0.5), T(0.5), T(0.5) });
    mask[0] = r.x >= T(0);
    mask[1] = r.y >= T(0);
    mask[2] = r.z >= T(0);
    return { max_f(r.x, T(0)), max_f(r.y, T(0)), max_f(r.z, T(0)) };
}

// grad/math.h:203-282.  Writes d/dsh for the first `stride` coefficients
// (those beyond the caller's stride are padded with `pad` and dropped, like the
// reference's cat + slice) and returns d/ddirection.
template <class T>
__device__ __forceinline__ V3<T> grad_sh_to_colour(const T* sh, uint32_t i, int stride, int deg, V3<T> dir, V3<T> g_in, const uint8_t* mask, T pad,
    T* g_sh_out, bool accumulate = false)
{
    const V3<T> g = { mask[0] ? g_in.x : T(0), mask[1] ? g_in.y : T(0), mask[2] ? g_in.z : T(0) };
    const auto put = [&](int j, T basis) {
        if (j < stride) {
            T* p = g_sh_out + (size_t(i) * stride + j) * 3;
            if (accumulate) {
                p[0] += g.x * basis;
                p[1] += g.y * basis;
                p[2] += g.z * basis;
            } else {
                p[0] = g.x * basis;
                p[1] = g.y * basis;
                p[2] = g.z * basis;
            }
        }
    };
    const auto S = [&](int j) { return sh_load(sh, i, stride, j, pad); };
    if (!accumulate) {
        for (int j = 0; j < stride; ++j) {
            T* p = g_sh_out + (size_t(i) * stride + j) * 3;
            p[0] = p[1] = p[2] = T(0);
        }
    }
    V3<T> dx = { 0, 0, 0 }, dy = { 0, 0, 0 }, dz = { 0, 0, 0 };
    const T x = dir.x, y = dir.y, z = dir.z;
    put(0, T(DGMR_SH_C0));
    if (deg > 0) {
        put(1, -T(DGMR_SH_C1) * y);
        put(2, T(DGMR_SH_C1) * z);
        put(3, -T(DGMR_SH_C1) * x);
        dx = mul3(S(3), -T(DGMR_SH_C1));
        dy = mul3(S(1), -T(DGMR_SH_C1));
        dz = mul3(S(2), T(DGMR_SH_C1));
        if (deg > 1) {
            const T xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            put(4, T(DGMR_SH_C2_0) * xy);
            put(5, T(DGMR_SH_C2_1) * yz);
            put(6, T(DGMR_SH_C2_2) * ((T(2) * zz - xx) - yy));
            put(7, T(DGMR_SH_C2_3) * xz);
            put(8, T(DGMR_SH_C2_4) * (xx - yy));
            dx = add3(dx, add3(add3(add3(mul3(S(4), T(DGMR_SH_C2_0) * y), mul3(S(6), T(DGMR_SH_C2_2) * T(2) * -x)), mul3(S(7), T(DGMR_SH_C2_3) * z)),
                              mul3(S(8), T(DGMR_SH_C2_4) * T(2) * x)));
            dy = add3(dy, add3(add3(add3(mul3(S(4), T(DGMR_SH_C2_0) * x), mul3(S(5), T(DGMR_SH_C2_1) * z)), mul3(S(6), T(DGMR_SH_C2_2) * T(2) * -y)),
                              mul3(S(8), T(DGMR_SH_C2_4) * T(2) * -y)));
            dz = add3(dz, add3(add3(mul3(S(5), T(DGMR_SH_C2_1) * y), mul3(S(6), T(DGMR_SH_C2_2) * T(4) * z)), mul3(S(7), T(DGMR_SH_C2_3) * x)));
            if (deg > 2) {
                put(9, T(DGMR_SH_C3_0) * y * (T(3) * xx - yy));
                put(10, T(DGMR_SH_C3_1) * xy * z);
                put(11, T(DGMR_SH_C3_2) * y * (T(4) * zz - xx - yy));
                put(12, T(DGMR_SH_C3_3) * z * (T(2) * zz - T(3) * xx - T(3) * yy));
                put(13, T(DGMR_SH_C3_4) * x * (T(4) * zz - xx - yy));
                put(14, T(DGMR_SH_C3_5) * z * (xx - yy));
                put(15, T(DGMR_SH_C3_6) * x * (xx - T(3) * yy));
                V3<T> ax = mul3(S(9), T(DGMR_SH_C3_0) * T(6) * xy);
                ax = add3(ax, mul3(S(10), T(DGMR_SH_C3_1) * yz));
                ax = add3(ax, mul3(S(11), T(DGMR_SH_C3_2) * T(-2) * xy));
                ax = add3(ax, mul3(S(12), T(DGMR_SH_C3_3) * T(-6) * xz));
                ax = add3(ax, mul3(S(13), T(DGMR_SH_C3_4) * (T(-3) * xx + T(4) * zz - yy)));
                ax = add3(ax, mul3(S(14), T(DGMR_SH_C3_5) * T(2) * xz));
                ax = add3(ax, mul3(S(15), T(DGMR_SH_C3_6) * T(3) * (xx - yy)));
                V3<T> ay = mul3(S(9), T(DGMR_SH_C3_0) * T(3) * (xx - yy));
                ay = add3(ay, mul3(S(10), T(DGMR_SH_C3_1) * xz));
                ay = add3(ay, mul3(S(11), T(DGMR_SH_C3_2) * (T(-3) * yy + T(4) * zz - xx)));
                ay = add3(ay, mul3(S(12), T(DGMR_SH_C3_3) * T(-6) * yz));
                ay = add3(ay, mul3(S(13), T(DGMR_SH_C3_4) * T(-2) * xy));
                ay = add3(ay, mul3(S(14), T(DGMR_SH_C3_5) * T(-2) * yz));
                ay = add3(ay, mul3(S(15), T(DGMR_SH_C3_6) * T(-6) * xy));
                V3<T> az = mul3(S(10), T(DGMR_SH_C3_1) * xy);
                az = add3(az, mul3(S(11), T(DGMR_SH_C3_2) * T(8) * yz));
                az = add3(az, mul3(S(12), T(DGMR_SH_C3_3) * T(3) * (T(2) * zz - xx - yy)));
                az = add3(az, mul3(S(13), T(DGMR_SH_C3_4) * T(8) * xz));
                az = add3(az, mul3(S(14), T(DGMR_SH_C3_5) * (xx - yy)));
                dx = add3(dx, ax);
                dy = add3(dy, ay);
                dz = add3(dz, az);
            }
        }
    }
    return { dot3(dx, g), dot3(dy, g), dot3(dz, g) };
}

// util.h:42-52 -- centroid as float, integer extents, 16-pixel tiles
struct TileRect {
    unsigned x0, y0, x1, y1;
};
__device__ __forceinline__ unsigned clamp_tile(unsigned g, int v) { return v < 0 ? 0u : (unsigned(v) < g ? unsigned(v) : g); }
__device__ __forceinline__ TileRect get_rect(float px, float py, int ex, int ey, unsigned gx, unsigned gy)
{
    TileRect r;
    r.x0 = clamp_tile(gx, dgmr_fm::to_int_rz((px - float(ex)) / 16.0f));
    r.y0 = clamp_tile(gy, dgmr_fm::to_int_rz((py - float(ey)) / 16.0f));
    r.x1 = clamp_tile(gx, dgmr_fm::to_int_rz((((px + float(ex)) + 16.0f) - 1.0f) / 16.0f));
    r.y1 = clamp_tile(gy, dgmr_fm::to_int_rz((((py + float(ey)) + 16.0f) - 1.0f) / 16.0f));
    return r;
}

// ---------------------------------------------------------------- 1-D along a ray
template <class T>
struct Gauss1d {
    T weight, centre, C;
};

// Line integral of the normalised N(mu, Q^-1) along o + t d (|d| = 1).
template <class T>
__device__ __forceinline__ Gauss1d<T> intersect_with_ray_inv_C(V3<T> mu, const S3<T>& Q, V3<T> o, V3<T> d)
{
    const V3<T> c = sub3(mu, o);
    const V3<T> Qd = { (Q.v[0] * d.x + Q.v[1] * d.y) + Q.v[2] * d.z, (Q.v[1] * d.x + Q.v[3] * d.y) + Q.v[4] * d.z, (Q.v[2] * d.x + Q.v[4] * d.y) + Q.v[5] * d.z };
    const V3<T> Qc = { (Q.v[0] * c.x + Q.v[1] * c.y) + Q.v[2] * c.z, (Q.v[1] * c.x + Q.v[3] * c.y) + Q.v[4] * c.z, (Q.v[2] * c.x + Q.v[4] * c.y) + Q.v[5] * c.z };
    const T a = dot3(d, Qd);
    const T b = dot3(c, Qd);
    const T k = dot3(c, Qc);
    Gauss1d<T> g;
    g.C = T(1) / a;
    g.centre = b / a;
    const T e = k - b * g.centre;
    g.weight = (dgmr_fm::sqrt_f(det_sym3(Q) / a) * T(0.15915494309189533577)) * dgmr_fm::exp_f(T(-0.5) * e);
    return g;
}

template <class T>
__device__ __forceinline__ T cdf_inv_SD_inline(T c, T inv_sd, T x)
{
    const T z = ((x - c) * inv_sd) * T(0.70710678118654752440);
    return T(0.5) * (T(1) + dgmr_fm::erf_f(z));
}

// The marcher's copies are out of line: its backward loop body (sections, bin
// fill, bin adjoints, per-Gaussian adjoints) would otherwise inline about a
// dozen erf / exp evaluations and stall on instruction fetch (one B200,
// 100k Gaussians at 512x512: backward -30 %, forward +1.4 %).  The
// arithmetic is the same as cdf_inv_SD_inline's.
template <class T>
__device__ __noinline__ T cdf_inv_SD(T c, T inv_sd, T x)
{
    return cdf_inv_SD_inline(c, inv_sd, x);
}

// The adjoint of cdf_inv_SD at x is the normal pdf there times (-inv_sd,
// x - c); the pdf is a call of its own so that the bin-adjoint loop, which
// needs it at both borders of every bin, evaluates it once per border.
template <class T>
__device__ __noinline__ T pdf_inv_SD(T c, T inv_sd, T x)
{
    const T u = (x - c) * inv_sd;
    return T(0.39894228040143267794) * dgmr_fm::exp_f(T(-0.5) * (u * u));
}

template <class T>
__device__ __forceinline__ void grad_cdf_inv_SD(T c, T inv_sd, T x, T g, T pdf, T* g_c, T* g_inv_sd)
{
    *g_c = *g_c - g * inv_sd * pdf;
    *g_inv_sd = *g_inv_sd + g * (x - c) * pdf;
}

template <class T>
__device__ __forceinline__ void grad_intersect_with_ray_inv_C(V3<T> mu, const S3<T>& Q, V3<T> o, V3<T> d, T g_weight, T g_centre, T g_C, V3<T>* g_mu,
    S3<T>* g_Q)
{
    const V3<T> c = sub3(mu, o);
    const V3<T> Qd = { (Q.v[0] * d.x + Q.v[1] * d.y) + Q.v[2] * d.z, (Q.v[1] * d.x + Q.v[3] * d.y) + Q.v[4] * d.z, (Q.v[2] * d.x + Q.v[4] * d.y) + Q.v[5] * d.z };
    const V3<T> Qc = { (Q.v[0] * c.x + Q.v[1] * c.y) + Q.v[2] * c.z, (Q.v[1] * c.x + Q.v[3] * c.y) + Q.v[4] * c.z, (Q.v[2] * c.x + Q.v[4] * c.y) + Q.v[5] * c.z };
    const T a = dot3(d, Qd);
    const T b = dot3(c, Qd);
    const T k = dot3(c, Qc);
    const T centre = b / a;
    const T e = k - b * centre;
    const T detQ = det_sym3(Q);
    const T r = detQ / a;
    const T sr = dgmr_fm::sqrt_f(r);
    const T weight = (sr * T(0.15915494309189533577)) * dgmr_fm::exp_f(T(-0.5) * e);
    const T g_e = g_weight * (T(-0.5) * weight);
    const T g_r = (r > T(0)) ? g_weight * weight / (T(2) * r) : T(0);
    const T inv_a = T(1) / a;
    const T inv_a2 = inv_a * inv_a;
    const T g_a = -g_C * inv_a2 - g_centre * b * inv_a2 + g_e * b * b * inv_a2 - g_r * detQ * inv_a2;
    const T g_b = g_centre * inv_a - g_e * T(2) * b * inv_a;
    const T g_k = g_e;
    const T g_det = g_r * inv_a;
    const T q0 = Q.v[0], q1 = Q.v[1], q2 = Q.v[2], q3 = Q.v[3], q4 = Q.v[4], q5 = Q.v[5];
    const T cof[6] = { q3 * q5 - q4 * q4, q2 * q4 - q1 * q5, q1 * q4 - q2 * q3, q0 * q5 - q2 * q2, q1 * q2 - q0 * q4, q0 * q3 - q1 * q1 };
    const T dv[3] = { d.x, d.y, d.z };
    const T cv[3] = { c.x, c.y, c.z };
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const int p = sym3_index(i, j);
            const T f = (i == j) ? T(1) : T(2);
            T gq = g_a * dv[i] * dv[j] * f;
            gq = gq + g_b * ((i == j) ? cv[i] * dv[i] : (cv[i] * dv[j] + cv[j] * dv[i]));
            gq = gq + g_k * cv[i] * cv[j] * f;
            gq = gq + g_det * cof[p] * f;
            g_Q->v[p] = g_Q->v[p] + gq;
        }
    g_mu->x = g_mu->x + g_b * Qd.x + g_k * T(2) * Qc.x;
    g_mu->y = g_mu->y + g_b * Qd.y + g_k * T(2) * Qc.y;
    g_mu->z = g_mu->z + g_b * Qd.z + g_k * T(2) * Qc.z;
}

} // namespace dgmr
