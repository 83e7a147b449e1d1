// TEST INFRASTRUCTURE ONLY -- the CPU oracle.  Nothing in the product links
// this file; tests/, bench.py's cpu_baseline leg and __graft_entry__.smoke()
// use it as the checker.
//
// Small-vector math restated from the reference's device headers:
//   src/dgmr/math.h        (forward per-Gaussian math)
//   src/dgmr/grad/math.h   (adjoints)
//   src/dgmr/util.h        (getRect, getHigherMsb)
//   src/dgmr/constants.h   (SH constants, 16x16 tiles)
// and the third-party primitives those call (cg-tuwien/cuda_stroke@main,
// unpinned, not vendored), restated from mathematics:
//   eval_exponential_inv_C, intersect_with_ray_inv_C, cdf_inv_SD,
//   integrate_normalised_inv_SD, integrate_exponential(Cov2), inverse, det.
// Matrices use glm's memory layout: m[c*4 + r] is row r, column c.
// Operation order is fixed and written out; the CUDA kernels follow the same
// order so float results agree bit for bit (both sides are compiled without
// FMA contraction; the oracle's exp / log / erf are its own restatement of
// the same published methods, dgmr_oracle_fmath.h).
#pragma once

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "dgmr_oracle_fmath.h"

// The oracle's exp / log / erf.  By default its own fixed-sequence routines
// (dgmr_oracle_fmath.h): the CUDA kernels follow the same published methods
// with the same roundings, so that every threshold decision (alpha >= 1/255,
// section mass >= 1/255, the ceil of a log-derived radius) comes out the same
// on both sides.  Built with
// -DDGMR_ORACLE_LIBM, the host C library's expf / logf / erff instead: the
// nearest stand-in here for the CUDA expf / erff the reference calls, used
// only to measure how far that choice moves images and decisions.
namespace ofm {
#if defined(DGMR_ORACLE_LIBM)
inline float exp_f(float x) { return std::exp(x); }
inline float log_f(float x) { return std::log(x); }
inline float erf_f(float x) { return std::erf(x); }
inline double exp_f(double x) { return std::exp(x); }
inline double log_f(double x) { return std::log(x); }
inline double erf_f(double x) { return std::erf(x); }
#else
using ofm_rs::erf_f;
using ofm_rs::exp_f;
using ofm_rs::log_f;
#endif
using ofm_rs::ceil_f;
using ofm_rs::isnan_f;
using ofm_rs::sqrt_f;
using ofm_rs::to_int_rz;
} // namespace ofm

namespace orc {

// Decision audit.  With audit().on set, the threshold decisions that depend
// on a transcendental -- a splat's alpha >= 1/255 (exp), a ray section's mass
// >= 1/255 (exp), a marcher rectangle's ceil of the 1/255 isoline radius
// (log) -- are also taken with the host libm's function on the same argument,
// and disagreements are counted; so are the decisions whose compared value
// lies within a relative 16 * 2^-23 of the threshold (16 float ulps), the
// only ones an implementation of exp / log within 16 ulps of ours could take
// the other way.  Float only; off by default.
enum AuditKind { AUDIT_ALPHA = 0, AUDIT_SECTION_MASS = 1, AUDIT_RECT = 2, AUDIT_KINDS = 3 };
struct DecisionAudit {
    std::atomic<int> on { 0 };
    std::atomic<long> seen[AUDIT_KINDS] = {};
    std::atomic<long> flipped[AUDIT_KINDS] = {};
    std::atomic<long> near[AUDIT_KINDS] = {};
    std::atomic<long> fills { 0 }; // marcher (ray, Gaussian, large step) bin fills, the march's work unit
};
inline DecisionAudit& audit()
{
    static DecisionAudit a;
    return a;
}
inline void audit_note(AuditKind k, bool shared, bool libm, double value, double threshold)
{
    DecisionAudit& a = audit();
    a.seen[k].fetch_add(1, std::memory_order_relaxed);
    if (shared != libm)
        a.flipped[k].fetch_add(1, std::memory_order_relaxed);
    if (std::fabs(value - threshold) <= std::fabs(value) * (16.0 / 8388608.0))
        a.near[k].fetch_add(1, std::memory_order_relaxed);
}

using ofm_rs::clamp_f;
using ofm_rs::max_f;
using ofm_rs::min_f;

template <class T>
struct V2 {
    T x, y;
};
template <class T>
struct V3 {
    T x, y, z;
    T& operator[](int i) { return (&x)[i]; }
    const T& operator[](int i) const { return (&x)[i]; }
};
template <class T>
struct V4 {
    T x, y, z, w;
};
// 3x3, row-major in the mathematical sense: m[r][c]
template <class T>
struct M3 {
    T m[3][3];
};
// symmetric packed (00, 01, 11)
template <class T>
struct S2 {
    T v[3];
};
// symmetric packed (00, 01, 02, 11, 12, 22)
template <class T>
struct S3 {
    T v[6];
};

template <class T>
inline V3<T> v3(T x, T y, T z) { return V3<T> { x, y, z }; }
template <class T>
inline V3<T> sub(V3<T> a, V3<T> b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
template <class T>
inline V3<T> add(V3<T> a, V3<T> b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
template <class T>
inline V3<T> mul(V3<T> a, T s) { return { a.x * s, a.y * s, a.z * s }; }
template <class T>
inline T dot(V3<T> a, V3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T>
inline T length(V3<T> a) { return ofm::sqrt_f(dot(a, a)); }

template <class T>
inline int sym3_idx(int i, int j)
{
    static const int idx[3][3] = { { 0, 1, 2 }, { 1, 3, 4 }, { 2, 4, 5 } };
    return idx[i][j];
}
template <class T>
inline T sym3(const S3<T>& s, int i, int j) { return s.v[sym3_idx<T>(i, j)]; }

// glm mat4 (column-major array) times (p, 1); sums left to right.
template <class T>
inline V4<T> mat4_mul_point(const T* m, V3<T> p)
{
    V4<T> r;
    r.x = ((m[0] * p.x + m[4] * p.y) + m[8] * p.z) + m[12];
    r.y = ((m[1] * p.x + m[5] * p.y) + m[9] * p.z) + m[13];
    r.z = ((m[2] * p.x + m[6] * p.y) + m[10] * p.z) + m[14];
    r.w = ((m[3] * p.x + m[7] * p.y) + m[11] * p.z) + m[15];
    return r;
}
template <class T>
inline V4<T> mat4_mul_vec4(const T* m, V4<T> p)
{
    V4<T> r;
    r.x = ((m[0] * p.x + m[4] * p.y) + m[8] * p.z) + m[12] * p.w;
    r.y = ((m[1] * p.x + m[5] * p.y) + m[9] * p.z) + m[13] * p.w;
    r.z = ((m[2] * p.x + m[6] * p.y) + m[10] * p.z) + m[14] * p.w;
    r.w = ((m[3] * p.x + m[7] * p.y) + m[11] * p.z) + m[15] * p.w;
    return r;
}

// upper-left 3x3 of a glm mat4 (math matrix)
template <class T>
inline M3<T> mat3_of(const T* m)
{
    M3<T> r;
    for (int rr = 0; rr < 3; ++rr)
        for (int c = 0; c < 3; ++c)
            r.m[rr][c] = m[c * 4 + rr];
    return r;
}

template <class T>
inline M3<T> matmul(const M3<T>& a, const M3<T>& b)
{
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[i][j] = (a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j]) + a.m[i][2] * b.m[2][j];
    return r;
}

template <class T>
inline T det3(const M3<T>& a)
{
    const auto& m = a.m;
    return (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]))
        + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

// d det / d a_ij = cofactor_ij
template <class T>
inline M3<T> cofactor3(const M3<T>& a)
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

// glm::toMat3 of a (w,x,y,z) quaternion, no normalisation (math.h:173 via glm)
template <class T>
inline M3<T> quat_to_mat3(const T* q)
{
    const T w = q[0], x = q[1], y = q[2], z = q[3];
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

// compute_cov (math.h:170-175): (R S)(R S)^T, packed
template <class T>
inline S3<T> compute_cov(V3<T> s, const T* q)
{
    const M3<T> R = quat_to_mat3<T>(q);
    M3<T> M;
    for (int r = 0; r < 3; ++r) {
        M.m[r][0] = R.m[r][0] * s.x;
        M.m[r][1] = R.m[r][1] * s.y;
        M.m[r][2] = R.m[r][2] * s.z;
    }
    S3<T> c;
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j)
            c.v[sym3_idx<T>(i, j)] = (M.m[i][0] * M.m[j][0] + M.m[i][1] * M.m[j][1]) + M.m[i][2] * M.m[j][2];
    return c;
}

// affine_transform_and_cut (math.h:65-73): upper 2x2 of A S A^T
template <class T>
inline S2<T> affine_transform_and_cut(const S3<T>& S, const M3<T>& A)
{
    T in0[3], in1[3];
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
inline T det2(const S2<T>& c) { return c.v[0] * c.v[2] - c.v[1] * c.v[1]; }

template <class T>
inline S2<T> inverse2(const S2<T>& c)
{
    const T d = det2(c);
    return S2<T> { { c.v[2] / d, -c.v[1] / d, c.v[0] / d } };
}

template <class T>
inline T det_sym3(const S3<T>& s)
{
    const T a = s.v[0], b = s.v[1], c = s.v[2], d = s.v[3], e = s.v[4], f = s.v[5];
    return (a * (d * f - e * e) - b * (b * f - e * c)) + c * (b * e - d * c);
}

template <class T>
inline S3<T> inverse_sym3(const S3<T>& s)
{
    const T a = s.v[0], b = s.v[1], c = s.v[2], d = s.v[3], e = s.v[4], f = s.v[5];
    const T A = d * f - e * e;
    const T B = c * e - b * f;
    const T C = b * e - c * d;
    const T det = (a * A + b * B) + c * C;
    return S3<T> { { A / det, B / det, C / det, (a * f - c * c) / det, (b * c - a * e) / det, (a * d - b * b) / det } };
}

template <class T>
inline constexpr T two_pi() { return T(6.283185307179586476925286766559); }
// sqrt((2 pi)^3)
template <class T>
inline constexpr T two_pi_pow_1_5() { return T(15.749609945722419); }

// math.h:75-87
template <class T>
inline T integrate_exponential2(V2<T> s) { return (two_pi<T>() * s.x) * s.y; }
template <class T>
inline T integrate_exponential3(V3<T> s) { return ((two_pi_pow_1_5<T>() * s.x) * s.y) * s.z; }
// stroke::gaussian::integrate_exponential(Cov2): integral of exp(-x^T C^-1 x / 2)
template <class T>
inline T integrate_exponential_cov2(const S2<T>& c) { return two_pi<T>() * ofm::sqrt_f(det2(c)); }

// math.h:112-155
template <class T>
inline V2<T> larger2(V3<T> v)
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
inline V2<T> smaller2(V3<T> v)
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
// grad/math.h:175-201
template <class T>
inline V3<T> grad_larger2(V3<T> v, V2<T> g)
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
template <class T>
inline V3<T> grad_smaller2(V3<T> v, V2<T> g)
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

enum class Formulation : int { Opacity = 0, Mass = 1, Density = 2, Ots = 3, Ols = 4 };

template <class T>
struct Camera {
    const T* view; // glm layout
    const T* proj; // full view-projection, glm layout
    T focal_x, focal_y, tan_fovx, tan_fovy;
    unsigned W, H;
};

template <class T>
struct Gaussian2d {
    T weight;
    V2<T> centroid;
    S2<T> cov;
};

// math.h:157-168 (rows of the matrix glm builds from three columns)
template <class T>
inline M3<T> make_jakobian(V3<T> t, T l, T fx, T fy)
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

// math.h:89-104
template <class T>
inline V3<T> project(V3<T> p, const T* P)
{
    const V4<T> pp = mat4_mul_point(P, p);
    const T d = pp.w + T(0.0000001);
    return { pp.x / d, pp.y / d, pp.z / d };
}
template <class T>
inline V2<T> ndc2screen(V3<T> p, unsigned W, unsigned H)
{
    return { ((p.x + T(1)) * T(int(W)) - T(1)) * T(0.5), ((p.y + T(1)) * T(int(H)) - T(1)) * T(0.5) };
}

// math.h:322-410 (formulation switch) with the 1.3*tanfov clamp of :334-340
template <class T>
inline Gaussian2d<T> splat(Formulation f, T weight, V3<T> centroid, V3<T> s, const T* q, const Camera<T>& cam, T filter)
{
    const V4<T> tu4 = mat4_mul_point(cam.view, centroid);
    const T lim_x = (T(1.3) * cam.tan_fovx) * tu4.z;
    const T lim_y = (T(1.3) * cam.tan_fovy) * tu4.z;
    const V3<T> t = { clamp_f(tu4.x, -lim_x, lim_x), clamp_f(tu4.y, -lim_y, lim_y), tu4.z };
    const T l = length(t);
    const M3<T> SJ = make_jakobian(t, l, cam.focal_x, cam.focal_y);
    const M3<T> W = mat3_of(cam.view);
    const M3<T> Tm = matmul(SJ, W);
    Gaussian2d<T> g;
    g.centroid = ndc2screen(project(centroid, cam.proj), cam.W, cam.H);
    const S3<T> cov3 = compute_cov(s, q);
    g.cov = affine_transform_and_cut(cov3, Tm);
    switch (f) {
    case Formulation::Opacity: {
        S2<T> nc = g.cov;
        nc.v[0] = nc.v[0] + filter;
        nc.v[2] = nc.v[2] + filter;
        const T factor = ofm::sqrt_f(max_f(T(0.000025), det2(g.cov) / det2(nc)));
        g.cov = nc;
        g.weight = weight * factor;
        break;
    }
    case Formulation::Mass: {
        g.cov.v[0] = g.cov.v[0] + filter;
        g.cov.v[2] = g.cov.v[2] + filter;
        const T detSJ = det3(SJ);
        g.weight = (weight * detSJ) * (T(1) / integrate_exponential_cov2(g.cov));
        break;
    }
    case Formulation::Density: {
        g.cov.v[0] = g.cov.v[0] + filter;
        g.cov.v[2] = g.cov.v[2] + filter;
        const T detSJ = det3(SJ);
        g.weight = ((weight * detSJ) * integrate_exponential3(s)) / integrate_exponential_cov2(g.cov);
        break;
    }
    case Formulation::Ots:
    case Formulation::Ols: {
        g.cov.v[0] = g.cov.v[0] + filter;
        g.cov.v[2] = g.cov.v[2] + filter;
        const T detSJ = det3(SJ);
        const T i2p = integrate_exponential2(f == Formulation::Ots ? larger2(s) : smaller2(s));
        g.weight = ((weight * detSJ) * i2p) / integrate_exponential_cov2(g.cov);
        break;
    }
    }
    return g;
}

// math.h:298-320
template <class T>
inline T weight_to_mass(Formulation f, T weight, V3<T> s, const S2<T>& cov2d)
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

// SH constants (constants.h:26-43)
constexpr double SH_C0 = 0.28209479177387814;
constexpr double SH_C1 = 0.4886025119029199;
constexpr double SH_C2[5] = { 1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396 };
constexpr double SH_C3[7] = { -0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658, 1.445305721320277, -0.5900435899266435 };

// SH coefficient j of Gaussian i; coefficients beyond the caller's stride read `pad`
template <class T>
inline V3<T> sh_coef(const T* sh, unsigned i, int stride, int j, T pad)
{
    if (j >= stride)
        return { pad, pad, pad };
    const T* p = sh + (size_t(i) * stride + j) * 3;
    return { p[0], p[1], p[2] };
}

// math.h:233-271
template <class T>
inline V3<T> sh_to_colour(const V3<T>* sh, int deg, V3<T> dir, bool clamped_out[3])
{
    V3<T> r = mul(sh[0], T(SH_C0));
    if (deg > 0) {
        const T x = dir.x, y = dir.y, z = dir.z;
        r = sub(add(sub(r, mul(sh[1], T(SH_C1) * y)), mul(sh[2], T(SH_C1) * z)), mul(sh[3], T(SH_C1) * x));
        if (deg > 1) {
            const T xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            V3<T> acc = mul(sh[4], T(SH_C2[0]) * xy);
            acc = add(acc, mul(sh[5], T(SH_C2[1]) * yz));
            acc = add(acc, mul(sh[6], T(SH_C2[2]) * ((T(2) * zz - xx) - yy)));
            acc = add(acc, mul(sh[7], T(SH_C2[3]) * xz));
            acc = add(acc, mul(sh[8], T(SH_C2[4]) * (xx - yy)));
            r = add(r, acc);
            if (deg > 2) {
                V3<T> a3 = mul(sh[9], (T(SH_C3[0]) * y) * (T(3) * xx - yy));
                a3 = add(a3, mul(sh[10], (T(SH_C3[1]) * xy) * z));
                a3 = add(a3, mul(sh[11], (T(SH_C3[2]) * y) * ((T(4) * zz - xx) - yy)));
                a3 = add(a3, mul(sh[12], (T(SH_C3[3]) * z) * ((T(2) * zz - T(3) * xx) - T(3) * yy)));
                a3 = add(a3, mul(sh[13], (T(SH_C3[4]) * x) * ((T(4) * zz - xx) - yy)));
                a3 = add(a3, mul(sh[14], (T(SH_C3[5]) * z) * (xx - yy)));
                a3 = add(a3, mul(sh[15], (T(SH_C3[6]) * x) * (xx - T(3) * yy)));
                r = add(r, a3);
            }
        }
    }
    r = add(r, V3<T> { T(0.5), T(0.5), T(0.5) });
    clamped_out[0] = r.x >= T(0);
    clamped_out[1] = r.y >= T(0);
    clamped_out[2] = r.z >= T(0);
    return { max_f(r.x, T(0)), max_f(r.y, T(0)), max_f(r.z, T(0)) };
}

// grad/math.h:203-282: gradient w.r.t. the 16 coefficients and the direction
template <class T>
inline V3<T> grad_sh_to_colour(const V3<T>* sh, int deg, V3<T> dir, V3<T> g_in, const bool clamped[3], V3<T>* g_sh)
{
    const V3<T> g = { clamped[0] ? g_in.x : T(0), clamped[1] ? g_in.y : T(0), clamped[2] ? g_in.z : T(0) };
    for (int j = 0; j < 16; ++j)
        g_sh[j] = { 0, 0, 0 };
    V3<T> dx = { 0, 0, 0 }, dy = { 0, 0, 0 }, dz = { 0, 0, 0 };
    const T x = dir.x, y = dir.y, z = dir.z;
    g_sh[0] = mul(g, T(SH_C0));
    if (deg > 0) {
        g_sh[1] = mul(g, -T(SH_C1) * y);
        g_sh[2] = mul(g, T(SH_C1) * z);
        g_sh[3] = mul(g, -T(SH_C1) * x);
        dx = mul(sh[3], -T(SH_C1));
        dy = mul(sh[1], -T(SH_C1));
        dz = mul(sh[2], T(SH_C1));
        if (deg > 1) {
            const T xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
            g_sh[4] = mul(g, T(SH_C2[0]) * xy);
            g_sh[5] = mul(g, T(SH_C2[1]) * yz);
            g_sh[6] = mul(g, T(SH_C2[2]) * ((T(2) * zz - xx) - yy));
            g_sh[7] = mul(g, T(SH_C2[3]) * xz);
            g_sh[8] = mul(g, T(SH_C2[4]) * (xx - yy));
            dx = add(dx, add(add(add(mul(sh[4], T(SH_C2[0]) * y), mul(sh[6], T(SH_C2[2]) * T(2) * -x)), mul(sh[7], T(SH_C2[3]) * z)), mul(sh[8], T(SH_C2[4]) * T(2) * x)));
            dy = add(dy, add(add(add(mul(sh[4], T(SH_C2[0]) * x), mul(sh[5], T(SH_C2[1]) * z)), mul(sh[6], T(SH_C2[2]) * T(2) * -y)), mul(sh[8], T(SH_C2[4]) * T(2) * -y)));
            dz = add(dz, add(add(mul(sh[5], T(SH_C2[1]) * y), mul(sh[6], T(SH_C2[2]) * T(4) * z)), mul(sh[7], T(SH_C2[3]) * x)));
            if (deg > 2) {
                g_sh[9] = mul(g, T(SH_C3[0]) * y * (T(3) * xx - yy));
                g_sh[10] = mul(g, T(SH_C3[1]) * xy * z);
                g_sh[11] = mul(g, T(SH_C3[2]) * y * (T(4) * zz - xx - yy));
                g_sh[12] = mul(g, T(SH_C3[3]) * z * (T(2) * zz - T(3) * xx - T(3) * yy));
                g_sh[13] = mul(g, T(SH_C3[4]) * x * (T(4) * zz - xx - yy));
                g_sh[14] = mul(g, T(SH_C3[5]) * z * (xx - yy));
                g_sh[15] = mul(g, T(SH_C3[6]) * x * (xx - T(3) * yy));
                V3<T> ax = mul(sh[9], T(SH_C3[0]) * T(6) * xy);
                ax = add(ax, mul(sh[10], T(SH_C3[1]) * yz));
                ax = add(ax, mul(sh[11], T(SH_C3[2]) * T(-2) * xy));
                ax = add(ax, mul(sh[12], T(SH_C3[3]) * T(-6) * xz));
                ax = add(ax, mul(sh[13], T(SH_C3[4]) * (T(-3) * xx + T(4) * zz - yy)));
                ax = add(ax, mul(sh[14], T(SH_C3[5]) * T(2) * xz));
                ax = add(ax, mul(sh[15], T(SH_C3[6]) * T(3) * (xx - yy)));
                V3<T> ay = mul(sh[9], T(SH_C3[0]) * T(3) * (xx - yy));
                ay = add(ay, mul(sh[10], T(SH_C3[1]) * xz));
                ay = add(ay, mul(sh[11], T(SH_C3[2]) * (T(-3) * yy + T(4) * zz - xx)));
                ay = add(ay, mul(sh[12], T(SH_C3[3]) * T(-6) * yz));
                ay = add(ay, mul(sh[13], T(SH_C3[4]) * T(-2) * xy));
                ay = add(ay, mul(sh[14], T(SH_C3[5]) * T(-2) * yz));
                ay = add(ay, mul(sh[15], T(SH_C3[6]) * T(-6) * xy));
                V3<T> az = mul(sh[10], T(SH_C3[1]) * xy);
                az = add(az, mul(sh[11], T(SH_C3[2]) * T(8) * yz));
                az = add(az, mul(sh[12], T(SH_C3[3]) * T(3) * (T(2) * zz - xx - yy)));
                az = add(az, mul(sh[13], T(SH_C3[4]) * T(8) * xz));
                az = add(az, mul(sh[14], T(SH_C3[5]) * (xx - yy)));
                dx = add(dx, ax);
                dy = add(dy, ay);
                dz = add(dz, az);
            }
        }
    }
    return { dot(dx, g), dot(dy, g), dot(dz, g) };
}

// util.h:42-52.  The centroid is converted to float (getRect takes glm::vec2),
// the extents are ints, the tile edge is 16.
struct URect {
    unsigned x0, y0, x1, y1;
};
inline URect get_rect(float px, float py, int ex, int ey, unsigned gx, unsigned gy)
{
    const auto clampu = [](unsigned g, int v) { return v < 0 ? 0u : (unsigned(v) < g ? unsigned(v) : g); };
    URect r;
    r.x0 = clampu(gx, ofm::to_int_rz((px - float(ex)) / 16.0f));
    r.y0 = clampu(gy, ofm::to_int_rz((py - float(ey)) / 16.0f));
    r.x1 = clampu(gx, ofm::to_int_rz((((px + float(ex)) + 16.0f) - 1.0f) / 16.0f));
    r.y1 = clampu(gy, ofm::to_int_rz((((py + float(ey)) + 16.0f) - 1.0f) / 16.0f));
    return r;
}

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

// ------------------------------------------------------------ 1-D Gaussians
template <class T>
struct Ray {
    V3<T> o, d;
};
template <class T>
struct Gauss1d {
    T weight, centre, C;
};

// Line integral of the normalised 3-D Gaussian N(mu, Q^-1) along o + t d
// (|d| = 1): weight * N1(t; centre, C) with a = d'Qd, b = d'Q(mu-o),
// C = 1/a, centre = b/a, weight = sqrt(det Q / a)/(2 pi) exp(-(c'Qc - b^2/a)/2).
template <class T>
inline Gauss1d<T> intersect_with_ray_inv_C(V3<T> mu, const S3<T>& Q, const Ray<T>& ray)
{
    const V3<T> c = sub(mu, ray.o);
    const V3<T> d = ray.d;
    const V3<T> Qd = { (Q.v[0] * d.x + Q.v[1] * d.y) + Q.v[2] * d.z, (Q.v[1] * d.x + Q.v[3] * d.y) + Q.v[4] * d.z, (Q.v[2] * d.x + Q.v[4] * d.y) + Q.v[5] * d.z };
    const V3<T> Qc = { (Q.v[0] * c.x + Q.v[1] * c.y) + Q.v[2] * c.z, (Q.v[1] * c.x + Q.v[3] * c.y) + Q.v[4] * c.z, (Q.v[2] * c.x + Q.v[4] * c.y) + Q.v[5] * c.z };
    const T a = dot(d, Qd);
    const T b = dot(c, Qd);
    const T k = dot(c, Qc);
    Gauss1d<T> g;
    g.C = T(1) / a;
    g.centre = b / a;
    const T e = k - b * g.centre;
    g.weight = (ofm::sqrt_f(det_sym3(Q) / a) * T(0.15915494309189533577)) * ofm::exp_f(T(-0.5) * e);
    return g;
}

// intersect_with_ray_inv_C's weight with the host libm's exp (decision audit only)
template <class T>
inline T intersect_weight_libm(V3<T> mu, const S3<T>& Q, const Ray<T>& ray)
{
    const V3<T> c = sub(mu, ray.o);
    const V3<T> d = ray.d;
    const V3<T> Qd = { (Q.v[0] * d.x + Q.v[1] * d.y) + Q.v[2] * d.z, (Q.v[1] * d.x + Q.v[3] * d.y) + Q.v[4] * d.z, (Q.v[2] * d.x + Q.v[4] * d.y) + Q.v[5] * d.z };
    const V3<T> Qc = { (Q.v[0] * c.x + Q.v[1] * c.y) + Q.v[2] * c.z, (Q.v[1] * c.x + Q.v[3] * c.y) + Q.v[4] * c.z, (Q.v[2] * c.x + Q.v[4] * c.y) + Q.v[5] * c.z };
    const T a = dot(d, Qd);
    const T b = dot(c, Qd);
    const T k = dot(c, Qc);
    const T centre = b / a;
    const T e = k - b * centre;
    return (ofm::sqrt_f(det_sym3(Q) / a) * T(0.15915494309189533577)) * std::exp(T(-0.5) * e);
}

// cdf of N(c, 1/inv_sd^2) at x
template <class T>
inline T cdf_inv_SD(T c, T inv_sd, T x)
{
    const T z = ((x - c) * inv_sd) * T(0.70710678118654752440);
    return T(0.5) * (T(1) + ofm::erf_f(z));
}
template <class T>
inline T integrate_normalised_inv_SD(T c, T inv_sd, T a, T b) { return cdf_inv_SD(c, inv_sd, b) - cdf_inv_SD(c, inv_sd, a); }

} // namespace orc
