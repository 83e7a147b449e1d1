// Adjoints of the per-Gaussian projection math (src/dgmr/grad/math.h
// restated).  Symmetric matrices are handled in packed form; the gradient of
// a packed off-diagonal entry counts both matrix entries it stands for.
#pragma once

#include "dgmr_device_math.cuh"

namespace dgmr {

// packed grad of M = P^-1 -> packed grad of P:  dL/dP = -M G M
template <class T>
__device__ __forceinline__ S3<T> grad_inverse_sym3(const S3<T>& P, const S3<T>& gM)
{
    const S3<T> M = inverse_sym3(P);
    T Mf[3][3], Gf[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Mf[i][j] = sym3(M, i, j);
            Gf[i][j] = (i == j) ? sym3(gM, i, j) : sym3(gM, i, j) / T(2);
        }
    T MG[3][3], H[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            MG[i][j] = (Mf[i][0] * Gf[0][j] + Mf[i][1] * Gf[1][j]) + Mf[i][2] * Gf[2][j];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            H[i][j] = -((MG[i][0] * Mf[0][j] + MG[i][1] * Mf[1][j]) + MG[i][2] * Mf[2][j]);
    S3<T> r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
            r.v[sym3_index(i, j)] = (i == j) ? H[i][j] : T(2) * H[i][j];
    return r;
}

// cut(A S A^T): grads w.r.t. packed S (accumulated) and rows 0-1 of A (optional)
template <class T>
__device__ __forceinline__ void grad_affine_transform_and_cut(const S3<T>& S, const M3<T>& A, const S2<T>& g, S3<T>* gS, M3<T>* gA)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const int p = sym3_index(i, j);
            T v;
            if (i == j)
                v = g.v[0] * A.m[0][i] * A.m[0][i] + g.v[1] * A.m[0][i] * A.m[1][i] + g.v[2] * A.m[1][i] * A.m[1][i];
            else
                v = g.v[0] * T(2) * A.m[0][i] * A.m[0][j] + g.v[1] * (A.m[0][i] * A.m[1][j] + A.m[0][j] * A.m[1][i]) + g.v[2] * T(2) * A.m[1][i] * A.m[1][j];
            gS->v[p] = gS->v[p] + v;
        }
    if (gA) {
        T Sa0[3], Sa1[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            Sa0[i] = (sym3(S, i, 0) * A.m[0][0] + sym3(S, i, 1) * A.m[0][1]) + sym3(S, i, 2) * A.m[0][2];
            Sa1[i] = (sym3(S, i, 0) * A.m[1][0] + sym3(S, i, 1) * A.m[1][1]) + sym3(S, i, 2) * A.m[1][2];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            gA->m[0][k] = gA->m[0][k] + g.v[0] * T(2) * Sa0[k] + g.v[1] * Sa1[k];
            gA->m[1][k] = gA->m[1][k] + g.v[1] * Sa0[k] + g.v[2] * T(2) * Sa1[k];
        }
    }
}

// compute_cov adjoint: grads w.r.t. scales and the (w,x,y,z) quaternion (accumulated)
template <class T>
__device__ __forceinline__ void grad_compute_cov(V3<T> s, T qw, T qx, T qy, T qz, const S3<T>& g, V3<T>* gs_out, T* gq)
{
    const M3<T> R = quat_to_mat3(qw, qx, qy, qz);
    const T sv[3] = { s.x, s.y, s.z };
    T M[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            M[r][c] = R.m[r][c] * sv[c];
    T G[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            G[i][j] = (i == j) ? sym3(g, i, j) : sym3(g, i, j) / T(2);
    T gR[3][3];
    T gs[3] = { 0, 0, 0 };
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T gM = T(2) * ((G[r][0] * M[0][c] + G[r][1] * M[1][c]) + G[r][2] * M[2][c]);
            gR[r][c] = gM * sv[c];
            gs[c] = gs[c] + gM * R.m[r][c];
        }
    gs_out->x = gs_out->x + gs[0];
    gs_out->y = gs_out->y + gs[1];
    gs_out->z = gs_out->z + gs[2];
    const T w = qw, x = qx, y = qy, z = qz;
    T gw = 0, gx = 0, gy = 0, gz = 0;
    gy += gR[0][0] * (T(-4) * y);
    gz += gR[0][0] * (T(-4) * z);
    gw += gR[1][0] * (T(2) * z);
    gx += gR[1][0] * (T(2) * y);
    gy += gR[1][0] * (T(2) * x);
    gz += gR[1][0] * (T(2) * w);
    gw += gR[2][0] * (T(-2) * y);
    gx += gR[2][0] * (T(2) * z);
    gy += gR[2][0] * (T(-2) * w);
    gz += gR[2][0] * (T(2) * x);
    gw += gR[0][1] * (T(-2) * z);
    gx += gR[0][1] * (T(2) * y);
    gy += gR[0][1] * (T(2) * x);
    gz += gR[0][1] * (T(-2) * w);
    gx += gR[1][1] * (T(-4) * x);
    gz += gR[1][1] * (T(-4) * z);
    gw += gR[2][1] * (T(2) * x);
    gx += gR[2][1] * (T(2) * w);
    gy += gR[2][1] * (T(2) * z);
    gz += gR[2][1] * (T(2) * y);
    gw += gR[0][2] * (T(2) * y);
    gx += gR[0][2] * (T(2) * z);
    gy += gR[0][2] * (T(2) * w);
    gz += gR[0][2] * (T(2) * x);
    gw += gR[1][2] * (T(-2) * x);
    gx += gR[1][2] * (T(-2) * w);
    gy += gR[1][2] * (T(2) * z);
    gz += gR[1][2] * (T(2) * y);
    gx += gR[2][2] * (T(-4) * x);
    gy += gR[2][2] * (T(-4) * y);
    gq[0] += gw;
    gq[1] += gx;
    gq[2] += gy;
    gq[3] += gz;
}

// Adjoint of splat_project for one Gaussian (grad/math.h:333-527 with the
// derivative of the fov clamp limits w.r.t. t.z included), every formulation.
// g_w2, g_xy, g_cov: adjoints of the screen-space weight, centroid and
// (filtered) covariance.
template <class T>
__device__ __forceinline__ void grad_splat(Formulation f, T weight, V3<T> mu, V3<T> s, T qw, T qx, T qy, T qz, const CameraT<T>& cam, T filter, T g_w2,
    V2<T> g_xy, S2<T> g_cov, T* g_weight, V3<T>* g_mu, V3<T>* g_s, T* g_q)
{
    const V4<T> tu = mat4_point(cam.view, mu);
    const T lim_x = (T(1.3) * cam.tan_fovx) * tu.z;
    const T lim_y = (T(1.3) * cam.tan_fovy) * tu.z;
    const V3<T> t = { clamp_f(tu.x, -lim_x, lim_x), clamp_f(tu.y, -lim_y, lim_y), tu.z };
    const T l = len3(t);
    const M3<T> SJ = make_jakobian(t, l, cam.focal_x, cam.focal_y);
    const M3<T> W = upper3(cam.view);
    const M3<T> Tm = matmul3(SJ, W);
    const M3<T> R = quat_to_mat3(qw, qx, qy, qz);
    const S3<T> cov3 = compute_cov(s, R);
    const S2<T> c = affine_transform_and_cut(cov3, Tm); // before the filter
    S2<T> cov2 = c;
    cov2.v[0] = cov2.v[0] + filter;
    cov2.v[2] = cov2.v[2] + filter;
    const T detSJ = det3(SJ);
    T g_detSJ = T(0);
    if (f == Formulation::Opacity) {
        // weight2d = w sqrt(max(eps, det c / det(c + filter)))
        const T dcv = det2(c), dn = det2(cov2);
        const T r = dcv / dn;
        const T factor = dgmr_fm::sqrt_f(max_f(T(0.000025), r));
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
        // weight2d = w detSJ A(s) / i2(cov2), A = 1 (Mass), i3(s) (Density), i2(larger / smaller two scales) (Ots / Ols)
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
        const T g_dc = (dc > T(0)) ? g_i2 * two_pi<T>() / (T(2) * dgmr_fm::sqrt_f(dc)) : T(0);
        g_cov.v[0] = g_cov.v[0] + g_dc * cov2.v[2];
        g_cov.v[1] = g_cov.v[1] - g_dc * T(2) * cov2.v[1];
        g_cov.v[2] = g_cov.v[2] + g_dc * cov2.v[0];
        if (f == Formulation::Density) {
            const T k = g_A * two_pi_pow_1_5<T>();
            *g_s = add3(*g_s, V3<T> { k * s.y * s.z, k * s.x * s.z, k * s.x * s.y });
        } else if (f == Formulation::Ots || f == Formulation::Ols) {
            const V2<T> l2 = f == Formulation::Ots ? larger2(s) : smaller2(s);
            const V2<T> g_l2 = { g_A * two_pi<T>() * l2.y, g_A * two_pi<T>() * l2.x };
            *g_s = add3(*g_s, f == Formulation::Ots ? grad_larger2(s, g_l2) : grad_smaller2(s, g_l2));
        }
    }
    M3<T> g_SJ = cofactor3(SJ);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            g_SJ.m[i][j] = g_SJ.m[i][j] * g_detSJ;
    S3<T> g_cov3 = { { 0, 0, 0, 0, 0, 0 } };
    M3<T> g_Tm = { { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } } };
    grad_affine_transform_and_cut(cov3, Tm, g_cov, &g_cov3, &g_Tm);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
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
    g_t = add3(g_t, mul3(t, g_l / l));
    V3<T> g_tu = { 0, 0, g_t.z };
    if (tu.x < -lim_x)
        g_tu.z = g_tu.z - g_t.x * (T(1.3) * cam.tan_fovx);
    else if (tu.x > lim_x)
        g_tu.z = g_tu.z + g_t.x * (T(1.3) * cam.tan_fovx);
    else
        g_tu.x = g_t.x;
    if (tu.y < -lim_y)
        g_tu.z = g_tu.z - g_t.y * (T(1.3) * cam.tan_fovy);
    else if (tu.y > lim_y)
        g_tu.z = g_tu.z + g_t.y * (T(1.3) * cam.tan_fovy);
    else
        g_tu.y = g_t.y;
    T gm[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        gm[c] = (W.m[0][c] * g_tu.x + W.m[1][c] * g_tu.y) + W.m[2][c] * g_tu.z;
    const V4<T> pp = mat4_point(cam.proj, mu);
    const T d = pp.w + T(0.0000001);
    const T g_px = g_xy.x * T(0.5) * T(int(cam.W));
    const T g_py = g_xy.y * T(0.5) * T(int(cam.H));
    const T g_ppx = g_px / d, g_ppy = g_py / d;
    const T g_ppw = -(g_px * pp.x + g_py * pp.y) / (d * d);
#pragma unroll
    for (int c = 0; c < 3; ++c)
        gm[c] = gm[c] + (cam.proj[c * 4 + 0] * g_ppx + cam.proj[c * 4 + 1] * g_ppy) + cam.proj[c * 4 + 3] * g_ppw;
    g_mu->x = g_mu->x + gm[0];
    g_mu->y = g_mu->y + gm[1];
    g_mu->z = g_mu->z + gm[2];
    grad_compute_cov(s, qw, qx, qy, qz, g_cov3, g_s, g_q);
}

} // namespace dgmr
