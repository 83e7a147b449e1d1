// Per-ray state of the volume marcher: the capacity-bounded section set that
// chooses sample positions, the 128-sample walk over it, and the adjoint of
// one Gaussian's bin masses (the forward accumulation and the blend live in
// the warp-per-ray march, dgmr_march_warp.cuh).
//
// Semantics follow src/dgmr/marching_steps.h:35-220 (DensityArray, sample),
// src/dgmr/math.h:412-468 (integrate_bins, sample_gaussian) and
// src/dgmr/grad/math.h:529-620 (their adjoints).  The section-insertion steps
// are kept step for step because which sections survive when the set is full
// is part of the rendered result (the reference's known-answer tests pin it).
#pragma once

#include "dgmr_device_math.cuh"
#include "dgmr_sections.h"

namespace dgmr {

constexpr unsigned kLargeSteps = 16; // vol_marcher.h:61 -- sections per large step
constexpr unsigned kSmallSteps = 128; // vol_marcher.h:62 -- samples per large step
constexpr unsigned kBins = kSmallSteps - 1;
constexpr unsigned kStepsPerGaussian = 32; // vol_marcher.h:63
constexpr float kRelevanceSigma = 3.f; // vol_marcher.h:65
constexpr float kFilterSD = 0.55f; // vol_marcher.h:60
constexpr unsigned kMaxLargeSteps = 4096; // a ray that makes no progress stops here and flags it

template <class T>
struct alignas(sizeof(T) * 4) Bin {
    T r, g, b, m;
};

// Early-outs of math.h:442-454.  Returns false when the Gaussian adds nothing.
template <class T>
__device__ __forceinline__ bool gaussian_on_ray(const Gauss1d<T>& g, T mass, T* sd_out, T* mor_out)
{
    const T sd = dgmr_fm::sqrt_f(g.C);
    const T mor = g.weight * mass;
    *sd_out = sd;
    *mor_out = mor;
    if (dgmr_fm::isnan_f(g.centre))
        return false;
    if (mor < T(1.0f / 255.f) || mor > T(1000))
        return false;
    if (sd <= T(0.0001) || dgmr_fm::isnan_f(sd) || dgmr_fm::isnan_f(mor) || mor > T(100000))
        return false;
    return true;
}

// Range of bins a 1-D Gaussian can put mass into.  cdf_inv_SD computes
// z = ((x - c) inv_sd) / sqrt(2) and 0.5 (1 + erf(z)); for float, erf_f is
// exactly -1 / +1 once |z| >= 3.92, so a bin whose two borders both lie at
// z <= -3.92 (or both at z >= 3.92) has a CDF difference of exactly zero and is
// skipped by the mass test anyway.  For double the cut is |z| >= 5, where the
// tail mass (< 1e-12) times the largest accepted mass on the ray (1000) stays
// far below the 1e-5 per-bin threshold.  The borders are non-decreasing, so
// both ends are found by binary search; the adjoint loop below then visits
// exactly the bins that could pass the test, in the same order, with the same
// values.
template <class T>
__device__ __forceinline__ T tail_z();
template <>
__device__ __forceinline__ float tail_z<float>() { return 3.92f; }
template <>
__device__ __forceinline__ double tail_z<double>() { return 5.0; }

template <class T>
__device__ __forceinline__ T border_z(T x, T c, T inv_sd) { return ((x - c) * inv_sd) * T(0.70710678118654752440); }

// first index i in [0, n) with z(borders[i]) > lim (strict) or >= lim, else n
template <class T, bool STRICT>
__device__ __forceinline__ int first_border(const T* borders, int n, T c, T inv_sd, T lim)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const T z = border_z(borders[mid], c, inv_sd);
        if (STRICT ? (z > lim) : (z >= lim))
            hi = mid;
        else
            lo = mid + 1;
    }
    return lo;
}

template <class T>
__device__ __forceinline__ void live_bins(const T* borders, T c, T inv_sd, int* k_first, int* k_last)
{
    const int i0 = first_border<T, true>(borders, int(kSmallSteps), c, inv_sd, -tail_z<T>());
    const int j1 = first_border<T, false>(borders, int(kSmallSteps), c, inv_sd, tail_z<T>());
    *k_first = i0 > 0 ? i0 - 1 : 0;
    *k_last = j1 - 1 < int(kBins) - 1 ? j1 - 1 : int(kBins) - 1;
}

// grad/math.h:559-620; accumulates into the outputs
template <class T>
__device__ __forceinline__ void grad_sample_gaussian(V3<T> mu, const S3<T>& Q, V3<T> o, V3<T> d, T mass, V3<T> rgb, const T* borders, const Bin<T>* gbins,
    T* g_mass, V3<T>* g_rgb, V3<T>* g_mu, S3<T>* g_Q, int live_end = int(kBins))
{
    const Gauss1d<T> g = intersect_with_ray_inv_C(mu, Q, o, d);
    T sd, mor;
    if (!gaussian_on_ray(g, mass, &sd, &mor))
        return;
    const T inv_sd = T(1) / sd;
    const T centre = g.centre;
    const T mib = mor * (cdf_inv_SD(centre, inv_sd, borders[kBins]) - cdf_inv_SD(centre, inv_sd, borders[0]));
    if (mib < T(0.0001f))
        return;
    T g_centre = 0, g_inv_sd = 0, g_mor = 0;
    V3<T> grgb = { 0, 0, 0 };
    int k0, k1;
    live_bins(borders, centre, inv_sd, &k0, &k1);
    // bins from live_end on have zero adjoints (the ray stopped before them):
    // they would add exact zeros
    k1 = k1 < live_end - 1 ? k1 : live_end - 1;
    T cdf_start = cdf_inv_SD(centre, inv_sd, borders[k0]);
    // the pdf at a bin's right border is its successor's left one: kept for it
    int pdf_border = -1;
    T pdf_right = T(0);
    for (int k = k0; k <= k1; ++k) {
        const T cdf_end = cdf_inv_SD(centre, inv_sd, borders[k + 1]);
        const T delta = cdf_end - cdf_start;
        const T m = max_f(T(0), delta * mor);
        cdf_start = cdf_end;
        if (m < T(0.00001f))
            continue;
        const Bin<T> gb = gbins[k];
        grgb.x = grgb.x + gb.r * m;
        grgb.y = grgb.y + gb.g * m;
        grgb.z = grgb.z + gb.b * m;
        const T g_m = ((gb.r * rgb.x + gb.g * rgb.y) + gb.b * rgb.z) + gb.m;
        if (delta * mor <= T(0))
            continue;
        g_mor = g_mor + g_m * delta;
        const T g_delta = g_m * mor;
        const T pdf_left = pdf_border == k ? pdf_right : pdf_inv_SD(centre, inv_sd, borders[k]);
        pdf_right = pdf_inv_SD(centre, inv_sd, borders[k + 1]);
        pdf_border = k + 1;
        grad_cdf_inv_SD(centre, inv_sd, borders[k], -g_delta, pdf_left, &g_centre, &g_inv_sd);
        grad_cdf_inv_SD(centre, inv_sd, borders[k + 1], g_delta, pdf_right, &g_centre, &g_inv_sd);
    }
    const T g_w1d = g_mor * mass;
    *g_mass = *g_mass + g_mor * g.weight;
    const T g_sd = -g_inv_sd / (sd * sd);
    const T g_var = g_sd / (T(2) * sd);
    *g_rgb = add3(*g_rgb, grgb);
    grad_intersect_with_ray_inv_C(mu, Q, o, d, g_w1d, g_centre, g_var, g_mu, g_Q);
}

} // namespace dgmr
