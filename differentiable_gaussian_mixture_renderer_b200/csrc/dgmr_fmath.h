// Elementary functions with one fixed operation sequence on host and device.
//
// The renderer makes hard decisions on transcendental results: a splat
// contributes only if alpha >= 1/255, a ray section is only opened if its mass
// on the ray exceeds 1/255, a tile rectangle is the ceil() of a log-derived
// radius.  If the GPU used CUDA's expf/logf/erff and a CPU checker used libm,
// the one-ulp disagreements between them would flip a few of those decisions
// per frame and make "bit-exact" impossible.  The float routines below are
// built only from IEEE-exact operations (+ - * / sqrt, fma, rint, bit
// manipulation), so a host build (no fast-math, -ffp-contract=off) and a device
// build (-fmad=false, IEEE div/sqrt) return identical bits.
//
// Methods:
//  * exp: Cody & Waite (1980) argument reduction x = n*ln2 + r with a split
//    ln2, then the degree-7 Taylor polynomial of e^r on |r| <= ln2/2
//    (truncation error < 6e-9 relative), scaled by 2^n through the exponent
//    field.
//  * log: x = m*2^e with m in [sqrt(1/2), sqrt(2)); log(m) = 2*atanh(s),
//    s = (m-1)/(m+1), by its odd power series to s^11 (|s| < 0.172).
//  * erf: for |x| < 1 the Maclaurin series (Abramowitz & Stegun, Handbook
//    of Mathematical Functions, eq. 7.1.5) to x^23; above, eq. 7.1.26
//    (Hastings' approximation, |error| <= 1.5e-7), saturated to +-1 for
//    |x| >= 3.92 where the true erf already rounds to 1 in float.
// Double-precision overloads forward to the platform's correctly-rounding-ish
// libraries; the float64 path is used for gradient checks, where one ulp in
// 1e-16 cannot flip a decision in practice.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define DGMR_HD __host__ __device__ __forceinline__
#else
#define DGMR_HD inline
#endif

namespace dgmr_fm {

DGMR_HD float fma_f(float a, float b, float c)
{
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

DGMR_HD float rint_f(float x)
{
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return std::nearbyint(x);
#endif
}

DGMR_HD float bits_to_float(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}

DGMR_HD uint32_t float_to_bits(float f)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}

// float -> int conversion with the device semantics (truncate toward zero,
// saturate at the int range, NaN -> 0) on both sides.  Plain (int) casts are
// undefined behaviour on the host for out-of-range values.
DGMR_HD int to_int_rz(float x)
{
    if (x != x)
        return 0;
    if (x >= 2147483648.0f)
        return 2147483647;
    if (x <= -2147483648.0f)
        return -2147483647 - 1;
    return int(x);
}
DGMR_HD int to_int_rz(double x)
{
    if (x != x)
        return 0;
    if (x >= 2147483648.0)
        return 2147483647;
    if (x <= -2147483648.0)
        return -2147483647 - 1;
    return int(x);
}

// ---------------------------------------------------------------- exp
DGMR_HD float exp_f(float x)
{
    if (x != x)
        return x;
    if (x < -104.0f)
        return 0.0f;
    if (x > 88.72f)
        return bits_to_float(0x7f800000u);
    const float log2e = 1.44269504088896341f;
    const float ln2_hi = 0.693145751953125f; // 16 significant bits: n*ln2_hi exact
    const float ln2_lo = 1.42860682030941723e-06f;
    const float n = rint_f(x * log2e);
    float r = fma_f(-n, ln2_hi, x);
    r = fma_f(-n, ln2_lo, r);
    // Taylor coefficients 1/k!
    float p = 1.98412698412698413e-04f; // 1/5040
    p = fma_f(p, r, 1.38888888888888889e-03f); // 1/720
    p = fma_f(p, r, 8.33333333333333333e-03f); // 1/120
    p = fma_f(p, r, 4.16666666666666667e-02f); // 1/24
    p = fma_f(p, r, 1.66666666666666667e-01f); // 1/6
    p = fma_f(p, r, 0.5f);
    p = fma_f(p, r, 1.0f);
    p = fma_f(p, r, 1.0f);
    int ni = int(n);
    if (ni > 127) { // x in (88.38, 88.72]: exact two-step scaling
        p = p * bits_to_float(uint32_t(127 + 127) << 23);
        return p * bits_to_float(uint32_t(ni - 127 + 127) << 23);
    }
    if (ni >= -126) {
        return p * bits_to_float(uint32_t(ni + 127) << 23);
    }
    // gradual underflow: two exact power-of-two scalings
    p = p * bits_to_float(uint32_t(ni + 64 + 127) << 23);
    return p * bits_to_float(uint32_t(-64 + 127) << 23);
}

// exp_f on [-87, 0] -- the same operations, without the tests for special
// cases that cannot arise there (NaN, overflow, gradual underflow); any other
// x takes exp_f itself.  Bit-identical to exp_f for every input.
DGMR_HD float exp_f_nonpos(float x)
{
    if (!(x >= -87.0f && x <= 0.0f))
        return exp_f(x);
    const float log2e = 1.44269504088896341f;
    const float ln2_hi = 0.693145751953125f;
    const float ln2_lo = 1.42860682030941723e-06f;
    // rint by the 1.5 * 2^23 shift (ties to even, exact for |t| < 2^22), and the
    // integer read from the shifted value's low bits: no conversion instructions
    const float magic = 12582912.0f;
    const float tm = x * log2e + magic;
    const float n = tm - magic;
    const int ni = int(float_to_bits(tm)) - int(float_to_bits(magic));
    float r = fma_f(-n, ln2_hi, x);
    r = fma_f(-n, ln2_lo, r);
    float p = 1.98412698412698413e-04f;
    p = fma_f(p, r, 1.38888888888888889e-03f);
    p = fma_f(p, r, 8.33333333333333333e-03f);
    p = fma_f(p, r, 4.16666666666666667e-02f);
    p = fma_f(p, r, 1.66666666666666667e-01f);
    p = fma_f(p, r, 0.5f);
    p = fma_f(p, r, 1.0f);
    p = fma_f(p, r, 1.0f);
    return p * bits_to_float(uint32_t(ni + 127) << 23); // n in [-126, 0]
}

DGMR_HD double exp_f(double x)
{
#if defined(__CUDA_ARCH__)
    return ::exp(x);
#else
    return std::exp(x);
#endif
}

// ---------------------------------------------------------------- log
DGMR_HD float log_f(float x)
{
    if (x != x || x < 0.0f)
        return bits_to_float(0x7fc00000u);
    if (x == 0.0f)
        return bits_to_float(0xff800000u);
    if (x == bits_to_float(0x7f800000u))
        return x;
    int e_adj = 0;
    if (x < 1.17549435e-38f) { // subnormal: scale into the normal range
        x = x * 8388608.0f; // 2^23
        e_adj = -23;
    }
    const uint32_t bits = float_to_bits(x);
    int e = int((bits >> 23) & 0xffu) - 127 + e_adj;
    float m = bits_to_float((bits & 0x007fffffu) | 0x3f800000u); // [1, 2)
    if (m > 1.41421356237309505f) {
        m = m * 0.5f;
        e += 1;
    }
    const float f = m - 1.0f; // exact (Sterbenz)
    const float s = f / (2.0f + f);
    const float z = s * s;
    // 2*atanh(s) = 2 s (1 + z/3 + z^2/5 + z^3/7 + z^4/9 + z^5/11)
    float p = 0.181818181818181818f; // 2/11
    p = fma_f(p, z, 0.222222222222222222f); // 2/9
    p = fma_f(p, z, 0.285714285714285714f); // 2/7
    p = fma_f(p, z, 0.4f); // 2/5
    p = fma_f(p, z, 0.666666666666666667f); // 2/3
    p = fma_f(p, z, 2.0f);
    const float logm = s * p;
    const float ef = float(e);
    const float ln2_hi = 0.693145751953125f;
    const float ln2_lo = 1.42860682030941723e-06f;
    return fma_f(ef, ln2_hi, fma_f(ef, ln2_lo, logm));
}

DGMR_HD double log_f(double x)
{
#if defined(__CUDA_ARCH__)
    return ::log(x);
#else
    return std::log(x);
#endif
}

// ---------------------------------------------------------------- erf
// 1 / d for d in [1.32, 2.29], the range of erf_f's 7.1.26 branch
// (d = 1 + 0.3275911 |x|, 1 <= |x| < 3.92), from fused multiply-adds alone: a
// quadratic seed (relative error below 0.005), two Newton steps
// y <- y + y (1 - d y) and a last residual step.  For every float d in that
// range this is the correctly rounded 1.0f / d -- checked input by input on
// the CPU (tests/test_reference_kats.py) -- once the one input 2 - 2^-23 is
// set explicitly (its reciprocal lies just above a tie that the residual step
// rounds down).  No division: the device's IEEE division carries a slow path
// for operands this range never has.
DGMR_HD float recip_hastings(float d)
{
    float y = fma_f(fma_f(0.17927061f, d, -0.971220434f), d, 1.72301638f);
    y = fma_f(y, fma_f(-d, y, 1.0f), y);
    y = fma_f(y, fma_f(-d, y, 1.0f), y);
    y = fma_f(y, fma_f(-d, y, 1.0f), y);
    return d == 0x1.fffffep+0f ? 0x1.000002p-1f : y;
}

DGMR_HD float erf_f(float x)
{
    if (x != x)
        return x;
    const float ax = x < 0.0f ? -x : x;
    float y;
    if (ax < 1.0f) {
        // Maclaurin series (A&S 7.1.5): erf(x) = 2/sqrt(pi) sum (-1)^n x^(2n+1) / (n! (2n+1)),
        // through n = 11 (truncation < 2e-9 at |x| = 1); avoids the cancellation of
        // 7.1.26 for small arguments
        const float z = ax * ax;
        float p = -1.22905553017179263e-09f; // -2/sqrt(pi) / 918086400
        p = fma_f(p, z, 1.48071928158792176e-08f); // 2/sqrt(pi) / 76204800
        p = fma_f(p, z, -1.63658446912349245e-07f); // -2/sqrt(pi) / 6894720
        p = fma_f(p, z, 1.64621143658892463e-06f); // 2/sqrt(pi) / 685440
        p = fma_f(p, z, -1.49256503584062504e-05f); // -2/sqrt(pi) / 75600
        p = fma_f(p, z, 1.20553329817896636e-04f); // 2/sqrt(pi) / 9360
        p = fma_f(p, z, -8.54832702345085225e-04f); // -2/sqrt(pi) / 1320
        p = fma_f(p, z, 5.22397762544218793e-03f); // 2/sqrt(pi) / 216
        p = fma_f(p, z, -2.68661706451312522e-02f); // -2/sqrt(pi) / 42
        p = fma_f(p, z, 1.12837916709551261e-01f); // 2/sqrt(pi) / 10
        p = fma_f(p, z, -3.76126389031837538e-01f); // -2/sqrt(pi) / 3
        p = fma_f(p, z, 1.12837916709551256e+00f); // 2/sqrt(pi) / 1
        y = ax * p;
    } else if (ax >= 3.92f) {
        y = 1.0f;
    } else {
        // Abramowitz & Stegun 7.1.26
        const float t = recip_hastings(fma_f(0.3275911f, ax, 1.0f)); // = 1.0f / (1 + 0.3275911 ax)
        float p = 1.061405429f;
        p = fma_f(p, t, -1.453152027f);
        p = fma_f(p, t, 1.421413741f);
        p = fma_f(p, t, -0.284496736f);
        p = fma_f(p, t, 0.254829592f);
        p = p * t;
        y = 1.0f - p * exp_f(-(ax * ax));
    }
    return x < 0.0f ? -y : y;
}

DGMR_HD double erf_f(double x)
{
#if defined(__CUDA_ARCH__)
    return ::erf(x);
#else
    return std::erf(x);
#endif
}

template <typename T>
DGMR_HD T sqrt_f(T x)
{
#if defined(__CUDA_ARCH__)
    return ::sqrt(x);
#else
    return std::sqrt(x);
#endif
}

template <typename T>
DGMR_HD T ceil_f(T x)
{
#if defined(__CUDA_ARCH__)
    return ::ceil(x);
#else
    return std::ceil(x);
#endif
}

template <typename T>
DGMR_HD bool isnan_f(T x) { return x != x; }

template <typename T>
DGMR_HD T min_f(T a, T b) { return b < a ? b : a; }
template <typename T>
DGMR_HD T max_f(T a, T b) { return a < b ? b : a; }
template <typename T>
DGMR_HD T clamp_f(T v, T lo, T hi) { return min_f(max_f(v, lo), hi); }

} // namespace dgmr_fm
