// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle.  Nothing in the product
// links this file.
//
// The oracle's own float exp / log / erf, written independently of the CUDA
// library's routines from the same published methods, so that the oracle
// compiles no product source.  The renderer takes hard decisions on these
// functions' results (alpha >= 1/255, a section's mass >= 1/255, the ceil of
// a log-derived radius), and the reference's CUDA expf / erff cannot run on a
// CPU; the two codings therefore follow one published method each, with the
// same float rounding at every step, and a CPU test compares them bit for bit
// over a sweep of every float exponent (tests/test_reference_kats.py).
//
// Methods, each restated from its source:
//  * exp: Cody & Waite, "Software Manual for the Elementary Functions"
//    (1980): x = n ln2 + r with ln2 split into a 16-bit head (n * head is
//    exact) and a tail, |r| <= ln2 / 2; e^r by its Taylor series through r^7
//    (coefficients 1/k!, evaluated by Horner's rule with fused multiply-adds);
//    the result scaled by 2^n with one rounding (ldexp).
//  * log: frexp split x = m 2^e, m moved into [sqrt(1/2), sqrt(2)], then
//    ln m = 2 atanh(s), s = (m - 1) / (m + 1), by the odd series
//    2 (s + s^3/3 + ... + s^11/11); ln x = e ln2 + ln m with the split ln2.
//  * erf: Abramowitz & Stegun, Handbook of Mathematical Functions, eq. 7.1.5
//    (the Maclaurin series, through x^23) for |x| < 1; eq. 7.1.26 (Hastings'
//    rational approximation, |error| <= 1.5e-7) for 1 <= |x| < 3.92; +-1
//    beyond, where erf already rounds to 1 in float.
// The series coefficients are computed here from their definitions (double,
// rounded once to float); the test above shows they round to the same floats
// as any other correct transcription.
//
// Compiled with -ffp-contract=off: every + - * / is rounded on its own, and
// fused multiply-adds appear only where std::fma is written.
#pragma once

#include <cmath>
#include <cstdint>

namespace ofm_rs {

namespace detail {

constexpr double factorial(int k) { return k <= 1 ? 1.0 : double(k) * factorial(k - 1); }

// 1/k! for k = 0..7, as floats
struct ExpSeries {
    float c[8];
    constexpr ExpSeries() : c {}
    {
        for (int k = 0; k < 8; ++k)
            c[k] = float(1.0 / factorial(k));
    }
};

// 2 / (2k + 1) for k = 0..5: the atanh series of ln m
struct LogSeries {
    float c[6];
    constexpr LogSeries() : c {}
    {
        for (int k = 0; k < 6; ++k)
            c[k] = float(2.0 / double(2 * k + 1));
    }
};

// (-1)^n (2 / sqrt(pi)) / (n! (2n + 1)) for n = 0..11: A&S 7.1.5
struct ErfSeries {
    float c[12];
    constexpr ErfSeries() : c {}
    {
        const double two_over_sqrt_pi = 1.12837916709551257390;
        for (int n = 0; n < 12; ++n) {
            const double mag = two_over_sqrt_pi / (factorial(n) * double(2 * n + 1));
            c[n] = float((n % 2) ? -mag : mag);
        }
    }
};

constexpr ExpSeries kExp {};
constexpr LogSeries kLog {};
constexpr ErfSeries kErf {};

// ln 2 = kLn2Head + kLn2Tail; the head has 16 significant bits, so n * head
// is exact for every |n| < 2^8
constexpr float kLn2Head = 0.693145751953125f;
constexpr float kLn2Tail = 1.42860682030941723e-06f;
constexpr float kLog2e = 1.44269504088896341f;

// Hastings' coefficients as printed in A&S 7.1.26
constexpr float kHastingsP = 0.3275911f;
constexpr float kHastingsA[5] = { 0.254829592f, -0.284496736f, 1.421413741f, -1.453152027f, 1.061405429f };

} // namespace detail

// float exp.  Below -104 the result rounds to +0, above 88.72 it overflows.
inline float exp_f(float x)
{
    using namespace detail;
    if (std::isnan(x))
        return x;
    if (x < -104.0f)
        return 0.0f;
    if (x > 88.72f)
        return HUGE_VALF;
    const float n = std::nearbyint(x * kLog2e);
    const float r = std::fma(-n, kLn2Tail, std::fma(-n, kLn2Head, x));
    float p = kExp.c[7];
    for (int k = 6; k >= 0; --k)
        p = std::fma(p, r, kExp.c[k]);
    return std::ldexp(p, int(n));
}

inline float log_f(float x)
{
    using namespace detail;
    if (std::isnan(x) || x < 0.0f)
        return NAN;
    if (x == 0.0f)
        return -HUGE_VALF;
    if (std::isinf(x))
        return x;
    int e = 0;
    float m = std::frexp(x, &e); // x = m 2^e, m in [1/2, 1)
    if (m <= 0.5f * 1.41421356237309505f) {
        m = m * 2.0f;
        e -= 1;
    }
    const float f = m - 1.0f;
    const float s = f / (2.0f + f);
    const float z = s * s;
    float p = kLog.c[5];
    for (int k = 4; k >= 0; --k)
        p = std::fma(p, z, kLog.c[k]);
    const float ef = float(e);
    return std::fma(ef, kLn2Head, std::fma(ef, kLn2Tail, s * p));
}

inline float erf_f(float x)
{
    using namespace detail;
    if (std::isnan(x))
        return x;
    const float ax = std::fabs(x);
    float y;
    if (ax < 1.0f) {
        const float z = ax * ax;
        float p = kErf.c[11];
        for (int n = 10; n >= 0; --n)
            p = std::fma(p, z, kErf.c[n]);
        y = ax * p;
    } else if (ax < 3.92f) {
        const float t = 1.0f / std::fma(kHastingsP, ax, 1.0f);
        float p = kHastingsA[4];
        for (int k = 3; k >= 0; --k)
            p = std::fma(p, t, kHastingsA[k]);
        y = 1.0f - (p * t) * exp_f(-(ax * ax));
    } else {
        y = 1.0f;
    }
    return std::signbit(x) ? -y : y; // odd: erf(-0) = -0
}

// double precision: the host C library (float64 runs are gradient checks,
// where an ulp of 1e-16 decides nothing)
inline double exp_f(double x) { return std::exp(x); }
inline double log_f(double x) { return std::log(x); }
inline double erf_f(double x) { return std::erf(x); }

template <class T>
inline T sqrt_f(T x) { return std::sqrt(x); }
template <class T>
inline T ceil_f(T x) { return std::ceil(x); }
template <class T>
inline bool isnan_f(T x) { return std::isnan(x); }

// the device's float -> int conversion: truncation toward zero, saturating at
// the int range, NaN -> 0 (a plain cast is undefined out of range on the host)
template <class T>
inline int to_int_rz(T x)
{
    if (std::isnan(x))
        return 0;
    if (x >= T(2147483648.0))
        return INT32_MAX;
    if (x <= T(-2147483648.0))
        return INT32_MIN;
    return int(std::trunc(x));
}

// min / max / clamp with the device's operand order (a NaN in the first
// argument is passed through; in the second it loses the comparison)
template <class T>
inline T min_f(T a, T b) { return (b < a) ? b : a; }
template <class T>
inline T max_f(T a, T b) { return (a < b) ? b : a; }
template <class T>
inline T clamp_f(T v, T lo, T hi) { return min_f(max_f(v, lo), hi); }

} // namespace ofm_rs
