// TEST INFRASTRUCTURE: exposes the product's host/device headers
// (differentiable_gaussian_mixture_renderer_b200/csrc/dgmr_sections.h and
// dgmr_volume_fit.h) through a C ABI so the reference's known-answer tests
// can run them on the CPU, the way the reference's own unit tests run its
// __host__ __device__ math on the host.  The oracle's separate restatement
// of the bin sizer and bin fit (oracle/dgmr_oracle_volume_fit.h) is exposed
// beside them, so the same tests pin both and a randomised comparison checks
// that the two codings agree bit for bit.  The same holds for the elementary
// functions: the product's csrc/dgmr_fmath.h and the oracle's own
// oracle/dgmr_oracle_fmath.h are compared over a sweep of float bit patterns.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../../differentiable_gaussian_mixture_renderer_b200/csrc/dgmr_sections.h"
#include "../../differentiable_gaussian_mixture_renderer_b200/csrc/dgmr_volume_fit.h"
#include "../../oracle/dgmr_oracle_volume_fit.h"

namespace {

template <unsigned CAP, class T>
int run_puts(T start, const T* ops, int n_ops, T* out_sections, T* out_end)
{
    dgmr::SectionSet<CAP, T> s;
    s.reset(start);
    for (int i = 0; i < n_ops; ++i)
        s.put({ ops[3 * i], ops[3 * i + 1], ops[3 * i + 2] });
    for (unsigned i = 0; i < s.n; ++i) {
        out_sections[3 * i] = s.e[i].start;
        out_sections[3 * i + 1] = s.e[i].end;
        out_sections[3 * i + 2] = s.e[i].delta_t;
    }
    *out_end = s.hi;
    return int(s.n);
}

template <class T>
int puts_dispatch(int cap, T start, const T* ops, int n_ops, T* out, T* end)
{
    switch (cap) {
    case 4:
        return run_puts<4, T>(start, ops, n_ops, out, end);
    case 8:
        return run_puts<8, T>(start, ops, n_ops, out, end);
    case 16:
        return run_puts<16, T>(start, ops, n_ops, out, end);
    }
    return -1;
}

template <unsigned CAP, class T>
void run_sample(T start, const T* ops, int n_ops, T* out)
{
    dgmr::SectionSet<CAP, T> s;
    s.reset(start);
    for (int i = 0; i < n_ops; ++i)
        s.put({ ops[3 * i], ops[3 * i + 1], ops[3 * i + 2] });
    dgmr::sample_positions_n<16>(s, out);
}

// unittests/marching_steps.cpp:939-1002 on a SectionSet<8, T>: std::srand(0),
// 1000 x 100 random puts, validity after each put and the stored delta_t at 50
// random points against the true minimum.  Returns the number of failed checks.
template <class T>
int randomised(int iters, int puts, int probes)
{
    std::srand(0);
    const auto r = []() { return T(std::rand()) / T(RAND_MAX); };
    int failures = 0;
    for (int i = 0; i < iters; ++i) {
        const T smallest = r();
        dgmr::SectionSet<8, T> arr;
        arr.reset(smallest);
        std::vector<dgmr::Section<T>> entries;
        for (int j = 0; j < puts; ++j) {
            const T start = r() * 10.0f;
            const T end = start + r();
            entries.push_back({ start, end, r() });
            arr.put(entries.back());
            if (arr.n) {
                failures += !(arr.e[0].start >= smallest);
                failures += !(arr.e[0].start < arr.e[0].end);
            }
            for (unsigned k = 1; k < arr.n; ++k) {
                const auto& a = arr.e[k - 1];
                const auto& b = arr.e[k];
                failures += !(a.start != b.start || a.end != b.end || a.delta_t != b.delta_t);
                failures += !(b.start < b.end);
                failures += !(a.end <= b.start);
            }
            if (arr.n == 0)
                continue;
            for (int l = 0; l < probes; ++l) {
                const T t = r() * (arr.e[arr.n - 1].end - smallest - 0.00001f) + smallest;
                T real = T(1) / T(0);
                for (const auto& e : entries)
                    if (e.start <= t && t < e.end)
                        real = dgmr_fm::min_f(real, e.delta_t);
                T comp = T(1) / T(0);
                for (unsigned k = 0; k < arr.n; ++k)
                    if (arr.e[k].start <= t && t < arr.e[k].end) {
                        comp = arr.e[k].delta_t;
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

int kat_density_array_f32(int cap, float start, const float* ops, int n_ops, float* out, float* end) { return puts_dispatch<float>(cap, start, ops, n_ops, out, end); }
int kat_density_array_f64(int cap, double start, const double* ops, int n_ops, double* out, double* end) { return puts_dispatch<double>(cap, start, ops, n_ops, out, end); }

void kat_density_combine_f32(const float* a, const float* b, float* out9)
{
    dgmr::Section<float> p[3];
    dgmr::SectionSet<4, float>::combine({ a[0], a[1], a[2] }, { b[0], b[1], b[2] }, p);
    for (int i = 0; i < 3; ++i) {
        out9[3 * i] = p[i].start;
        out9[3 * i + 1] = p[i].end;
        out9[3 * i + 2] = p[i].delta_t;
    }
}
void kat_density_combine_f64(const double* a, const double* b, double* out9)
{
    dgmr::Section<double> p[3];
    dgmr::SectionSet<4, double>::combine({ a[0], a[1], a[2] }, { b[0], b[1], b[2] }, p);
    for (int i = 0; i < 3; ++i) {
        out9[3 * i] = p[i].start;
        out9[3 * i + 1] = p[i].end;
        out9[3 * i + 2] = p[i].delta_t;
    }
}

void kat_density_sample16_f32(float start, const float* ops, int n_ops, float* out) { run_sample<4, float>(start, ops, n_ops, out); }

int kat_density_randomised_f32(int iters, int puts, int probes) { return randomised<float>(iters, puts, probes); }
int kat_density_randomised_f64(int iters, int puts, int probes) { return randomised<double>(iters, puts, probes); }

// FunctionGroup packed as d0[4] k0[4] t1[4] t2[4] k2[4] t_right (21 doubles)
static dgmr::FunctionGroup<double> unpack(const double* p)
{
    dgmr::FunctionGroup<double> f;
    for (int i = 0; i < 4; ++i) {
        f.d0[i] = p[i];
        f.k0[i] = p[4 + i];
        f.t1[i] = p[8 + i];
        f.t2[i] = p[12 + i];
        f.k2[i] = p[16 + i];
    }
    f.t_right = p[20];
    return f;
}
static void pack(const dgmr::FunctionGroup<double>& f, double* p)
{
    for (int i = 0; i < 4; ++i) {
        p[i] = f.d0[i];
        p[4 + i] = f.k0[i];
        p[8 + i] = f.t1[i];
        p[12 + i] = f.t2[i];
        p[16 + i] = f.k2[i];
    }
    p[20] = f.t_right;
}

void kat_pl_sample(const double* packed, double t, double* out4)
{
    const auto f = unpack(packed);
    for (int i = 0; i < 4; ++i)
        out4[i] = f.sample(i, t);
}
int kat_pl_valid(const double* packed) { return unpack(packed).valid() ? 1 : 0; }
void kat_pl_create(const double* mpl, const double* mt, const double* el, const double* er, double t_right, double* packed_out)
{
    pack(dgmr::create_approximation<double>(mpl, mt, el, er, t_right), packed_out);
}
void kat_pl_volume_integrate(const double* packed, int n, int steps, double* out3)
{
    std::vector<dgmr::FunctionGroup<double>> g;
    for (int i = 0; i < n; ++i)
        g.push_back(unpack(packed + 21 * i));
    dgmr::volume_integrate<double>(g.data(), unsigned(n), unsigned(steps), out3);
}

// RasterBinSizer<4>: adds (mass, centre, sd) triples; reports is_full after
// every add, then finalises and reports is_full and begin/end of each bin.
void kat_rbs4(float sigma, float transmission_threshold, const float* adds, int n, int* full_after_add, int* full_after_finalise, float* begin4,
    float* end4)
{
    dgmr::RasterBinSizer<4> s;
    s.init(sigma, transmission_threshold);
    for (int i = 0; i < n; ++i) {
        s.add_gaussian(adds[3 * i], adds[3 * i + 1], adds[3 * i + 2]);
        full_after_add[i] = s.is_full() ? 1 : 0;
    }
    s.finalise();
    *full_after_finalise = s.is_full() ? 1 : 0;
    for (unsigned i = 0; i < 4; ++i) {
        begin4[i] = s.begin_of(i);
        end4[i] = s.end_of(i);
    }
}

// the oracle's restatement, same packing and calls as above (float inside)
void kat_pl_create_oracle(const double* mpl, const double* mt, const double* el, const double* er, double t_right, double* packed_out)
{
    for (int i = 0; i < 4; ++i) {
        const oracle_vf::BinChannel c = oracle_vf::fit_channel(float(mpl[i]), float(mt[i]), float(el[i]), float(er[i]), float(t_right));
        packed_out[i] = c.d0;
        packed_out[4 + i] = c.k0;
        packed_out[8 + i] = c.t1;
        packed_out[12 + i] = c.t2;
        packed_out[16 + i] = c.k2;
    }
    packed_out[20] = t_right;
}

void kat_pl_volume_integrate_oracle(const double* packed, int n, int steps, double* out3)
{
    float rgb[3] = { 0.f, 0.f, 0.f };
    float tr = 1.f;
    for (int g = 0; g < n; ++g) {
        const double* p = packed + 21 * g;
        oracle_vf::BinChannel ch[4];
        for (int i = 0; i < 4; ++i)
            ch[i] = oracle_vf::BinChannel { float(p[i]), float(p[4 + i]), float(p[8 + i]), float(p[12 + i]), float(p[16 + i]) };
        oracle_vf::integrate_bin(ch, float(p[20]), unsigned(steps), rgb, tr);
    }
    for (int i = 0; i < 3; ++i)
        out3[i] = rgb[i];
}

void kat_rbs4_oracle(float sigma, float transmission_threshold, const float* adds, int n, int* full_after_add, int* full_after_finalise, float* begin4,
    float* end4)
{
    oracle_vf::DepthBins<4> s;
    s.reset(sigma, transmission_threshold);
    for (int i = 0; i < n; ++i) {
        s.add(adds[3 * i], adds[3 * i + 1], adds[3 * i + 2]);
        full_after_add[i] = s.saturated() ? 1 : 0;
    }
    s.close();
    *full_after_finalise = s.saturated() ? 1 : 0;
    for (unsigned i = 0; i < 4; ++i) {
        begin4[i] = s.lower(i);
        end4[i] = s.upper(i);
    }
}

} // extern "C"

namespace {

bool same_bits(float a, float b) { return std::memcmp(&a, &b, sizeof a) == 0; }

// Random add sequences (masses, centres and sds spread as along real rays,
// with repeated centres for ties) through the product's RasterBinSizer<NB>
// and the oracle's DepthBins<NB>; counts sequences whose saturation flags or
// final borders differ in any bit.
template <unsigned NB>
long compare_sizers(unsigned seed, int trials)
{
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> u(0.f, 1.f);
    long bad = 0;
    for (int t = 0; t < trials; ++t) {
        dgmr::RasterBinSizer<NB> a;
        oracle_vf::DepthBins<NB> b;
        a.init(3.f, 0.005f);
        b.reset(3.f, 0.005f);
        const int n = 1 + int(u(rng) * 80.f);
        bool ok = true;
        float prev_centre = 2.f;
        for (int i = 0; i < n && ok; ++i) {
            const float mass = u(rng) < 0.1f ? 0.00005f : 0.0002f + 0.6f * u(rng) * u(rng);
            const float centre = u(rng) < 0.1f ? prev_centre : 2.f + 3.f * u(rng);
            prev_centre = centre;
            const float sd = 0.005f + 0.1f * u(rng);
            a.add_gaussian(mass, centre, sd);
            b.add(mass, centre, sd);
            ok = a.is_full() == b.saturated();
        }
        a.finalise();
        b.close();
        for (unsigned i = 0; i < NB && ok; ++i)
            ok = same_bits(a.begin_of(i), b.lower(i)) && same_bits(a.end_of(i), b.upper(i));
        bad += ok ? 0 : 1;
    }
    return bad;
}

} // namespace

extern "C" long kat_compare_sizers(unsigned seed, int trials) { return compare_sizers<32>(seed, trials) + compare_sizers<4>(seed + 1, trials); }

// Random bin fits (float) through the product's create_approximation and the
// oracle's fit_channel: counts channels whose five parameters differ in any bit.
extern "C" long kat_compare_fits(unsigned seed, int trials)
{
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> u(0.f, 1.f);
    long bad = 0;
    for (int t = 0; t < trials; ++t) {
        float mpl[4], mt[4], el[4], er[4];
        for (int i = 0; i < 4; ++i) {
            mpl[i] = u(rng) < 0.3f ? 0.5f : u(rng);
            mt[i] = u(rng) < 0.1f ? 0.0000005f : 2.f * u(rng) * u(rng);
            el[i] = 0.001f + 2.f * u(rng);
            er[i] = 0.001f + 2.f * u(rng);
        }
        const float tr = 0.001f + 3.f * u(rng);
        const dgmr::FunctionGroup<float> f = dgmr::create_approximation<float>(mpl, mt, el, er, tr);
        for (int i = 0; i < 4; ++i) {
            const oracle_vf::BinChannel c = oracle_vf::fit_channel(mpl[i], mt[i], el[i], er[i], tr);
            const bool ok = same_bits(f.d0[i], c.d0) && same_bits(f.k0[i], c.k0) && same_bits(f.t1[i], c.t1) && same_bits(f.t2[i], c.t2)
                && same_bits(f.k2[i], c.k2);
            bad += ok ? 0 : 1;
        }
    }
    return bad;
}

namespace {

// Random insertion sequences (coarse values make equal ends and steps common):
// for every insertion that SectionSet::put_leaves_unchanged accepts, the set
// after put must be the set before, bit for bit.  Returns the mismatches;
// *covered counts the accepted insertions.
template <class T>
long check_unchanged(unsigned seed, int trials, long* covered)
{
    std::mt19937 rng(seed);
    long bad = 0, cov = 0;
    for (int trial = 0; trial < trials; ++trial) {
        dgmr::SectionSet<16, T> sec;
        sec.reset(T(rng() % 3) * T(0.5));
        const int n_put = 5 + int(rng() % 60);
        for (int k = 0; k < n_put; ++k) {
            T c = T(std::uniform_real_distribution<double>(0.0, 10.0)(rng));
            T w = T(0.05 + std::uniform_real_distribution<double>(0.0, 2.0)(rng));
            if (rng() % 2) {
                c = T(int(c * T(4))) / T(4);
                w = T(1 + rng() % 8) / T(4);
            }
            const T dt = (rng() % 3 == 0) ? T(1 + rng() % 4) / T(32) : w / T(31);
            const dgmr::Section<T> s { c - w, c + w, dt };
            const bool reaches = !(s.end <= sec.lo || s.start >= sec.hi);
            const bool same_claim = reaches && sec.put_leaves_unchanged(s);
            const dgmr::SectionSet<16, T> before = sec;
            sec.put(s);
            if (!same_claim)
                continue;
            ++cov;
            bool same = before.n == sec.n && before.lo == sec.lo && before.hi == sec.hi;
            for (unsigned q = 0; same && q < sec.n; ++q)
                same = std::memcmp(&before.e[q], &sec.e[q], sizeof(dgmr::Section<T>)) == 0;
            bad += same ? 0 : 1;
        }
    }
    *covered = cov;
    return bad;
}

// The same kind of sequences, inserted into two sets: one by put(), one by
// put_by_pieces() (the merged pieces written after the kept prefix, then the
// kept tail, cut to the capacity).  After every insertion both sets must be
// the same bits.  Returns the mismatches; *merges counts insertions that went
// through the merge (not an append or a full-set cut).
template <class T, unsigned MAX>
long check_by_pieces(unsigned seed, int trials, long* merges)
{
    std::mt19937 rng(seed);
    long bad = 0, merged = 0;
    for (int trial = 0; trial < trials; ++trial) {
        dgmr::SectionSet<MAX, T> a, b;
        a.reset(T(rng() % 3) * T(0.5));
        b = a;
        const int n_put = 5 + int(rng() % 80);
        for (int k = 0; k < n_put; ++k) {
            T c = T(std::uniform_real_distribution<double>(0.0, 10.0)(rng));
            T w = T(0.02 + std::uniform_real_distribution<double>(0.0, 2.0)(rng));
            if (rng() % 2) {
                c = T(int(c * T(4))) / T(4);
                w = T(1 + rng() % 8) / T(4);
            }
            const T dt = (rng() % 3 == 0) ? T(1 + rng() % 4) / T(32) : w / T(31);
            const dgmr::Section<T> s { c - w, c + w, dt };
            const unsigned n0 = a.n;
            a.put(s);
            b.put_by_pieces(s);
            if (a.n != n0 || a.n == MAX)
                ++merged;
            bool same = a.n == b.n && std::memcmp(&a.lo, &b.lo, sizeof(T)) == 0 && std::memcmp(&a.hi, &b.hi, sizeof(T)) == 0;
            for (unsigned q = 0; same && q < a.n; ++q)
                same = std::memcmp(&a.e[q], &b.e[q], sizeof(dgmr::Section<T>)) == 0;
            if (!same) {
                ++bad;
                b = a; // continue the sequence from the reference state
            }
        }
    }
    *merges = merged;
    return bad;
}

// Sample positions of random section sets (built by random insertion
// sequences; some with very small steps, so that the 128-sample cap cuts a
// section short) by sample_positions_n and by sample_positions_by_sections:
// the same bits.  Returns the mismatching sets; *sets counts those compared.
template <class T>
long check_samples_by_sections(unsigned seed, int trials, long* sets)
{
    std::mt19937 rng(seed);
    long bad = 0, n_sets = 0;
    for (int trial = 0; trial < trials; ++trial) {
        dgmr::SectionSet<16, T> sec;
        sec.reset(T(rng() % 3) * T(0.5));
        const bool fine = rng() % 4 == 0;
        const int n_put = 1 + int(rng() % 40);
        for (int k = 0; k < n_put; ++k) {
            T c = T(std::uniform_real_distribution<double>(0.0, 10.0)(rng));
            T w = T(0.02 + std::uniform_real_distribution<double>(0.0, 2.0)(rng));
            if (rng() % 2) {
                c = T(int(c * T(4))) / T(4);
                w = T(1 + rng() % 8) / T(4);
            }
            T dt = (rng() % 3 == 0) ? T(1 + rng() % 4) / T(32) : w / T(31);
            if (fine)
                dt = dt / T(16);
            sec.put(dgmr::Section<T> { c - w, c + w, dt });
            if (rng() % 3 == 0 || k == n_put - 1) {
                T a[128], b[128];
                dgmr::sample_positions_n<128>(sec, a);
                dgmr::sample_positions_by_sections<128>(sec, b);
                ++n_sets;
                bad += std::memcmp(a, b, sizeof a) == 0 ? 0 : 1;
            }
        }
    }
    *sets = n_sets;
    return bad;
}

} // namespace

extern "C" long kat_samples_by_sections_f32(unsigned seed, int trials, long* sets) { return check_samples_by_sections<float>(seed, trials, sets); }
extern "C" long kat_samples_by_sections_f64(unsigned seed, int trials, long* sets) { return check_samples_by_sections<double>(seed, trials, sets); }

extern "C" long kat_section_by_pieces_f32(unsigned seed, int trials, long* merges)
{
    long m1 = 0, m2 = 0;
    const long bad = check_by_pieces<float, 16>(seed, trials, &m1) + check_by_pieces<float, 4>(seed + 7, trials, &m2);
    *merges = m1 + m2;
    return bad;
}
extern "C" long kat_section_by_pieces_f64(unsigned seed, int trials, long* merges)
{
    long m1 = 0, m2 = 0;
    const long bad = check_by_pieces<double, 16>(seed, trials, &m1) + check_by_pieces<double, 4>(seed + 7, trials, &m2);
    *merges = m1 + m2;
    return bad;
}

extern "C" long kat_section_unchanged_f32(unsigned seed, int trials, long* covered) { return check_unchanged<float>(seed, trials, covered); }
extern "C" long kat_section_unchanged_f64(unsigned seed, int trials, long* covered) { return check_unchanged<double>(seed, trials, covered); }

// exp_f_nonpos against exp_f, bit for bit, on every float in [lo, hi] stepped
// by `stride` representable values, plus special values.  Returns mismatches.
extern "C" long kat_exp_nonpos_mismatches(float lo, float hi, unsigned stride)
{
    long bad = 0;
    const float special[] = { 0.0f, -0.0f, -87.0f, -87.5f, -88.0f, -104.0f, -1e30f, 1e-30f, 0.5f, 88.0f, 89.0f };
    for (float x : special) {
        const float a = dgmr_fm::exp_f(x), b = dgmr_fm::exp_f_nonpos(x);
        bad += std::memcmp(&a, &b, sizeof(float)) != 0;
    }
    for (float x = lo; x <= hi;) {
        const float a = dgmr_fm::exp_f(x), b = dgmr_fm::exp_f_nonpos(x);
        bad += std::memcmp(&a, &b, sizeof(float)) != 0;
        uint32_t u;
        std::memcpy(&u, &x, sizeof(u));
        u = (x < 0.0f) ? (u >= stride ? u - stride : 0u) : u + stride; // toward +inf by stride ulps
        if (x < 0.0f && u == 0u)
            u = 0u;
        std::memcpy(&x, &u, sizeof(u));
    }
    return bad;
}

// The product's exp / log / erf (csrc/dgmr_fmath.h) against the oracle's own
// coding of the same methods (oracle/dgmr_oracle_fmath.h): every float bit
// pattern u = first, first + stride, ... below 2^32 (both signs, every
// exponent, NaNs and infinities included), plus every pattern of [lo, hi]
// exhaustively.  which: 0 exp, 1 log, 2 erf.  Returns the count of inputs
// whose results differ in any bit (NaN payloads aside); *checked = inputs seen.
extern "C" long kat_fmath_mismatches(int which, unsigned first, unsigned stride, float lo, float hi, long* checked)
{
    auto same = [](float a, float b) {
        if (a != a && b != b)
            return true;
        return std::memcmp(&a, &b, sizeof(float)) == 0;
    };
    auto eval = [which](float x, float* a, float* b) {
        switch (which) {
        case 0:
            *a = dgmr_fm::exp_f(x);
            *b = ofm_rs::exp_f(x);
            break;
        case 1:
            *a = dgmr_fm::log_f(x);
            *b = ofm_rs::log_f(x);
            break;
        default:
            *a = dgmr_fm::erf_f(x);
            *b = ofm_rs::erf_f(x);
            break;
        }
    };
    long bad = 0, n = 0;
    for (uint64_t u = first; u < (uint64_t(1) << 32); u += stride) {
        const uint32_t w = uint32_t(u);
        float x, a, b;
        std::memcpy(&x, &w, sizeof(x));
        eval(x, &a, &b);
        bad += !same(a, b);
        ++n;
    }
    if (lo <= hi) {
        for (float x = lo;;) {
            float a, b;
            eval(x, &a, &b);
            bad += !same(a, b);
            ++n;
            if (x >= hi)
                break;
            x = std::nextafter(x, hi);
        }
    }
    *checked = n;
    return bad;
}

// dgmr_fm::recip_hastings against the correctly rounded 1.0f / d for every
// float d in [lo, hi]; returns the count that differ in any bit, *checked the
// inputs seen.
extern "C" long kat_recip_mismatches(float lo, float hi, long* checked)
{
    long bad = 0, n = 0;
    for (float d = lo; d <= hi; d = std::nextafter(d, 2.0f * hi)) {
        const float a = 1.0f / d, b = dgmr_fm::recip_hastings(d);
        bad += std::memcmp(&a, &b, sizeof(float)) != 0;
        ++n;
    }
    *checked = n;
    return bad;
}

// Random insertion sequences into a set sitting in front of a guard region:
// returns how many insertions left more than 16 sections or wrote past the
// set.  (The marcher keeps one set per warp in shared memory, next to other
// warps' data.)
extern "C" long kat_section_overflows(unsigned seed, int trials)
{
    struct Guarded {
        dgmr::SectionSet<16, float> s;
        float guard[64];
    };
    std::mt19937 rng(seed);
    long bad = 0;
    for (int trial = 0; trial < trials; ++trial) {
        Guarded g;
        for (float& x : g.guard)
            x = 12345.f;
        g.s.reset(float(rng() % 3) * 0.5f);
        const int n_put = 5 + int(rng() % 80);
        for (int k = 0; k < n_put; ++k) {
            float c = std::uniform_real_distribution<float>(0.f, 10.f)(rng);
            float w = 0.02f + std::uniform_real_distribution<float>(0.f, 2.f)(rng);
            if (rng() % 2) {
                c = float(int(c * 4)) / 4;
                w = float(1 + rng() % 8) / 4;
            }
            const float dt = (rng() % 3 == 0) ? float(1 + rng() % 4) / 32 : w / 31.f;
            g.s.put({ c - w, c + w, dt });
            bool hit = g.s.n > 16;
            for (float x : g.guard)
                hit = hit || x != 12345.f;
            if (hit) {
                ++bad;
                break;
            }
        }
    }
    return bad;
}

// The volume rasteriser's warp-parallel bin sizer (csrc/dgmr_raster_warp.cuh),
// its lanes emulated as arrays: the insertion position from the "not greater"
// ballot (highest set lane + 1), the shift, the left-to-right transmittance
// product, the lane-parallel merge costs and the first-of-equals minimum --
// against RasterBinSizer<32> on random add sequences; counts sequences whose
// saturation flags or final borders differ in any bit.
namespace {

struct WarpSizerEmu {
    float mass[32], border[32], sd[32];
    float total = 0.f, far = 0.f, full_mass = 0.f;

    void init(float transmission_threshold)
    {
        for (int i = 0; i < 32; ++i) {
            mass[i] = 0.f;
            border[i] = 1.f / 0.f;
            sd[i] = 0.f;
        }
        full_mass = -dgmr_fm::log_f(transmission_threshold);
    }

    void add(float m, float centre, float s, float sigma)
    {
        if (m < 0.0001f)
            return;
        const float reach = centre + s * sigma;
        const float on_ray = m * (dgmr::RasterBinSizer<32>::cdf(centre, s, reach) - dgmr::RasterBinSizer<32>::cdf(centre, s, 0.f));
        far = dgmr_fm::max_f(reach, far);
        total = total + on_ray;
        uint32_t not_greater = 0;
        for (int l = 0; l < 31; ++l)
            if (!(border[l] > centre))
                not_greater |= 1u << l;
        int p = 0;
        for (int l = 31; l >= 0; --l)
            if (not_greater >> l & 1u) {
                p = l + 1;
                break;
            }
        for (int l = 31; l > p; --l) {
            mass[l] = mass[l - 1];
            border[l] = border[l - 1];
            sd[l] = sd[l - 1];
        }
        mass[p] = on_ray;
        border[p] = centre;
        sd[p] = s;
        if (!(mass[31] > 0.f))
            return;
        float front[32];
        float run = 1.f;
        front[0] = 1.f;
        for (int i = 0; i < 31; ++i) {
            run = run * dgmr_fm::exp_f(-mass[i]);
            front[i + 1] = run;
        }
        float key[31], mm[31], mc[31], msd[31];
        for (int j = 0; j < 31; ++j) {
            const float sa = front[j] * mass[j], sb = front[j + 1] * mass[j + 1];
            const float pa = (sa + sb >= 0.0000001f) ? dgmr_fm::min_f(sa / (sa + sb), 0.999999f) : 0.5f;
            const float pb = 1.f - pa;
            const float c = pa * border[j] + pb * border[j + 1];
            const float va = sd[j] * sd[j], vb = sd[j + 1] * sd[j + 1];
            const float v = pa * (va + (border[j] - c) * (border[j] - c)) + pb * (vb + (border[j + 1] - c) * (border[j + 1] - c));
            mm[j] = mass[j] + mass[j + 1];
            mc[j] = c;
            msd[j] = dgmr_fm::sqrt_f(v);
            const auto kl = [](float c1, float sd1, float c2, float sd2) {
                return ((c1 - c2) * (c1 - c2) + sd1 * sd1 - sd2 * sd2) / (2.f * sd2 * sd2) + dgmr_fm::log_f(sd2 / sd1);
            };
            const float cost = front[j + 1] * (kl(border[j], sd[j], c, msd[j]) + kl(border[j + 1], sd[j + 1], c, msd[j]));
            key[j] = cost < 1.f / 0.f ? cost : 1.f / 0.f;
        }
        float lo = 1.f / 0.f;
        for (int j = 0; j < 31; ++j)
            lo = std::fmin(lo, key[j]);
        if (!(lo < 1.f / 0.f))
            return;
        int pick = 0;
        while (!(key[pick] == lo))
            ++pick;
        mass[pick] = mm[pick];
        border[pick] = mc[pick];
        sd[pick] = msd[pick];
        for (int l = pick + 1; l < 31; ++l) {
            mass[l] = mass[l + 1];
            border[l] = border[l + 1];
            sd[l] = sd[l + 1];
        }
    }

    void finalise()
    {
        float prev = 0.f;
        for (int i = 0; i < 32; ++i) {
            float b = border[i];
            const bool empty = b == 1.f / 0.f;
            if (!empty)
                b = dgmr_fm::max_f(b, prev + 0.00001f);
            else
                b = prev + (far - prev) / float(32 - i);
            prev = b;
            border[i] = b;
            if (empty)
                mass[i] = 0.f;
        }
    }
};

} // namespace

extern "C" long kat_compare_warp_sizer(unsigned seed, int trials)
{
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> u(0.f, 1.f);
    long bad = 0;
    for (int t = 0; t < trials; ++t) {
        dgmr::RasterBinSizer<32> a;
        WarpSizerEmu w;
        a.init(3.f, 0.005f);
        w.init(0.005f);
        const int n = 1 + int(u(rng) * 90.f);
        bool ok = true;
        float prev_centre = 2.f;
        for (int i = 0; i < n && ok; ++i) {
            const float mass = u(rng) < 0.1f ? 0.00005f : 0.0002f + 0.6f * u(rng) * u(rng);
            const float centre = u(rng) < 0.1f ? prev_centre : 2.f + 3.f * u(rng);
            prev_centre = centre;
            const float sd = 0.005f + 0.1f * u(rng);
            a.add_gaussian(mass, centre, sd);
            w.add(mass, centre, sd, 3.f);
            ok = a.is_full() == (w.total >= w.full_mass);
        }
        a.finalise();
        w.finalise();
        for (unsigned i = 0; i < 32 && ok; ++i) {
            const float e = i == 31 ? w.far : w.border[i];
            ok = same_bits(a.end_of(i), e);
        }
        bad += ok ? 0 : 1;
    }
    return bad;
}
