// TEST INFRASTRUCTURE ONLY -- the CPU oracle (see dgmr_oracle_math.h).
//
// Restatement of the marching-step sampler, src/dgmr/marching_steps.h:
//   DensityEntry / DensityArray   :28-200
//   sample<n_samples>             :202-220
// and of the volume-marcher bin helpers in src/dgmr/math.h:412-468 and their
// adjoints in src/dgmr/grad/math.h:529-620.
//
// DensityArray is a capacity-bounded, sorted set of non-overlapping sections
// {start, end, delta_t}.  Inserting a section that overlaps existing ones
// splits them and keeps the smaller delta_t on the overlap; when the set is
// full, sections that no longer fit are dropped and the array's end is pulled
// in.  The exact insertion steps (and therefore which sections survive
// truncation) are what the reference's known-answer tests pin, so the steps
// below follow the reference's put() one to one.
#pragma once

#include "dgmr_oracle_math.h"

namespace orc {

template <class T>
struct Section {
    T start, end, delta_t;
};

template <unsigned MAX, class T>
class DensityArray {
public:
    unsigned n = 0;
    Section<T> e[MAX];
    T lo;
    T hi;

    explicit DensityArray(T start)
        : lo(start)
        , hi(T(1) / T(0))
    {
    }
    unsigned size() const { return n; }
    T end() const { return hi; }
    const Section<T>& operator[](unsigned i) const { return e[i]; }

    // marching_steps.h:72-101: the three pieces [before | overlap | after]
    static void combine(const Section<T>& a, const Section<T>& b, Section<T> out[3])
    {
        if (a.start < b.start)
            out[0] = { a.start, min_f(a.end, b.start), a.delta_t };
        else
            out[0] = { b.start, min_f(b.end, a.start), b.delta_t };
        if (b.end < a.end)
            out[2] = { b.end, a.end, a.delta_t };
        else
            out[2] = { a.end, b.end, b.delta_t };
        out[1] = { out[0].end, out[2].start, min_f(a.delta_t, b.delta_t) };
    }

    // marching_steps.h:103-199
    void put(Section<T> s)
    {
        if (s.end <= lo)
            return;
        if (s.start >= hi)
            return;
        s.start = max_f(lo, s.start);
        s.end = min_f(hi, s.end);

        unsigned first = n;
        for (unsigned i = 0; i < n; ++i)
            if (e[i].end > s.start) {
                first = i;
                break;
            }
        if (first >= n) {
            if (first < MAX)
                e[n++] = s;
            else
                hi = s.start;
            return;
        }
        unsigned last = n;
        for (unsigned i = first; i < n; ++i)
            if (e[i].end > s.end) {
                last = i;
                break;
            }
        if (last < n && e[last].start < s.end)
            ++last;

        // in-place merge with a ring buffer holding entries displaced by growth
        Section<T> ring[MAX];
        unsigned r_read = 0, r_write = 0;
        unsigned i_read = first, i_write = first;
        unsigned grown = 0;
        while (i_read < last + grown && i_write < MAX) {
            if (i_read < n)
                ring[(r_write++) % MAX] = e[i_read++];
            if (r_read >= r_write)
                break;
            const Section<T>& head = ring[r_read % MAX];
            if (head.end <= s.start) {
                e[i_write++] = ring[(r_read++) % MAX];
                continue;
            }
            if (head.start >= s.end)
                break;
            Section<T> p[3];
            combine(ring[(r_read++) % MAX], s, p);
            if (p[0].delta_t == p[1].delta_t) { // compact: fold piece 0 into piece 1
                p[1].start = p[0].start;
                p[0].end = p[0].start;
            }
            s = p[2];
            if (p[0].end - p[0].start <= 0) {
                if (p[1].delta_t == p[2].delta_t) {
                    s.start = p[1].start;
                    continue;
                }
                e[i_write++] = p[1];
            } else {
                e[i_write++] = p[0];
                if (p[1].delta_t == p[2].delta_t) {
                    s.start = p[1].start;
                    continue;
                }
                ++grown;
                ring[(--r_read) % MAX] = p[1];
            }
        }
        if (s.end - s.start > 0 && i_write < MAX) {
            if (i_read < n)
                ring[(r_write++) % MAX] = e[i_read++];
            e[i_write++] = s;
        }
        while (r_write - r_read && i_write < MAX) {
            if (i_read < n)
                ring[(r_write++) % MAX] = e[i_read++];
            e[i_write++] = ring[(r_read++) % MAX];
        }
        n = i_write + n - i_read;
        if (n == MAX)
            hi = min_f(hi, e[n - 1].end);
    }
};

// marching_steps.h:202-220
template <unsigned NS, unsigned MAX, class T>
inline void sample(const DensityArray<MAX, T>& d, T out[NS])
{
    if (d.size() == 0) {
        for (unsigned i = 0; i < NS; ++i)
            out[i] = T(0);
        return;
    }
    out[0] = d[0].start;
    unsigned cur = 0;
    for (unsigned i = 1; i < NS; ++i) {
        const T v = min_f(d[cur].end, out[i - 1] + d[cur].delta_t);
        out[i] = v;
        if (cur < d.size() - 1 && v == d[cur].end)
            ++cur;
    }
}

template <class T>
struct Bin4 {
    T r, g, b, m; // colour mass, mass
};

// math.h:430-468
template <class T, unsigned NB>
inline void sample_gaussian(T mass, V3<T> rgb, V3<T> pos, const S3<T>& inv_cov, const Ray<T>& ray, const T* borders, Bin4<T>* bins)
{
    const Gauss1d<T> g = intersect_with_ray_inv_C(pos, inv_cov, ray);
    const T centre = g.centre;
    const T sd = ofm::sqrt_f(g.C);
    const T inv_sd = T(1) / sd;
    const T mass_on_ray = g.weight * mass;
    if (ofm::isnan_f(centre))
        return;
    if (mass_on_ray < T(1.0f / 255.f) || mass_on_ray > T(1000))
        return;
    if (sd <= T(0.0001) || ofm::isnan_f(sd) || ofm::isnan_f(mass_on_ray) || mass_on_ray > T(100000))
        return;
    const T mass_in_bins = mass_on_ray * integrate_normalised_inv_SD(centre, inv_sd, borders[0], borders[NB]);
    if (mass_in_bins < T(0.0001f))
        return;
    if (audit().on.load(std::memory_order_relaxed))
        audit().fills.fetch_add(1, std::memory_order_relaxed);
    T cdf_start = cdf_inv_SD(centre, inv_sd, borders[0]);
    for (unsigned k = 0; k < NB; ++k) {
        const T cdf_end = cdf_inv_SD(centre, inv_sd, borders[k + 1]);
        const T m = max_f(T(0), (cdf_end - cdf_start) * mass_on_ray);
        cdf_start = cdf_end;
        if (m < T(0.00001f))
            continue;
        bins[k].r = bins[k].r + rgb.x * m;
        bins[k].g = bins[k].g + rgb.y * m;
        bins[k].b = bins[k].b + rgb.z * m;
        bins[k].m = bins[k].m + m;
    }
}

// math.h:412-428
template <class T, unsigned NB>
inline void integrate_bins(V3<T>& colour, T& transparency, const Bin4<T>* bins)
{
    for (unsigned k = 0; k < NB; ++k) {
        const T tk = ofm::exp_f(-bins[k].m);
        colour.x = colour.x + bins[k].r * transparency;
        colour.y = colour.y + bins[k].g * transparency;
        colour.z = colour.z + bins[k].b * transparency;
        transparency = transparency * tk;
        if (transparency < T(1. / 255.))
            break;
    }
}

// grad/math.h:529-557: colour peeling, front to back
template <class T, unsigned NB>
inline void grad_integrate_bins(V3<T>& colour, T& transparency, T final_transparency, const Bin4<T>* bins, V3<T> g_colour, T g_transparency,
    Bin4<T>* g_bins)
{
    for (unsigned k = 0; k < NB; ++k)
        g_bins[k] = { T(0), T(0), T(0), T(0) };
    for (unsigned k = 0; k < NB; ++k) {
        g_bins[k].r = g_bins[k].r + transparency * g_colour.x;
        g_bins[k].g = g_bins[k].g + transparency * g_colour.y;
        g_bins[k].b = g_bins[k].b + transparency * g_colour.z;
        const T tk = ofm::exp_f(-bins[k].m);
        const T inv_tk = min_f(T(255), T(1) / tk);
        colour.x = (colour.x - bins[k].r) * inv_tk;
        colour.y = (colour.y - bins[k].g) * inv_tk;
        colour.z = (colour.z - bins[k].b) * inv_tk;
        const T g_tk = (final_transparency * inv_tk) * g_transparency + dot(g_colour, colour) * transparency;
        g_bins[k].m = g_bins[k].m - g_tk * tk;
        transparency = transparency * tk;
        if (transparency < T(1. / 255.))
            break;
    }
}

// d cdf_inv_SD / d(centre, inv_sd)
template <class T>
inline void grad_cdf_inv_SD(T c, T inv_sd, T x, T g, T* g_c, T* g_inv_sd)
{
    const T u = (x - c) * inv_sd;
    const T pdf = T(0.39894228040143267794) * ofm::exp_f(T(-0.5) * (u * u));
    *g_c = *g_c - g * inv_sd * pdf;
    *g_inv_sd = *g_inv_sd + g * (x - c) * pdf;
}

// Adjoint of intersect_with_ray_inv_C w.r.t. (mu, Q packed); derived from the
// closed form above.  Off-diagonal packed gradients count both matrix entries.
template <class T>
inline void grad_intersect_with_ray_inv_C(V3<T> mu, const S3<T>& Q, const Ray<T>& ray, T g_weight, T g_centre, T g_C, V3<T>* g_mu, S3<T>* g_Q)
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
    const T detQ = det_sym3(Q);
    const T r = detQ / a;
    const T sr = ofm::sqrt_f(r);
    const T weight = (sr * T(0.15915494309189533577)) * ofm::exp_f(T(-0.5) * e);

    const T g_e = g_weight * (T(-0.5) * weight);
    const T g_r = (r > T(0)) ? g_weight * weight / (T(2) * r) : T(0);
    const T inv_a = T(1) / a;
    const T inv_a2 = inv_a * inv_a;
    const T g_a = -g_C * inv_a2 - g_centre * b * inv_a2 + g_e * b * b * inv_a2 - g_r * detQ * inv_a2;
    const T g_b = g_centre * inv_a - g_e * T(2) * b * inv_a;
    const T g_k = g_e;
    const T g_det = g_r * inv_a;

    // d detQ / dQ = cofactor matrix (symmetric)
    const T q0 = Q.v[0], q1 = Q.v[1], q2 = Q.v[2], q3 = Q.v[3], q4 = Q.v[4], q5 = Q.v[5];
    const T cof[6] = { q3 * q5 - q4 * q4, q2 * q4 - q1 * q5, q1 * q4 - q2 * q3, q0 * q5 - q2 * q2, q1 * q2 - q0 * q4, q0 * q3 - q1 * q1 };
    const T dv[3] = { d.x, d.y, d.z };
    const T cv[3] = { c.x, c.y, c.z };
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            const int p = (i == 0) ? j : (i == 1 ? 2 + j : 5);
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

// grad/math.h:559-620
template <class T, unsigned NB>
inline void grad_sample_gaussian(T mass, V3<T> rgb, V3<T> pos, const S3<T>& inv_cov, const Ray<T>& ray, const T* borders, const Bin4<T>* g_bins,
    T* g_mass, V3<T>* g_rgb, V3<T>* g_pos, S3<T>* g_inv_cov)
{
    const Gauss1d<T> g = intersect_with_ray_inv_C(pos, inv_cov, ray);
    const T centre = g.centre;
    const T var = g.C;
    const T sd = ofm::sqrt_f(var);
    const T inv_sd = T(1) / sd;
    const T mass_on_ray = g.weight * mass;
    if (ofm::isnan_f(centre))
        return;
    if (mass_on_ray < T(1.0f / 255.f) || mass_on_ray > T(1000))
        return;
    if (sd <= T(0.0001) || ofm::isnan_f(sd) || ofm::isnan_f(mass_on_ray) || mass_on_ray > T(100000))
        return;
    const T mass_in_bins = mass_on_ray * integrate_normalised_inv_SD(centre, inv_sd, borders[0], borders[NB]);
    if (mass_in_bins < T(0.0001f))
        return;
    T g_centre = 0, g_inv_sd = 0, g_mor = 0;
    V3<T> grgb = { 0, 0, 0 };
    T cdf_start = cdf_inv_SD(centre, inv_sd, borders[0]);
    for (unsigned k = 0; k < NB; ++k) {
        const T cdf_end = cdf_inv_SD(centre, inv_sd, borders[k + 1]);
        const T delta = cdf_end - cdf_start;
        const T m = max_f(T(0), delta * mass_on_ray);
        cdf_start = cdf_end;
        if (m < T(0.00001f))
            continue;
        grgb.x = grgb.x + g_bins[k].r * m;
        grgb.y = grgb.y + g_bins[k].g * m;
        grgb.z = grgb.z + g_bins[k].b * m;
        const T g_m = ((g_bins[k].r * rgb.x + g_bins[k].g * rgb.y) + g_bins[k].b * rgb.z) + g_bins[k].m;
        if (delta * mass_on_ray <= T(0))
            continue;
        g_mor = g_mor + g_m * delta;
        const T g_delta = g_m * mass_on_ray;
        grad_cdf_inv_SD(centre, inv_sd, borders[k], -g_delta, &g_centre, &g_inv_sd);
        grad_cdf_inv_SD(centre, inv_sd, borders[k + 1], g_delta, &g_centre, &g_inv_sd);
    }
    const T g_w1d = g_mor * mass;
    *g_mass = *g_mass + g_mor * g.weight;
    const T g_sd = -g_inv_sd / (sd * sd);
    const T g_var = g_sd / (T(2) * sd);
    *g_rgb = add(*g_rgb, grgb);
    grad_intersect_with_ray_inv_C(pos, inv_cov, ray, g_w1d, g_centre, g_var, g_pos, g_inv_cov);
}

} // namespace orc
