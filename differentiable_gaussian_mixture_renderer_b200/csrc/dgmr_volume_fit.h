// Per-ray depth binning and piecewise-linear volume integration (host and
// device code), restating
//   src/dgmr/piecewise_linear.h:28-181  (FunctionGroup, create_approximation,
//                                         volume_integrate)
//   src/dgmr/raster_bin_sizers.h:271-485 (RasterBinSizer)
// Their only caller in the reference is the volume rasteriser
// (vol_raster_forward.cu:292-477), which bins each ray's Gaussians into
// depth bins and integrates colour and density over each bin with a
// four-channel piecewise-linear model.
#pragma once

#include "dgmr_fmath.h"

namespace dgmr {

// ---------------------------------------------------------------- piecewise linear

// Four channels (r, g, b, density) over one bin [0, t_right].  Channel i is
// d0 + k0 t on [0, t1], zero on (t1, t2], and rises again as
// d0 + t1 k0 + (t - t2) k2 after t2 (piecewise_linear.h:28-58).
template <class T>
struct FunctionGroup {
    T d0[4], k0[4], t1[4], t2[4], k2[4];
    T t_right;

    DGMR_HD T sample(int i, T t) const
    {
        if (t <= t1[i])
            return d0[i] + k0[i] * t;
        if (t <= t2[i])
            return T(0);
        const T tp = t - t2[i];
        return d0[i] + t1[i] * k0[i] + tp * k2[i];
    }

    // the invariants the reference asserts (non-negative start and end values, ordered knots)
    DGMR_HD bool valid() const
    {
        for (int i = 0; i < 4; ++i) {
            if (!(d0[i] >= T(0)) || !(t1[i] >= T(0)) || !(t2[i] >= t1[i]) || !(d0[i] + t1[i] * k0[i] >= T(0)))
                return false;
        }
        return true;
    }
};

// Fit of one bin (piecewise_linear.h:60-158): the channel's value at both ends
// and its mass are matched; a channel whose two straight lines would cross is
// given a shared middle value dm instead, from the quadratic of the mass
// constraint.  Channels with (almost) no mass are zero.
template <class T>
DGMR_HD FunctionGroup<T> create_approximation(const T* masses_percent_left, const T* masses_total, const T* eval_left, const T* eval_right, T t_right)
{
    FunctionGroup<T> f;
    f.t_right = t_right;
    for (int i = 0; i < 4; ++i) {
        const T m_l = masses_percent_left[i] * masses_total[i];
        const T m_r = masses_total[i] - m_l;
        f.d0[i] = eval_left[i];
        f.k0[i] = T(0);
        f.t1[i] = T(2) * m_l / eval_left[i];
        f.t2[i] = t_right - T(2) * m_r / eval_right[i];
        f.k2[i] = T(0);
        if (masses_total[i] <= T(0.000001)) {
            f.d0[i] = T(0);
            f.k0[i] = T(0);
            f.t1[i] = T(0);
            f.t2[i] = t_right;
            f.k2[i] = T(0);
            continue;
        }
        if (f.t2[i] > f.t1[i]) {
            f.k0[i] = -eval_left[i] * eval_left[i] / (T(2) * m_l);
            f.k2[i] = eval_right[i] * eval_right[i] / (T(2) * m_r);
            continue;
        }
        const T m = masses_total[i];
        const T gl = eval_left[i];
        const T gr = eval_right[i];
        const T tw = t_right; // the bin starts at t = 0
        const T c1 = T(2) * m - (gl + gr) * tw;
        const T c2 = gr * m_l + gl * m_r;
        const T c3 = gl * gr * tw;
        const T dm = dgmr_fm::max_f(T(0), (c1 + dgmr_fm::sqrt_f(c1 * c1 + T(4) * tw * (T(2) * c2 - c3))) / (T(2) * tw));
        T tl, tr;
        if (m_r > m_l) {
            tr = T(2) * m_r / (dm + gr);
            tl = dgmr_fm::max_f(T(0), tw - tr);
        } else {
            tl = T(2) * m_l / (dm + gl);
            tr = dgmr_fm::max_f(T(0), tw - tl);
        }
        f.k0[i] = (tl == T(0)) ? T(0) : -(gl - dm) / tl;
        f.t1[i] = tl;
        f.t2[i] = tl;
        f.k2[i] = (tr == T(0)) ? T(0) : (gr - dm) / tr;
    }
    return f;
}

// Midpoint-rule emission-absorption integral over consecutive bins
// (piecewise_linear.h:160-181); writes the rgb result.
template <class T>
DGMR_HD void volume_integrate(const FunctionGroup<T>* groups, unsigned n_groups, unsigned n_steps_per_bin, T* rgb_out)
{
    T r = T(0), g = T(0), b = T(0);
    T transparency = T(1);
    for (unsigned n = 0; n < n_groups; ++n) {
        const FunctionGroup<T>& f = groups[n];
        const T dt = f.t_right / T(n_steps_per_bin);
        T t = dt / T(2);
        for (unsigned s = 0; s < n_steps_per_bin; ++s) {
            const T v0 = f.sample(0, t), v1 = f.sample(1, t), v2 = f.sample(2, t), v3 = f.sample(3, t);
            r = r + v0 * transparency * dt;
            g = g + v1 * transparency * dt;
            b = b + v2 * transparency * dt;
            transparency = transparency * dgmr_fm::max_f(T(0), T(1) - v3 * dt);
            t = t + dt;
        }
    }
    rgb_out[0] = r;
    rgb_out[1] = g;
    rgb_out[2] = b;
}

// ---------------------------------------------------------------- depth bins

// Online sizing of N_BINS depth bins along one ray (raster_bin_sizers.h:271-485).
// Each added 1-D Gaussian (mass, centre, sd) goes into a spare last slot, is
// insertion-sorted by centre, and -- once every slot holds mass -- the
// neighbouring pair whose moment-matched merge costs the least
// (transmittance-weighted KL divergence) is merged, keeping N_BINS slots.
// finalise() turns the slot centres into monotone bin borders.
template <unsigned N_BINS>
struct RasterBinSizer {
    float relevance_sigma; // gaussians count up to centre + sigma * sd
    float mass_threshold; // -log(transmission threshold)
    float masses[N_BINS];
    float borders[N_BINS];
    float sds[N_BINS];
    float accumulated_mass;
    float max_depth;

    DGMR_HD void init(float sigma, float transmission_threshold)
    {
        relevance_sigma = sigma;
        mass_threshold = -dgmr_fm::log_f(transmission_threshold);
        for (unsigned i = 0; i < N_BINS; ++i) {
            masses[i] = 0.f;
            borders[i] = 1.f / 0.f;
            sds[i] = 0.f;
        }
        accumulated_mass = 0.f;
        max_depth = 0.f;
    }

    DGMR_HD float end_of(unsigned i) const { return i == N_BINS - 1 ? max_depth : borders[i]; }
    DGMR_HD float begin_of(unsigned i) const { return i == 0 ? 0.f : end_of(i - 1); }
    DGMR_HD bool is_full() const { return accumulated_mass >= mass_threshold; }

    DGMR_HD static float cdf(float centre, float sd, float x) { return 0.5f * (1.f + dgmr_fm::erf_f((x - centre) / (sd * 1.41421356237309505f))); }

    DGMR_HD void add_gaussian(float mass, float centre, float sd)
    {
        if (mass < 0.0001f)
            return;
        constexpr unsigned last = N_BINS - 1;
        const float t_rel = centre + sd * relevance_sigma;
        const float added = mass * (cdf(centre, sd, t_rel) - cdf(centre, sd, 0.f));
        max_depth = dgmr_fm::max_f(t_rel, max_depth);
        accumulated_mass = accumulated_mass + added;
        masses[last] = added;
        borders[last] = centre;
        sds[last] = sd;
        for (unsigned i = last; i > 0; --i) {
            if (borders[i - 1] > borders[i]) {
                swap(borders[i - 1], borders[i]);
                swap(sds[i - 1], sds[i]);
                swap(masses[i - 1], masses[i]);
                continue;
            }
            break;
        }
        // transmittance in front of each slot
        float trans[N_BINS];
        float tr = 1.f;
        for (unsigned i = 0; i < last; ++i) {
            tr = tr * dgmr_fm::exp_f(-masses[i]);
            trans[i] = tr;
        }
        const auto before = [&](int idx) { return idx <= 0 ? 1.f : trans[idx - 1]; };
        struct Merged {
            float mass, centre, sd;
        };
        const auto merge = [&](int a, int b) {
            const float sa = before(a) * masses[a];
            const float sb = before(b) * masses[b];
            const float pa = (sa + sb >= 0.0000001f) ? dgmr_fm::min_f(sa / (sa + sb), 0.999999f) : 0.5f;
            const float pb = 1.f - pa;
            const float c = pa * borders[a] + pb * borders[b];
            const float va = sds[a] * sds[a], vb = sds[b] * sds[b];
            const float v = pa * (va + (borders[a] - c) * (borders[a] - c)) + pb * (vb + (borders[b] - c) * (borders[b] - c));
            return Merged { masses[a] + masses[b], c, dgmr_fm::sqrt_f(v) };
        };
        const auto kl = [](float c1, float sd1, float c2, float sd2) {
            return ((c1 - c2) * (c1 - c2) + sd1 * sd1 - sd2 * sd2) / (2.f * sd2 * sd2) + dgmr_fm::log_f(sd2 / sd1);
        };
        if (masses[last] > 0.f) {
            int best = -1;
            float best_cost = 1.f / 0.f;
            for (int j = 0; j < int(last); ++j) {
                const Merged m = merge(j, j + 1);
                const float cost = before(j + 1) * (kl(borders[j], sds[j], m.centre, m.sd) + kl(borders[j + 1], sds[j + 1], m.centre, m.sd));
                if (cost < best_cost) {
                    best_cost = cost;
                    best = j;
                }
            }
            if (best >= 0) {
                const Merged m = merge(best, best + 1);
                borders[best] = m.centre;
                masses[best] = m.mass;
                sds[best] = m.sd;
                for (unsigned j = unsigned(best) + 1; j < last; ++j) {
                    borders[j] = borders[j + 1];
                    masses[j] = masses[j + 1];
                    sds[j] = sds[j + 1];
                }
            }
        }
    }

    DGMR_HD void finalise()
    {
        float prev = 0.f;
        for (unsigned i = 0; i < N_BINS; ++i) {
            float& b = borders[i];
            if (!(b == 1.f / 0.f)) {
                b = dgmr_fm::max_f(b, prev + 0.00001f);
                prev = b;
            } else {
                b = prev + (max_depth - prev) / float(N_BINS - i);
                prev = b;
                masses[i] = 0.f;
            }
        }
    }

private:
    DGMR_HD static void swap(float& a, float& b)
    {
        const float t = a;
        a = b;
        b = t;
    }
};

} // namespace dgmr
