// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle, never linked into the
// product.  The oracle's own restatement of the volume rasteriser's per-ray
// depth binning and piecewise-linear bin model, written independently of the
// product's device header so that the vol_raster parity test compares two
// separate codings of the reference's steps:
//   src/dgmr/raster_bin_sizers.h:271-485  (RasterBinSizer: online merging of
//                                          1-D Gaussians into depth bins)
//   src/dgmr/piecewise_linear.h:60-158    (create_approximation: the
//                                          four-channel fit of one bin)
// The float operations are those of the reference, in its order (which bins
// merge and where a bin's knots land are decided by them); the data layout
// and control structure are this file's own: a bin is a Lobe record, the
// sizer keeps its lobes sorted by centre, and a channel fit is a value type.
#pragma once

#include <cmath>

#include "dgmr_oracle_math.h"

namespace oracle_vf {

// One 1-D Gaussian along the ray: the mass it puts on [0, centre + sigma sd]
// (raster_bin_sizers.h:356-360), its centre and standard deviation.
struct Lobe {
    float mass;
    float centre;
    float sd;
};

inline float normal_cdf(float centre, float sd, float x)
{
    return 0.5f * (1.f + ofm::erf_f((x - centre) / (sd * 1.41421356237309505f)));
}

// KL divergence of N(c1, sd1) from N(c2, sd2) (raster_bin_sizers.h:409-411).
inline float kl_normal(float c1, float sd1, float c2, float sd2)
{
    const float num = (c1 - c2) * (c1 - c2) + sd1 * sd1 - sd2 * sd2;
    return num / (2.f * sd2 * sd2) + ofm::log_f(sd2 / sd1);
}

// N lobes sorted by centre; a new lobe takes the spare last place, sinks to
// its sorted position, and once all N places hold mass the adjacent pair
// whose moment-matched merge is cheapest (KL of both halves to the merged
// lobe, weighted by the transmittance in front of the pair) becomes one lobe.
template <unsigned N>
class DepthBins {
public:
    void reset(float relevance_sigma, float transmission_threshold)
    {
        sigma_ = relevance_sigma;
        full_mass_ = -ofm::log_f(transmission_threshold);
        for (Lobe& l : lobe_)
            l = Lobe { 0.f, 1.f / 0.f, 0.f };
        total_ = 0.f;
        far_ = 0.f;
    }

    bool saturated() const { return total_ >= full_mass_; }

    // bin i covers [lower(i), upper(i)) after close()
    float upper(unsigned i) const { return i + 1 == N ? far_ : lobe_[i].centre; }
    float lower(unsigned i) const { return i == 0 ? 0.f : upper(i - 1); }

    void add(float mass, float centre, float sd)
    {
        if (mass < 0.0001f)
            return;
        const float reach = centre + sd * sigma_;
        const float on_ray = mass * (normal_cdf(centre, sd, reach) - normal_cdf(centre, sd, 0.f));
        far_ = reach < far_ ? far_ : reach;
        total_ = total_ + on_ray;

        unsigned at = N - 1;
        lobe_[at] = Lobe { on_ray, centre, sd };
        while (at > 0 && lobe_[at - 1].centre > lobe_[at].centre) {
            const Lobe t = lobe_[at - 1];
            lobe_[at - 1] = lobe_[at];
            lobe_[at] = t;
            --at;
        }
        if (!(lobe_[N - 1].mass > 0.f))
            return;

        // in_front[i] = transmittance in front of lobe i
        float in_front[N];
        in_front[0] = 1.f;
        float running = 1.f;
        for (unsigned i = 0; i + 1 < N; ++i) {
            running = running * ofm::exp_f(-lobe_[i].mass);
            in_front[i + 1] = running;
        }
        unsigned pick = 0;
        float pick_cost = 1.f / 0.f;
        bool found = false;
        for (unsigned j = 0; j + 1 < N; ++j) {
            const Lobe m = merged(j, in_front);
            const float cost = in_front[j + 1]
                * (kl_normal(lobe_[j].centre, lobe_[j].sd, m.centre, m.sd) + kl_normal(lobe_[j + 1].centre, lobe_[j + 1].sd, m.centre, m.sd));
            if (cost < pick_cost) {
                pick_cost = cost;
                pick = j;
                found = true;
            }
        }
        if (!found)
            return;
        lobe_[pick] = merged(pick, in_front);
        for (unsigned j = pick + 1; j + 1 < N; ++j)
            lobe_[j] = lobe_[j + 1];
    }

    // Unused places get evenly spaced borders up to the far end and no mass;
    // used borders are made strictly increasing (raster_bin_sizers.h:469-483).
    void close()
    {
        float prev = 0.f;
        for (unsigned i = 0; i < N; ++i) {
            Lobe& l = lobe_[i];
            if (std::isinf(l.centre)) {
                l.centre = prev + (far_ - prev) / float(N - i);
                l.mass = 0.f;
            } else if (l.centre < prev + 0.00001f) {
                l.centre = prev + 0.00001f;
            }
            prev = l.centre;
        }
    }

private:
    // lobes a, a + 1 as one, by their transmittance-weighted shares
    Lobe merged(unsigned a, const float* in_front) const
    {
        const Lobe& p = lobe_[a];
        const Lobe& q = lobe_[a + 1];
        const float wp = in_front[a] * p.mass;
        const float wq = in_front[a + 1] * q.mass;
        float sp = 0.5f;
        if (wp + wq >= 0.0000001f) {
            sp = wp / (wp + wq);
            sp = 0.999999f < sp ? 0.999999f : sp;
        }
        const float sq = 1.f - sp;
        const float c = sp * p.centre + sq * q.centre;
        const float var = sp * (p.sd * p.sd + (p.centre - c) * (p.centre - c)) + sq * (q.sd * q.sd + (q.centre - c) * (q.centre - c));
        return Lobe { p.mass + q.mass, c, ofm::sqrt_f(var) };
    }

    Lobe lobe_[N];
    float sigma_ = 3.f;
    float full_mass_ = 0.f;
    float total_ = 0.f;
    float far_ = 0.f;
};

// One channel of one bin [0, width]: a line from the value at the left end
// down to the knot t1, zero up to t2, a line up to the value at the right end
// -- or, when the two lines would overlap, both lines meeting in one knot at
// a shared middle value.  Its integral equals the channel's mass, its ends the
// channel's values (piecewise_linear.h:60-158).
struct BinChannel {
    float d0 = 0.f, k0 = 0.f, t1 = 0.f, t2 = 0.f, k2 = 0.f;

    float at(float t) const
    {
        if (t <= t1)
            return d0 + k0 * t;
        if (t <= t2)
            return 0.f;
        return d0 + t1 * k0 + (t - t2) * k2;
    }
};

inline BinChannel fit_channel(float share_left, float mass, float at_left, float at_right, float width)
{
    BinChannel ch;
    if (mass <= 0.000001f) { // no mass in this channel: zero over the bin
        ch.t2 = width;
        return ch;
    }
    const float left = share_left * mass;
    const float right = mass - left;
    ch.d0 = at_left;
    ch.t1 = 2.f * left / at_left;
    ch.t2 = width - 2.f * right / at_right;
    if (ch.t2 > ch.t1) { // two separate triangles
        ch.k0 = -at_left * at_left / (2.f * left);
        ch.k2 = at_right * at_right / (2.f * right);
        return ch;
    }
    // one knot at the middle value dm: the mass constraint is a quadratic in dm
    const float a1 = 2.f * mass - (at_left + at_right) * width;
    const float a2 = at_right * left + at_left * right;
    const float a3 = at_left * at_right * width;
    float dm = (a1 + ofm::sqrt_f(a1 * a1 + 4.f * width * (2.f * a2 - a3))) / (2.f * width);
    dm = dm > 0.f ? dm : 0.f;
    float tl, tr;
    if (right > left) {
        tr = 2.f * right / (dm + at_right);
        tl = width - tr > 0.f ? width - tr : 0.f;
    } else {
        tl = 2.f * left / (dm + at_left);
        tr = width - tl > 0.f ? width - tl : 0.f;
    }
    ch.k0 = tl == 0.f ? 0.f : -(at_left - dm) / tl;
    ch.t1 = tl;
    ch.t2 = tl;
    ch.k2 = tr == 0.f ? 0.f : (at_right - dm) / tr;
    return ch;
}

} // namespace oracle_vf

namespace oracle_vf {

// Midpoint-rule emission-absorption over one bin of `width` (channels r, g,
// b, density), continuing the ray's colour and transmittance
// (piecewise_linear.h:160-181).
inline void integrate_bin(const BinChannel* ch, float width, unsigned steps, float* rgb, float& transmittance)
{
    const float dt = width / float(steps);
    float t = dt / 2.f;
    for (unsigned s = 0; s < steps; ++s) {
        const float r = ch[0].at(t), g = ch[1].at(t), b = ch[2].at(t), d = ch[3].at(t);
        rgb[0] = rgb[0] + (r * transmittance) * dt;
        rgb[1] = rgb[1] + (g * transmittance) * dt;
        rgb[2] = rgb[2] + (b * transmittance) * dt;
        const float keep = 1.f - d * dt;
        transmittance = transmittance * (0.f < keep ? keep : 0.f);
        t = t + dt;
    }
}

} // namespace oracle_vf
