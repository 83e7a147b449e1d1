// Volume rasteriser with one warp per ray (included by dgmr_raster.cu).
//
// A ray has 32 depth bins and a warp has 32 lanes: lane q owns bin q.
//  * Pass A: the bin sizer's 32 slots live one per lane (mass, border, sd).
//    The tile list is walked 32 entries at a time (ray intersection, gates
//    and the added mass computed lane-parallel), then the qualifying entries
//    are added in list order: the insertion position is one ballot (the
//    first slot from the right whose border is not greater), the shift one
//    shuffle; once every slot holds mass, lane j prices merging slots j and
//    j+1 and a warp minimum picks the cheapest (the first of equals).
//    The transmittance in front of each slot is the same left-to-right
//    product as the one-thread sizer's, so every merge decision matches it.
//  * Pass B: for each Gaussian of the tile, lane q evaluates the CDF at its
//    bin's right border (the left one is its neighbour's) and accumulates its
//    bin's four masses and border values in registers -- per bin the same
//    Gaussian order and operations as the one-thread loop.
//  * Blend: lane q fits its bin and integrates its 256 steps from T = 1; the
//    bins' colours and transmittances are then chained in bin order.
// The one-thread-per-pixel kernel this replaces kept ~1 KB of bins and the
// sizer per thread (local memory) and ran 32 x 256 integration steps on one
// lane.  Warps are independent (no block barrier); rays outside the frame
// leave at once.
#pragma once

namespace dgmr {

constexpr unsigned kVrRayWarps = 4; // rays per block

// eval_exponential_1d as a call: the warp kernel is large enough to stall on
// instruction fetch with every exp inlined (same arithmetic, same bits)
__device__ __noinline__ float eval_exponential_1d_call(float c, float var, float x) { return eval_exponential_1d(c, var, x); }

struct RayEntryVr {
    uint32_t id;
    V3<float> mu;
    S3<float> Q;
    float mass;
};

// the sizer's slot held by this lane, and the ray-wide totals
struct WarpBinSizer {
    float mass, border, sd;
    float total, far, full_mass, sigma;
};

__device__ __forceinline__ void wbs_init(WarpBinSizer& s, float sigma, float transmission_threshold)
{
    s.mass = 0.f;
    s.border = 1.f / 0.f;
    s.sd = 0.f;
    s.total = 0.f;
    s.far = 0.f;
    s.sigma = sigma;
    s.full_mass = -dgmr_fm::log_f(transmission_threshold);
}

__device__ __forceinline__ float wbs_kl(float c1, float sd1, float c2, float sd2)
{
    return ((c1 - c2) * (c1 - c2) + sd1 * sd1 - sd2 * sd2) / (2.f * sd2 * sd2) + dgmr_fm::log_f(sd2 / sd1);
}

// RasterBinSizer::add_gaussian with the slots spread over the lanes; the
// arguments are the same on every lane (on_ray and reach precomputed by the
// entry's lane with RasterBinSizer's own cdf)
__device__ __forceinline__ void wbs_add(WarpBinSizer& s, unsigned lane, float mass, float centre, float sd, float on_ray, float reach)
{
    constexpr unsigned kFull = 0xffffffffu;
    if (mass < 0.0001f)
        return;
    s.far = max_f(reach, s.far);
    s.total = s.total + on_ray;
    // the new lobe enters the spare last slot and moves left past every border
    // strictly greater than its centre: it stops after the first slot (from
    // the right) that is not greater
    const unsigned not_greater = __ballot_sync(kFull, lane < kVrBins - 1 && !(s.border > centre));
    const unsigned p = not_greater ? 32u - unsigned(__clz(int(not_greater))) : 0u;
    const float um = __shfl_up_sync(kFull, s.mass, 1), ub = __shfl_up_sync(kFull, s.border, 1), us = __shfl_up_sync(kFull, s.sd, 1);
    if (lane > p) {
        s.mass = um;
        s.border = ub;
        s.sd = us;
    } else if (lane == p) {
        s.mass = on_ray;
        s.border = centre;
        s.sd = sd;
    }
    if (!(__shfl_sync(kFull, s.mass, kVrBins - 1) > 0.f))
        return;
    // transmittance in front of each slot: the one-thread sizer's left-to-right product
    const float ex = dgmr_fm::exp_f(-s.mass);
    float run = 1.f, front = 1.f;
#pragma unroll 1
    for (unsigned i = 0; i + 1 < kVrBins; ++i) {
        run = run * __shfl_sync(kFull, ex, int(i));
        if (lane == i + 1)
            front = run;
    }
    // lane j < 31: the merge of slots j and j + 1 and its cost
    const float nm = __shfl_down_sync(kFull, s.mass, 1), nb = __shfl_down_sync(kFull, s.border, 1), nsd = __shfl_down_sync(kFull, s.sd, 1);
    const float nfront = __shfl_down_sync(kFull, front, 1);
    const float sa = front * s.mass, sb = nfront * nm;
    const float pa = (sa + sb >= 0.0000001f) ? min_f(sa / (sa + sb), 0.999999f) : 0.5f;
    const float pb = 1.f - pa;
    const float c = pa * s.border + pb * nb;
    const float va = s.sd * s.sd, vb = nsd * nsd;
    const float v = pa * (va + (s.border - c) * (s.border - c)) + pb * (vb + (nb - c) * (nb - c));
    const float m_mass = s.mass + nm, m_sd = dgmr_fm::sqrt_f(v);
    const float cost = nfront * (wbs_kl(s.border, s.sd, c, m_sd) + wbs_kl(nb, nsd, c, m_sd));
    // the one-thread loop keeps the first index of the smallest cost below +inf
    const float key = (lane < kVrBins - 1 && cost < 1.f / 0.f) ? cost : 1.f / 0.f;
    float lo = key;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1)
        lo = fminf(lo, __shfl_xor_sync(kFull, lo, o));
    if (!(lo < 1.f / 0.f))
        return;
    const unsigned pick = unsigned(__ffs(int(__ballot_sync(kFull, key == lo))) - 1);
    // the merged lobe takes slot pick, the slots behind it move one left, the last stays
    if (lane == pick) {
        s.mass = m_mass;
        s.border = c;
        s.sd = m_sd;
    } else if (lane > pick && lane + 1 < kVrBins) {
        s.mass = nm;
        s.border = nb;
        s.sd = nsd;
    }
}

// RasterBinSizer::finalise: monotone borders, empty slots spread to the far end
__device__ __forceinline__ void wbs_finalise(WarpBinSizer& s, unsigned lane)
{
    float prev = 0.f;
#pragma unroll 1
    for (unsigned i = 0; i < kVrBins; ++i) {
        float b = __shfl_sync(0xffffffffu, s.border, int(i));
        const bool empty = b == 1.f / 0.f;
        if (!empty)
            b = max_f(b, prev + 0.00001f);
        else
            b = prev + (s.far - prev) / float(kVrBins - i);
        prev = b;
        if (lane == i) {
            s.border = b;
            if (empty)
                s.mass = 0.f;
        }
    }
}

__device__ __forceinline__ RayEntryVr load_vr_entry(const VrRender& a, int32_t k)
{
    RayEntryVr en;
    uint32_t id = a.list[k];
    if (id >= a.N) {
        flag_bounds(a.stats, 0x41u);
        id = 0;
    }
    en.id = id;
    en.mu = { a.centroids[3 * size_t(id)], a.centroids[3 * size_t(id) + 1], a.centroids[3 * size_t(id) + 2] };
#pragma unroll
    for (int c = 0; c < 6; ++c)
        en.Q.v[c] = a.inv_cov[6 * size_t(id) + c];
    en.mass = a.masses[id];
    return en;
}

// vol_raster_forward.cu:253-517, one warp per ray
__global__ void __launch_bounds__(kVrRayWarps * 32) k_vr_render_warp(VrRender a, CameraT<float> cam)
{
    constexpr unsigned kFull = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned per_tile = kTilePixels / kVrRayWarps;
    const unsigned tile = blockIdx.x / per_tile;
    const unsigned pix_in_tile = (blockIdx.x % per_tile) * kVrRayWarps + (threadIdx.x >> 5);
    const unsigned tx = tile % cam.gx, ty = tile / cam.gx;
    const unsigned px = tx * kTile + (pix_in_tile % kTile), py = ty * kTile + (pix_in_tile / kTile);
    if (px >= cam.W || py >= cam.H)
        return; // the whole warp
    const V3<float> o = { cam.campos[0], cam.campos[1], cam.campos[2] };
    const V3<float> d = vr_pixel_dir(cam, px, py);
    int32_t b = a.ranges[2 * tile], e = a.ranges[2 * tile + 1];
    if (b < 0 || e < b || uint32_t(e) > a.cap) {
        if (lane == 0)
            flag_bounds(a.stats, 0x42u);
        b = e = 0;
    }
    // pass A: bin sizes, until the ray's mass is used up
    WarpBinSizer sz;
    wbs_init(sz, kVrRelevanceSigma, kVrTransmission);
    bool full = false;
    for (int32_t base = b; base < e && !full; base += 32) {
        float mor = 0.f, centre = 0.f, sd = 0.f, on_ray = 0.f, reach = 0.f;
        bool ok = false;
        if (base + int32_t(lane) < e) {
            const RayEntryVr en = load_vr_entry(a, base + int32_t(lane));
            const Gauss1d<float> g = intersect_with_ray_inv_C(en.mu, en.Q, o, d);
            mor = g.weight * en.mass;
            ok = !(mor < 0.001f || mor > 1000.f) && !(g.C + 0.f <= 0.f);
            if (ok) {
                centre = g.centre;
                sd = dgmr_fm::sqrt_f(g.C + 0.f);
                reach = centre + sd * kVrRelevanceSigma;
                on_ray = mor * (RasterBinSizer<kVrBins>::cdf(centre, sd, reach) - RasterBinSizer<kVrBins>::cdf(centre, sd, 0.f));
            }
        }
        uint32_t m = __ballot_sync(kFull, ok);
        while (m) {
            const int j = __ffs(int(m)) - 1;
            m &= m - 1u;
            wbs_add(sz, lane, __shfl_sync(kFull, mor, j), __shfl_sync(kFull, centre, j), __shfl_sync(kFull, sd, j), __shfl_sync(kFull, on_ray, j),
                __shfl_sync(kFull, reach, j));
            if (sz.total >= sz.full_mass) {
                full = true;
                break;
            }
        }
    }
    wbs_finalise(sz, lane);
    // this lane's bin: [begin, end)
    const float end = lane == kVrBins - 1 ? sz.far : sz.border;
    const float begin_up = __shfl_up_sync(kFull, end, 1);
    const float begin = lane == 0 ? 0.f : begin_up;
    float res0 = 0.f, res1 = 0.f, res2 = 0.f, transparency = 1.f; // the final colour adds T = 1 x background in Full and Bins mode
    if (a.mode == DGMR_RENDER_FULL) {
        // pass B: bin masses and border values of every Gaussian of the tile
        float bm[4] = { 0.f, 0.f, 0.f, 0.f }, be[4] = { 0.f, 0.f, 0.f, 0.f }, be_last[4] = { 0.f, 0.f, 0.f, 0.f };
        const float max_distance = sz.far;
        for (int32_t base = b; base < e; base += 32) {
            float centre = 0.f, inv_sd = 0.f, variance = 0.f, weight = 0.f;
            V3<float> rgb = { 0.f, 0.f, 0.f };
            bool ok = false;
            if (base + int32_t(lane) < e) {
                const RayEntryVr en = load_vr_entry(a, base + int32_t(lane));
                const Gauss1d<float> g = intersect_with_ray_inv_C(en.mu, en.Q, o, d);
                centre = g.centre;
                variance = g.C + 0.f;
                const float sd = dgmr_fm::sqrt_f(variance);
                inv_sd = 1.f / sd;
                weight = g.weight * en.mass;
                ok = !(variance <= 0.f || dgmr_fm::isnan_f(variance) || dgmr_fm::isnan_f(weight) || weight > 100000.f)
                    && !(weight * (cdf_inv_SD_inline(centre, inv_sd, max_distance) - cdf_inv_SD_inline(centre, inv_sd, 0.f)) <= 0.001f);
                if (ok)
                    rgb = { a.rgb[3 * size_t(en.id)], a.rgb[3 * size_t(en.id) + 1], a.rgb[3 * size_t(en.id) + 2] };
            }
            uint32_t m = __ballot_sync(kFull, ok);
            while (m) {
                const int j = __ffs(int(m)) - 1;
                m &= m - 1u;
                const float cj = __shfl_sync(kFull, centre, j), ij = __shfl_sync(kFull, inv_sd, j);
                const float vj = __shfl_sync(kFull, variance, j), wj = __shfl_sync(kFull, weight, j);
                const float r = __shfl_sync(kFull, rgb.x, j), gg = __shfl_sync(kFull, rgb.y, j), bb = __shfl_sync(kFull, rgb.z, j);
                const float cdf_end = cdf_inv_SD(cj, ij, end);
                const float cdf_left = __shfl_up_sync(kFull, cdf_end, 1);
                const float cdf_start = lane == 0 ? cdf_inv_SD(cj, ij, 0.f) : cdf_left;
                const float mass = (cdf_end - cdf_start) * wj;
                if (!(mass < 0.0001f)) {
                    bm[0] = bm[0] + r * mass;
                    bm[1] = bm[1] + gg * mass;
                    bm[2] = bm[2] + bb * mass;
                    bm[3] = bm[3] + mass;
                    const float ev = wj * eval_exponential_1d_call(cj, vj, begin);
                    be[0] = be[0] + r * ev;
                    be[1] = be[1] + gg * ev;
                    be[2] = be[2] + bb * ev;
                    be[3] = be[3] + ev;
                }
                if (lane == kVrBins - 1) {
                    const float ev = wj * eval_exponential_1d_call(cj, vj, max_distance);
                    be_last[0] = be_last[0] + r * ev;
                    be_last[1] = be_last[1] + gg * ev;
                    be_last[2] = be_last[2] + bb * ev;
                    be_last[3] = be_last[3] + ev;
                }
            }
        }
        // blend: lane q fits bin q (the split of a bin's mass between its halves is
        // 0.5 for every bin and channel, vol_raster_forward.cu:473) and integrates
        // it from T = 1; then the bins are chained in order
        float right[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float nxt = __shfl_down_sync(kFull, be[c], 1);
            right[c] = lane == kVrBins - 1 ? be_last[c] : nxt;
        }
        const float t_right = end - begin;
        float l0 = 0.f, l1 = 0.f, l2 = 0.f, cur = 1.f;
        if (t_right > 0.f) {
            const float half[4] = { 0.5f, 0.5f, 0.5f, 0.5f };
            const FunctionGroup<float> f = create_approximation(half, bm, be, right, t_right);
            const float dt = f.t_right / float(kVrStepsPerBin);
            float t = dt / 2.f;
            for (unsigned s = 0; s < kVrStepsPerBin; ++s) {
                const float e0 = f.sample(0, t), e1 = f.sample(1, t), e2 = f.sample(2, t), e3 = f.sample(3, t);
                l0 = l0 + (e0 * cur) * dt;
                l1 = l1 + (e1 * cur) * dt;
                l2 = l2 + (e2 * cur) * dt;
                cur = cur * max_f(0.f, 1.f - e3 * dt);
                t = t + dt;
            }
        }
        float tr = 1.f;
#pragma unroll 1
        for (unsigned q = 0; q < kVrBins; ++q) {
            res0 = res0 + tr * __shfl_sync(kFull, l0, int(q));
            res1 = res1 + tr * __shfl_sync(kFull, l1, int(q));
            res2 = res2 + tr * __shfl_sync(kFull, l2, int(q));
            tr = tr * __shfl_sync(kFull, cur, int(q));
        }
    } else if (a.mode == DGMR_RENDER_DEPTH) {
        // vol_raster_forward.cu:495-507
        const unsigned bin = min(unsigned(a.debug_bin), kVrBins - 1);
        const float distance = __shfl_sync(kFull, end, int(bin));
        float c0 = distance / a.max_depth, c1 = c0, c2 = c0;
        if (distance == 0.f) {
            c0 = 0.f;
            c1 = 1.f;
            c2 = 0.f;
        }
        if (dgmr_fm::isnan_f(distance)) {
            c0 = 1.f;
            c1 = 0.f;
            c2 = 0.5f;
        }
        if (distance < 0.f) {
            c0 = 1.f;
            c1 = 0.5f;
            c2 = 0.f;
        }
        res0 = c0;
        res1 = c1;
        res2 = c2;
        transparency = 0.f;
    }
    if (lane == 0) {
        const size_t pix = size_t(py) * cam.W + px;
        const size_t plane = size_t(cam.W) * cam.H;
        a.fb[pix] = res0 + transparency * cam.bg[0];
        a.fb[plane + pix] = res1 + transparency * cam.bg[1];
        a.fb[2 * plane + pix] = res2 + transparency * cam.bg[2];
    }
}

} // namespace dgmr
