// Volume march with one warp per ray (included by dgmr_marcher.cu).
//
// A ray's work is mostly its pass 2: for every Gaussian it can use, 127
// CDF differences -- and the heaviest rays of a frame set its duration.  With
// one thread per ray that work is a long dependent chain on one lane (with
// the 127 bins in local memory), so the kernel ends up waiting on a few
// rays while the SMs idle.  Here the 32 lanes of a warp share one ray:
//  * the tile list is walked 32 entries at a time, one entry per lane
//    (intersection with the ray, gates), results exchanged by shuffles;
//  * lane l owns bins l, l+32, l+64, l+96 (four register bins); for each
//    Gaussian, in list order, every lane evaluates the CDF at its own
//    borders and takes the next border's value from its neighbour;
//  * the strictly sequential parts -- section insertion (pass 1), sample
//    positions, the blend and its adjoint peel -- run on every lane in
//    lockstep from shared values, so no lane waits on another.
// Per bin, Gaussian order and every arithmetic operation are those of the
// one-thread loops (vol_marcher_forward.cu:295-501, math.h:412-468), so the
// image is the same bits.  Warps are independent (no block barrier); blocks
// of kRayWarps rays are launched heaviest tile first.
#pragma once

namespace dgmr {

constexpr unsigned kRayWarps = 4; // rays per block
constexpr unsigned kRayRounds = 4; // 4 x 32 lanes >= 128 borders
constexpr unsigned kRayMaskRegs = 4; // ray masks kept in registers: 4 x 32 batches of 32 entries

// A ray's section set lives in shared memory, once per warp: lane 0 inserts,
// every lane reads it after a __syncwarp (kept per lane, the 32 identical
// copies and the insertion's scratch went to local memory).
template <class T>
struct RayWarpShared {
    T borders[kSmallSteps];
    Bin<T> bins[kSmallSteps]; // forward: (r, g, b, exp(-mass)); backward: (r, g, b, mass)
    SectionSet<kLargeSteps, T> sec;
    Section<T> pieces[2 * kLargeSteps + 1]; // warp_put: the merged sections of one insertion
};

template <class T>
struct RayWarpSharedBwd {
    T borders[kSmallSteps];
    Bin<T> bins[kSmallSteps];
    Bin<T> gbins[kSmallSteps]; // bin adjoints
    int32_t queue[32]; // pass 3: list entries waiting for a lane
    SectionSet<kLargeSteps, T> sec;
    Section<T> pieces[2 * kLargeSteps + 1];
};

static_assert(kLargeSteps <= 16, "warp_put moves the kept sections on lanes 0-15 and writes pieces on lanes 16-31");

// The gates of both passes (see ray_can_use) as a 32-bit mask per batch of 32
// list entries, held in registers: lane l keeps the masks of batches l, l+32,
// l+64, l+96.  Batches past that get every entry (the gates are re-checked).
struct WarpRayMasks {
    uint32_t r[kRayMaskRegs];
    __device__ __forceinline__ uint32_t get(unsigned i) const
    {
        if (i >= 32 * kRayMaskRegs)
            return 0xffffffffu;
        const unsigned q = i >> 5;
        uint32_t v = r[0];
#pragma unroll
        for (unsigned k = 1; k < kRayMaskRegs; ++k)
            if (q == k)
                v = r[k];
        return __shfl_sync(0xffffffffu, v, int(i & 31u));
    }
    __device__ __forceinline__ void set(unsigned i, uint32_t m, unsigned lane)
    {
        if (i >= 32 * kRayMaskRegs || (i & 31u) != lane)
            return;
#pragma unroll
        for (unsigned k = 0; k < kRayMaskRegs; ++k)
            if ((i >> 5) == k)
                r[k] = m;
    }
};

__device__ __forceinline__ uint32_t lanes_below(int n) { return n >= 32 ? 0xffffffffu : ((1u << n) - 1u); }

// One list entry as seen by its lane.
template <class T>
struct RayEntry {
    uint32_t id;
    V3<T> mu;
    S3<T> Q;
    T mass;
};

template <class T>
__device__ __forceinline__ RayEntry<T> load_entry(const VmMarch<T>& a, int32_t k)
{
    RayEntry<T> en;
    en.id = uint32_t(a.list[k]);
    const size_t id = en.id;
    en.mu = { a.centroids[3 * id], a.centroids[3 * id + 1], a.centroids[3 * id + 2] };
#pragma unroll
    for (int c = 0; c < 6; ++c)
        en.Q.v[c] = a.inv_cov[6 * id + c];
    en.mass = a.masses[id];
    return en;
}

// The frames a march launch covers.  A single frame: one camera (a kernel
// parameter) and the image planes of VmMarch.  A batch (VmBatchFrames, float)
// looks each tile's view up in its view table; its tiles are numbered across
// views and its rays index one array of all views' pixels.
template <class T>
struct VmSingleFrame {
    CameraT<T> cam0;
    __device__ __forceinline__ unsigned view(unsigned) const { return 0u; }
    __device__ __forceinline__ const CameraT<T>& cam(unsigned) const { return cam0; }
    __device__ __forceinline__ unsigned tile_base(unsigned) const { return 0u; }
    __device__ __forceinline__ size_t px_base(unsigned) const { return 0; }
    __device__ __forceinline__ size_t rays() const { return size_t(cam0.W) * cam0.H; }
    __device__ __forceinline__ T* fb(unsigned, const VmMarch<T>& a) const { return a.fb; }
    __device__ __forceinline__ T* remaining_T(unsigned, const VmMarch<T>& a) const { return a.remaining_T; }
    __device__ __forceinline__ const T* grad_fb(unsigned, const VmMarch<T>& a) const { return a.grad_fb; }
};

// Tile work order for the march: heaviest tile first (k_tile_order), so the
// longest rays start at the head of the grid.  tile = the launch-wide tile
// (it indexes the ranges), view = its frame, (px, py) = the ray's pixel there.
template <class T, class Frames>
__device__ __forceinline__ bool ray_pixel(const Frames& frames, const uint32_t* order, unsigned* tile, unsigned* view, unsigned* px, unsigned* py)
{
    const unsigned groups = kTilePixels / kRayWarps;
    const unsigned item = blockIdx.x / groups, group = blockIdx.x % groups;
    *tile = order ? order[item] : item;
    *view = frames.view(*tile);
    const CameraT<T>& cam = frames.cam(*view);
    const unsigned lt = *tile - frames.tile_base(*view);
    const unsigned p = group * kRayWarps + (threadIdx.x >> 5);
    *px = (lt % cam.gx) * kTile + (p % kTile);
    *py = (lt / cam.gx) * kTile + (p / kTile);
    return *px < cam.W && *py < cam.H;
}

// pass 0: the ray's masks (one intersection per list entry, lane-parallel)
template <class T>
__device__ __forceinline__ WarpRayMasks warp_ray_masks(const VmMarch<T>& a, int32_t b, int32_t e, V3<T> o, V3<T> d, unsigned lane)
{
    WarpRayMasks rm;
#pragma unroll
    for (unsigned k = 0; k < kRayMaskRegs; ++k)
        rm.r[k] = 0u;
    unsigned i = 0;
    for (int32_t base = b; base < e && i < 32 * kRayMaskRegs; base += 32, ++i) {
        const int32_t k = base + int32_t(lane);
        bool can = false;
        if (k < e) {
            const RayEntry<T> en = load_entry(a, k);
            can = ray_can_use(intersect_with_ray_inv_C(en.mu, en.Q, o, d), en.mass);
        }
        rm.set(i, __ballot_sync(0xffffffffu, can), lane);
    }
    return rm;
}

} // namespace dgmr

namespace dgmr {

// SectionSet::put_leaves_unchanged (dgmr_sections.h) with lane i (< kLargeSteps)
// testing section i: whether inserting s would leave the warp's set exactly as
// it is, so that the insertion (and lane 0's serial walk) can be skipped.
template <class T>
__device__ __forceinline__ bool warp_section_covered(const SectionSet<kLargeSteps, T>& sec, const Section<T>& s, unsigned lane)
{
    const T cs = max_f(sec.lo, s.start), ce = min_f(sec.hi, s.end);
    const unsigned n = sec.n;
    if (n == kLargeSteps && sec.e[kLargeSteps - 1].end < sec.hi)
        return false;
    Section<T> my = { T(0), T(0), T(0) };
    if (lane < n)
        my = sec.e[lane];
    const bool ov = lane < n && my.end > cs && my.start < ce;
    const uint32_t ovm = __ballot_sync(0xffffffffu, ov);
    const T next_start = __shfl_down_sync(0xffffffffu, my.start, 1);
    const T next_dt = __shfl_down_sync(0xffffffffu, my.delta_t, 1);
    if (!ovm)
        return false;
    const unsigned f = unsigned(__ffs(int(ovm)) - 1), l = 31u - unsigned(__clz(int(ovm)));
    bool bad = ov && my.delta_t > s.delta_t;
    if (ov && lane < l && (my.end != next_start || (my.delta_t == s.delta_t && next_dt == s.delta_t)))
        bad = true; // a gap, or two neighbours that the insertion would merge
    if (lane == f && my.start > cs)
        bad = true;
    if (lane == l && my.end < ce)
        bad = true;
    return __ballot_sync(0xffffffffu, bad) == 0u;
}

// SectionSet::put (dgmr_sections.h) by the whole warp, for an s that reaches
// into [lo, hi): the overlapped range [first, last) found by ballots, the
// merged sections by lane 0 (merge_pieces, into the warp's scratch), then the
// kept tail moved (lanes 0-15) and the pieces written (lanes 16-31) in one
// step -- put()'s set, bit for bit (put_by_pieces, the serial form of this
// split, is tested against put() on random insertion sequences).  put() on one
// lane moved every section after the insertion through a ring buffer in local
// memory, one dependent access at a time: most of the march's pass 1.
template <class T>
__device__ __forceinline__ void warp_put(SectionSet<kLargeSteps, T>& sec, Section<T>* pieces, Section<T> s, unsigned lane)
{
    s.start = max_f(sec.lo, s.start);
    s.end = min_f(sec.hi, s.end);
    const unsigned n = sec.n;
    Section<T> my = { T(0), T(0), T(0) };
    if (lane < n)
        my = sec.e[lane];
    const uint32_t after = __ballot_sync(0xffffffffu, lane < n && my.end > s.start);
    const unsigned first = after ? unsigned(__ffs(int(after)) - 1) : n;
    if (first >= n) {
        if (lane == 0) {
            if (first < kLargeSteps) {
                sec.e[n] = s;
                sec.n = n + 1;
            } else {
                sec.hi = s.start;
            }
        }
        __syncwarp();
        return;
    }
    const uint32_t beyond = __ballot_sync(0xffffffffu, lane >= first && lane < n && my.end > s.end);
    unsigned last = beyond ? unsigned(__ffs(int(beyond)) - 1) : n;
    const T last_start = __shfl_sync(0xffffffffu, my.start, int(last < n ? last : 0u));
    if (last < n && last_start < s.end)
        ++last;
    unsigned np = 0, end = last;
    if (lane == 0)
        np = sec.merge_pieces(s, first, last, pieces, &end);
    np = __shfl_sync(0xffffffffu, np, 0);
    end = __shfl_sync(0xffffffffu, end, 0);
    __syncwarp();
    const unsigned k = lane - 16u;
    const bool move = lane >= end && lane < n && first + np + (lane - end) < kLargeSteps;
    const bool write = lane >= 16u && k < np && first + k < kLargeSteps;
    Section<T> pv = { T(0), T(0), T(0) };
    if (write)
        pv = pieces[k];
    __syncwarp();
    if (move)
        sec.e[first + np + (lane - end)] = my;
    if (write)
        sec.e[first + k] = pv;
    __syncwarp();
    if (lane == 0) {
        const unsigned nn = min(kLargeSteps, first + np + (n - end));
        sec.n = nn;
        if (nn == kLargeSteps)
            sec.hi = min_f(sec.hi, sec.e[kLargeSteps - 1].end);
    }
    __syncwarp();
}

// warp_put as a call: the backward march, whose loop is sensitive to its code
// size (instruction fetch), is faster with the insertion out of line (53.2 ms
// per frame at 100k Gaussians, 512^2, against 58.3 inline and 54.2 with put()
// on lane 0); the forward inlines it.
template <class T>
__device__ __noinline__ void warp_put_call(SectionSet<kLargeSteps, T>& sec, Section<T>* pieces, Section<T> s, unsigned lane)
{
    warp_put(sec, pieces, s, lane);
}

enum class PutMode { Inline, Call };

// sample_positions (marching_steps.h:202-220) by the warp, in the form of
// sample_positions_by_sections (dgmr_sections.h): lane j < n runs section j's
// chain -- counting its samples, then, after a prefix over the counts, writing
// them behind the samples of the sections before it -- and the lanes fill the
// rest with the last section's end.  The same positions, bit for bit, with the
// longest section's chain as the critical path instead of all 128 samples.
template <class T>
__device__ __forceinline__ void warp_sample_positions(const SectionSet<kLargeSteps, T>& d, T* out, unsigned lane)
{
    const unsigned n = d.n;
    if (n == 0) {
        for (unsigned k = lane; k < kSmallSteps; k += 32)
            out[k] = T(0);
        __syncwarp();
        return;
    }
    const unsigned len = lane < n ? section_samples<kSmallSteps>(d, lane) : 0u;
    unsigned incl = len;
#pragma unroll
    for (unsigned o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o)
            incl += t;
    }
    const unsigned off = 1u + incl - len; // out[0] is the first section's start
    const unsigned filled = 1u + __shfl_sync(0xffffffffu, incl, 31);
    if (lane == 0)
        out[0] = d.e[0].start;
    if (lane < n) {
        const T end = d.e[lane].end, dt = d.e[lane].delta_t;
        T v = lane == 0 ? d.e[0].start : d.e[lane - 1].end;
        for (unsigned k = 0; k < len && off + k < kSmallSteps; ++k) {
            v = min_f(end, v + dt);
            out[off + k] = v;
        }
    }
    const T last = d.e[n - 1].end;
    for (unsigned k = filled + lane; k < kSmallSteps; k += 32)
        out[k] = last;
    __syncwarp();
}

// Pass 1 (vol_marcher_forward.cu:351-403): the masked entries of a batch are
// intersected lane-parallel, then walked in list order and inserted into the
// warp's section set (in shared memory, warp_put), which every lane reads.
template <PutMode kPut = PutMode::Inline, class T>
__device__ __forceinline__ void warp_collect(SectionSet<kLargeSteps, T>& sec, Section<T>* pieces, const VmMarch<T>& a, int32_t b, int32_t e, V3<T> o,
    V3<T> d, const WarpRayMasks& rm, unsigned lane)
{
    if (a.cs.n > 0) {
        if (lane == 0)
            for (int i = 0; i < a.cs.n; ++i)
                sec.put(Section<T> { a.cs.s[i][0], a.cs.s[i][1], a.cs.s[i][2] });
        __syncwarp();
        return;
    }
    unsigned i = 0;
    for (int32_t base = b; base < e; base += 32, ++i) {
        uint32_t m = rm.get(i) & lanes_below(e - base);
        if (!m)
            continue;
        T depth = T(0), s0 = T(0), s1 = T(0), dt = T(0);
        bool ok = false;
        if ((m >> lane) & 1u) {
            const RayEntry<T> en = load_entry(a, base + int32_t(lane));
            const Gauss1d<T> g = intersect_with_ray_inv_C(en.mu, en.Q, o, d);
            const T sd = dgmr_fm::sqrt_f(g.C);
            depth = a.depths[en.id];
            const T mor = g.weight * en.mass;
            ok = !(mor <= T(1.0f / 255.f) || mor > T(1000)) && !(g.C <= T(0)) && !dgmr_fm::isnan_f(g.centre);
            s0 = g.centre - sd * T(kRelevanceSigma);
            s1 = g.centre + sd * T(kRelevanceSigma);
            dt = ((sd * T(kRelevanceSigma)) * T(2)) / T(float(kStepsPerGaussian - 1));
        }
        const uint32_t okm = __ballot_sync(0xffffffffu, ok);
        bool stop = false;
        while (m) {
            const int j = __ffs(int(m)) - 1;
            m &= m - 1u;
            const T dj = __shfl_sync(0xffffffffu, depth, j);
            if (sec.hi < dj) {
                stop = true;
                break;
            }
            if (!((okm >> j) & 1u))
                continue;
            const Section<T> sj = { __shfl_sync(0xffffffffu, s0, j), __shfl_sync(0xffffffffu, s1, j), __shfl_sync(0xffffffffu, dt, j) };
            // put() returns at once for a section outside [lo, hi) and leaves the
            // set unchanged for a covered one: skip both without the call
            if (sj.end <= sec.lo || sj.start >= sec.hi || warp_section_covered(sec, sj, lane))
                continue;
            if (kPut == PutMode::Inline)
                warp_put(sec, pieces, sj, lane);
            else
                warp_put_call(sec, pieces, sj, lane);
        }
        if (stop)
            break;
    }
}

// CDF differences of one Gaussian into the lane's bins 32 r + lane
// (math.h:461-467).  Every lane evaluates the CDF at its own borders; the
// right border of a bin is the next lane's left one.
template <class T>
__device__ __forceinline__ void warp_bins(Bin<T> (&acc)[kRayRounds], const T* borders, T centre, T inv_sd, T mor, V3<T> rgb, unsigned lane)
{
    T cs[kRayRounds];
#pragma unroll
    for (unsigned r = 0; r < kRayRounds; ++r) {
        const unsigned k = 32 * r + lane;
        cs[r] = (k <= kBins) ? cdf_inv_SD(centre, inv_sd, borders[k]) : T(0);
    }
#pragma unroll
    for (unsigned r = 0; r < kRayRounds; ++r) {
        T ce = __shfl_down_sync(0xffffffffu, cs[r], 1);
        const T next = (r + 1 < kRayRounds) ? __shfl_sync(0xffffffffu, cs[(r + 1 < kRayRounds) ? r + 1 : r], 0) : T(0);
        if (lane == 31)
            ce = next;
        const unsigned k = 32 * r + lane;
        if (k < kBins) {
            const T m = max_f(T(0), (ce - cs[r]) * mor);
            if (!(m < T(0.00001f))) {
                acc[r].r = acc[r].r + rgb.x * m;
                acc[r].g = acc[r].g + rgb.y * m;
                acc[r].b = acc[r].b + rgb.z * m;
                acc[r].m = acc[r].m + m;
            }
        }
    }
}

// The 1-D Gaussian of a masked entry if it reaches the bins (the early-outs of
// math.h:442-459); the same test in the forward and backward.
template <class T>
__device__ __forceinline__ bool warp_entry_on_bins(const RayEntry<T>& en, V3<T> o, V3<T> d, const T* borders, Gauss1d<T>* g_out, T* sd_out, T* inv_sd_out,
    T* mor_out)
{
    const Gauss1d<T> g = intersect_with_ray_inv_C(en.mu, en.Q, o, d);
    T sd, mor;
    if (!gaussian_on_ray(g, en.mass, &sd, &mor))
        return false;
    const T inv_sd = T(1) / sd;
    const T mib = mor * (cdf_inv_SD(g.centre, inv_sd, borders[kBins]) - cdf_inv_SD(g.centre, inv_sd, borders[0]));
    if (mib < T(0.0001f))
        return false;
    *g_out = g;
    *sd_out = sd;
    *inv_sd_out = inv_sd;
    *mor_out = mor;
    return true;
}

// Pass 2 (vol_marcher_forward.cu:405-437): Gaussians in list order, bins spread
// over the lanes; returns how many Gaussians filled the bins (the same on every lane)
template <class T>
__device__ __forceinline__ unsigned warp_fill(Bin<T> (&acc)[kRayRounds], const T* borders, const VmMarch<T>& a, int32_t b, int32_t e, V3<T> o, V3<T> d,
    const WarpRayMasks& rm, unsigned lane)
{
#pragma unroll
    for (unsigned r = 0; r < kRayRounds; ++r)
        acc[r] = Bin<T> { T(0), T(0), T(0), T(0) };
    unsigned i = 0, fills = 0;
    for (int32_t base = b; base < e; base += 32, ++i) {
        const uint32_t m = rm.get(i) & lanes_below(e - base);
        if (!m)
            continue;
        T centre = T(0), inv_sd = T(0), mor = T(0);
        V3<T> rgb = { T(0), T(0), T(0) };
        bool ok = false;
        if ((m >> lane) & 1u) {
            const RayEntry<T> en = load_entry(a, base + int32_t(lane));
            Gauss1d<T> g;
            T sd;
            ok = warp_entry_on_bins(en, o, d, borders, &g, &sd, &inv_sd, &mor);
            if (ok) {
                centre = g.centre;
                rgb = { a.rgb[3 * size_t(en.id)], a.rgb[3 * size_t(en.id) + 1], a.rgb[3 * size_t(en.id) + 2] };
            }
        }
        uint32_t okm = __ballot_sync(0xffffffffu, ok);
        fills += unsigned(__popc(okm));
        while (okm) {
            const int j = __ffs(int(okm)) - 1;
            okm &= okm - 1u;
            const V3<T> c = { __shfl_sync(0xffffffffu, rgb.x, j), __shfl_sync(0xffffffffu, rgb.y, j), __shfl_sync(0xffffffffu, rgb.z, j) };
            warp_bins(acc, borders, __shfl_sync(0xffffffffu, centre, j), __shfl_sync(0xffffffffu, inv_sd, j), __shfl_sync(0xffffffffu, mor, j), c, lane);
        }
    }
    return fills;
}

// bins to shared memory in order (.m = exp(-mass) for the blend, the mass itself for the peel)
template <class T>
__device__ __forceinline__ void warp_store_bins(Bin<T>* bins, const Bin<T> (&acc)[kRayRounds], unsigned lane, bool transmittance)
{
#pragma unroll
    for (unsigned r = 0; r < kRayRounds; ++r) {
        const unsigned k = 32 * r + lane;
        if (k < kBins)
            bins[k] = Bin<T> { acc[r].r, acc[r].g, acc[r].b, transmittance ? dgmr_fm::exp_f(-acc[r].m) : acc[r].m };
    }
    __syncwarp();
}

template <class T, class Frames>
__global__ void __launch_bounds__(kRayWarps * 32, sizeof(T) == 4 ? 8 : 2) k_vm_march_warp(VmMarch<T> a, const __grid_constant__ Frames frames,
    const uint32_t* __restrict__ order)
{
    __shared__ RayWarpShared<T> shared_rays[kRayWarps];
    RayWarpShared<T>& sm = shared_rays[threadIdx.x >> 5];
    const unsigned lane = threadIdx.x & 31u;
    unsigned tile, view, px, py;
    if (!ray_pixel<T>(frames, order, &tile, &view, &px, &py))
        return; // the whole warp: no block-level barrier below
    const CameraT<T>& cam = frames.cam(view);
    const V3<T> o = { cam.campos[0], cam.campos[1], cam.campos[2] };
    const V3<T> d = pixel_dir(cam, px, py);
    const int32_t b = a.ranges[2 * tile], e = a.ranges[2 * tile + 1];
    const WarpRayMasks rm = warp_ray_masks(a, b, e, o, d, lane);
    V3<T> colour = { T(0), T(0), T(0) };
    T tr = T(1);
    T start = T(0);
    T distance = T(0); // Depth mode
    SectionSet<kLargeSteps, T>& sec = sm.sec;
    unsigned long long fills = 0;
    for (unsigned step = 0;; ++step) {
        if (step >= kMaxLargeSteps) {
            if (lane == 0)
                atomicOr(&a.stats[1], DGMR_FLAG_STEP_LIMIT);
            break;
        }
        if (lane == 0)
            sec.reset(start);
        __syncwarp();
        warp_collect(sec, sm.pieces, a, b, e, o, d, rm, lane);
        warp_sample_positions(sec, sm.borders, lane);
        if (step < a.store_steps) {
            // keep this step's samples for the backward (coalesced: 32 lanes x 4 rounds)
            const size_t ray = frames.px_base(view) + size_t(py) * cam.W + px, rays = frames.rays();
            T* dst = a.store_borders + (size_t(step) * rays + ray) * kSmallSteps;
#pragma unroll
            for (unsigned r = 0; r < kRayRounds; ++r)
                dst[32 * r + lane] = sm.borders[32 * r + lane];
            if (lane == 0)
                a.store_sections[size_t(step) * rays + ray] = int32_t(sec.n);
        }
        Bin<T> acc[kRayRounds];
        fills += warp_fill(acc, sm.borders, a, b, e, o, d, rm, lane);
        warp_store_bins(sm.bins, acc, lane, a.mode != DGMR_RENDER_BINS);
        if (a.mode == DGMR_RENDER_FULL) {
            // math.h:412-428, identical on every lane
            for (unsigned k = 0; k < kBins; ++k) {
                const Bin<T> bk = sm.bins[k];
                colour.x = colour.x + bk.r * tr;
                colour.y = colour.y + bk.g * tr;
                colour.z = colour.z + bk.b * tr;
                tr = tr * bk.m;
                if (tr < T(1. / 255.))
                    break;
            }
        } else if (a.mode == DGMR_RENDER_BINS) {
            // vol_marcher_forward.cu:453-465: the sum of one bin's four channels
            const Bin<T> bk = sm.bins[min(unsigned(a.debug_bin), kBins - 1)];
            const T mass = ((bk.r + bk.g) + bk.b) + bk.m;
            colour = { mass * a.max_depth, mass * a.max_depth, mass * a.max_depth };
            if (mass == T(0))
                colour = { T(0), T(1), T(0) };
            if (dgmr_fm::isnan_f(mass))
                colour = { T(1), T(0), T(0.5) };
            if (mass < T(0))
                colour = { T(1), T(0), T(0) };
            tr = T(0);
        } else {
            // vol_marcher_forward.cu:466-481: the distance marched so far
            for (unsigned k = 0; k < kBins; ++k)
                tr = tr * sm.bins[k].m;
            distance = max_f(sec.hi, distance);
            const T dd = distance / a.max_depth;
            colour = { dd, dd, dd };
        }
        const bool done = sec.n == 0 || tr < T(1.f / 255.f);
        start = sm.borders[kSmallSteps - 1];
        __syncwarp();
        if (done)
            break;
    }
    if (lane == 0) {
        if (a.work)
            atomicAdd(a.work, fills);
        const size_t pix = size_t(py) * cam.W + px;
        const size_t plane = size_t(cam.W) * cam.H;
        T* fb = frames.fb(view, a);
        fb[pix] = colour.x + tr * cam.bg[0];
        fb[plane + pix] = colour.y + tr * cam.bg[1];
        fb[2 * plane + pix] = colour.z + tr * cam.bg[2];
        frames.remaining_T(view, a)[pix] = tr;
    }
}

} // namespace dgmr

namespace dgmr {

// Adjoint of one Gaussian's bin masses (grad/math.h:559-620), run by one lane
// over the bins in shared memory -- in bin order, so its sums round exactly
// as the one-thread loop does -- then added to the per-Gaussian accumulators.
template <class T>
__device__ __noinline__ void lane_grad_entry(const VmMarch<T>& a, int32_t k, const Bin<T>* gbins, const T* borders, V3<T> o, V3<T> d, int live_end)
{
    const RayEntry<T> en = load_entry(a, k);
    const V3<T> rgb = { a.rgb[3 * size_t(en.id)], a.rgb[3 * size_t(en.id) + 1], a.rgb[3 * size_t(en.id) + 2] };
    T g_mass = T(0);
    V3<T> grgb = { T(0), T(0), T(0) }, gmu = { T(0), T(0), T(0) };
    S3<T> gQ = { { T(0), T(0), T(0), T(0), T(0), T(0) } };
    grad_sample_gaussian(en.mu, en.Q, o, d, en.mass, rgb, borders, gbins, &g_mass, &grgb, &gmu, &gQ, live_end);
    // summed in double: a Gaussian's 13 totals collect terms from every ray and
    // large step that reaches it, in no fixed order, and many cancel; float
    // sums of that kind drift by far more than the gradients' 1e-3 tolerance
    double* dst = a.acc + size_t(en.id) * kVmAcc;
    const T v[kVmAcc] = { g_mass, grgb.x, grgb.y, grgb.z, gQ.v[0], gQ.v[1], gQ.v[2], gQ.v[3], gQ.v[4], gQ.v[5], gmu.x, gmu.y, gmu.z };
#pragma unroll
    for (int q = 0; q < int(kVmAcc); ++q)
        if (v[q] != T(0))
            atomicAdd(dst + q, double(v[q]));
}

// Pass 3: the ray's Gaussians that reach the bins are gathered, in list
// order, into a queue of 32 and run one per lane, so the lanes stay busy
// however sparse the ray's entries are in the tile list.  (Each Gaussian's
// adjoint is independent of the others'; only the atomic additions of
// different pixels meet, in no fixed order, as in the one-thread kernel.)
// live_end: the bins from there on have zero adjoints (the ray stopped before
// them), so a Gaussian whose live bins all lie there adds nothing and is not
// queued (its atomics would all be skipped as zeros).
template <class T>
__device__ __forceinline__ void warp_grad(const Bin<T>* gbins, const T* borders, int32_t* queue, const VmMarch<T>& a, int32_t b, int32_t e, V3<T> o, V3<T> d,
    const WarpRayMasks& rm, unsigned lane, int live_end)
{
    unsigned i = 0, fill = 0;
    for (int32_t base = b; base < e; base += 32, ++i) {
        const uint32_t m = rm.get(i) & lanes_below(e - base);
        if (!m)
            continue;
        bool ok = false;
        if ((m >> lane) & 1u) {
            const RayEntry<T> en = load_entry(a, base + int32_t(lane));
            Gauss1d<T> g;
            T sd, inv_sd, mor;
            ok = warp_entry_on_bins(en, o, d, borders, &g, &sd, &inv_sd, &mor);
            if (ok && live_end < int(kBins)) {
                int k0, k1;
                live_bins(borders, g.centre, inv_sd, &k0, &k1);
                ok = k0 < live_end;
            }
        }
        const uint32_t okm = __ballot_sync(0xffffffffu, ok);
        const unsigned n_ok = unsigned(__popc(okm));
        if (ok) {
            const unsigned slot = fill + unsigned(__popc(okm & lanes_below(int(lane))));
            if (slot < 32)
                queue[slot] = base + int32_t(lane);
        }
        __syncwarp();
        if (fill + n_ok >= 32) {
            lane_grad_entry(a, queue[lane], gbins, borders, o, d, live_end);
            __syncwarp();
            // the entries that did not fit go to the front of the emptied queue
            const unsigned left = fill + n_ok - 32;
            if (ok) {
                const unsigned slot = fill + unsigned(__popc(okm & lanes_below(int(lane))));
                if (slot >= 32)
                    queue[slot - 32] = base + int32_t(lane);
            }
            __syncwarp();
            fill = left;
        } else {
            fill += n_ok;
        }
    }
    if (lane < fill)
        lane_grad_entry(a, queue[lane], gbins, borders, o, d, live_end);
    __syncwarp();
}

// vol_marcher_backward.cu:115-319 with one warp per ray
template <class T, class Frames>
__global__ void __launch_bounds__(kRayWarps * 32, sizeof(T) == 4 ? 6 : 2) k_vm_march_warp_bwd(VmMarch<T> a, const __grid_constant__ Frames frames,
    const uint32_t* __restrict__ order)
{
    __shared__ RayWarpSharedBwd<T> shared_rays[kRayWarps];
    RayWarpSharedBwd<T>& sm = shared_rays[threadIdx.x >> 5];
    const unsigned lane = threadIdx.x & 31u;
    unsigned tile, view, px, py;
    if (!ray_pixel<T>(frames, order, &tile, &view, &px, &py))
        return;
    const T* grad_fb = frames.grad_fb(view, a);
    if (!grad_fb) // a view of a batch without an image gradient
        return;
    const CameraT<T>& cam = frames.cam(view);
    const V3<T> o = { cam.campos[0], cam.campos[1], cam.campos[2] };
    const V3<T> d = pixel_dir(cam, px, py);
    const int32_t b = a.ranges[2 * tile], e = a.ranges[2 * tile + 1];
    const WarpRayMasks rm = warp_ray_masks(a, b, e, o, d, lane);
    const size_t pix = size_t(py) * cam.W + px;
    const size_t plane = size_t(cam.W) * cam.H;
    const T* fb = frames.fb(view, a);
    const T final_T = frames.remaining_T(view, a)[pix];
    V3<T> colour = { fb[pix] - final_T * cam.bg[0], fb[plane + pix] - final_T * cam.bg[1], fb[2 * plane + pix] - final_T * cam.bg[2] };
    const V3<T> gc = { grad_fb[pix], grad_fb[plane + pix], grad_fb[2 * plane + pix] };
    const T gt = (gc.x * cam.bg[0] + gc.y * cam.bg[1]) + gc.z * cam.bg[2];
    T tr = T(1);
    T start = T(0);
    SectionSet<kLargeSteps, T>& sec = sm.sec;
    for (unsigned step = 0;; ++step) {
        if (step >= kMaxLargeSteps) {
            if (lane == 0)
                atomicOr(&a.stats[1], DGMR_FLAG_STEP_LIMIT);
            break;
        }
        int n_sections;
        if (step < a.store_steps) {
            // the forward kept this step's samples: no section set, no sampling
            const size_t ray = frames.px_base(view) + size_t(py) * cam.W + px, rays = frames.rays();
            const T* src = a.store_borders + (size_t(step) * rays + ray) * kSmallSteps;
#pragma unroll
            for (unsigned r = 0; r < kRayRounds; ++r)
                sm.borders[32 * r + lane] = src[32 * r + lane];
            n_sections = a.store_sections[size_t(step) * rays + ray];
            __syncwarp();
        } else {
            if (lane == 0)
                sec.reset(start);
            __syncwarp();
            warp_collect<PutMode::Call>(sec, sm.pieces, a, b, e, o, d, rm, lane);
            warp_sample_positions(sec, sm.borders, lane);
            n_sections = int(sec.n);
        }
        Bin<T> acc[kRayRounds];
        warp_fill(acc, sm.borders, a, b, e, o, d, rm, lane);
        warp_store_bins(sm.bins, acc, lane, false);
        // grad/math.h:529-557, identical on every lane; lane 0 stores the bin adjoints
        unsigned k = 0;
        for (; k < kBins; ++k) {
            const Bin<T> bk = sm.bins[k];
            Bin<T> gb;
            gb.r = tr * gc.x;
            gb.g = tr * gc.y;
            gb.b = tr * gc.z;
            const T tk = dgmr_fm::exp_f(-bk.m);
            const T inv_tk = min_f(T(255), T(1) / tk);
            colour.x = (colour.x - bk.r) * inv_tk;
            colour.y = (colour.y - bk.g) * inv_tk;
            colour.z = (colour.z - bk.b) * inv_tk;
            const T g_tk = (final_T * inv_tk) * gt + dot3(gc, colour) * tr;
            gb.m = T(0) - g_tk * tk;
            if (lane == 0)
                sm.gbins[k] = gb;
            tr = tr * tk;
            if (tr < T(1. / 255.)) {
                ++k;
                break;
            }
        }
        const int live_end = int(k);
        for (; k < kBins; ++k)
            if (lane == 0)
                sm.gbins[k] = Bin<T> { T(0), T(0), T(0), T(0) };
        __syncwarp();
        warp_grad(sm.gbins, sm.borders, sm.queue, a, b, e, o, d, rm, lane, live_end);
        const bool done = n_sections == 0 || tr < T(1.f / 255.f);
        start = sm.borders[kSmallSteps - 1];
        __syncwarp();
        if (done)
            break;
    }
}

} // namespace dgmr
