// Capacity-bounded set of sample sections of the volume marcher and the walk
// that turns it into sample positions (host and device code).
//
// Semantics follow src/dgmr/marching_steps.h:35-220 (DensityArray, sample).
// A section {start, end, delta_t} asks for samples at most delta_t apart
// inside [start, end).  Inserting a section that overlaps existing ones splits
// them and keeps the smaller delta_t on the overlap; when the set is full,
// sections that no longer fit are dropped and the set's end is pulled in.
// Which sections survive that truncation is part of the rendered result and
// is pinned by the reference's known-answer tests, so the insertion steps are
// kept one to one.
#pragma once

#include "dgmr_fmath.h"

#if defined(__CUDACC__)
#define DGMR_HD_NOINLINE __host__ __device__ __noinline__
#else
#define DGMR_HD_NOINLINE
#endif

namespace dgmr {

using dgmr_fm::max_f;
using dgmr_fm::min_f;

template <class T>
struct Section {
    T start, end, delta_t;
};

template <unsigned MAX, class T>
struct SectionSet {
    unsigned n;
    T lo, hi;
    Section<T> e[MAX];

    DGMR_HD void reset(T start)
    {
        n = 0;
        lo = start;
        hi = T(1) / T(0);
    }

    DGMR_HD static void combine(const Section<T>& a, const Section<T>& b, Section<T> out[3])
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

    // Whether put(s) would leave the set exactly as it is, for an s that
    // reaches into [lo, hi): the sections overlapping s (clipped to [lo, hi))
    // cover it without a gap, none has a larger step, no two consecutive ones
    // both have s's step (put would merge those), and a full set already has
    // hi at its last end (put would pull hi in).  Then put only splits each
    // covering section against s and merges the pieces back into it, bit for
    // bit.  The marcher's device code skips such insertions (a lane-parallel
    // form of this test); tests check the claim on random insertion sequences.
    DGMR_HD bool put_leaves_unchanged(Section<T> s) const
    {
        const T cs = max_f(lo, s.start), ce = min_f(hi, s.end);
        if (n == MAX && e[MAX - 1].end < hi)
            return false;
        unsigned f = n, l = n;
        for (unsigned i = 0; i < n; ++i)
            if (e[i].end > cs && e[i].start < ce) {
                if (f == n)
                    f = i;
                l = i;
            }
        if (f == n)
            return false;
        if (e[f].start > cs || e[l].end < ce)
            return false;
        for (unsigned i = f; i <= l; ++i) {
            if (e[i].delta_t > s.delta_t)
                return false;
            if (i < l && (e[i].end != e[i + 1].start || (e[i].delta_t == s.delta_t && e[i + 1].delta_t == s.delta_t)))
                return false;
        }
        return true;
    }

    DGMR_HD_NOINLINE void put(Section<T> s)
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
        Section<T> ring[MAX];
        unsigned r_read = 0, r_write = 0;
        unsigned i_read = first, i_write = first;
        unsigned grown = 0;
        while (i_read < last + grown && i_write < MAX) {
            if (i_read < n)
                ring[(r_write++) % MAX] = e[i_read++];
            if (r_read >= r_write)
                break;
            const Section<T> head = ring[r_read % MAX];
            if (head.end <= s.start) {
                e[i_write++] = ring[(r_read++) % MAX];
                continue;
            }
            if (head.start >= s.end)
                break;
            Section<T> p[3];
            combine(ring[(r_read++) % MAX], s, p);
            if (p[0].delta_t == p[1].delta_t) {
                p[1].start = p[0].start;
                p[0].end = p[0].start;
            }
            s = p[2];
            if (p[0].end - p[0].start <= T(0)) {
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
        if (s.end - s.start > T(0) && i_write < MAX) {
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

    // put() for an s (clipped to [lo, hi)) that overlaps the set from
    // e[first] (the first section ending after s.start) up to e[last - 1]
    // (last: one past the last section starting before s.end), split in two
    // steps.  merge_pieces() walks the overlapped sections in order, as put()'s
    // ring loop does, and returns the pieces that replace e[first, *end); the
    // set is then e[0, first) + pieces + e[*end, n), cut to MAX sections (hi
    // pulled in to the last end when it is full).  put()'s ring exists only to
    // write that sequence in place; the marcher's warps instead move the kept
    // tail and write the pieces lane-parallel (put_by_pieces is the serial
    // form, checked against put() on random insertion sequences).
    DGMR_HD unsigned merge_pieces(Section<T> s, unsigned first, unsigned last, Section<T>* pieces, unsigned* end) const
    {
        unsigned np = 0, i = first;
        for (; i < last; ++i) {
            const Section<T> head = e[i];
            if (head.end <= s.start) {
                pieces[np++] = head;
                continue;
            }
            if (head.start >= s.end)
                break;
            Section<T> p[3];
            combine(head, s, p);
            if (p[0].delta_t == p[1].delta_t) {
                p[1].start = p[0].start;
                p[0].end = p[0].start;
            }
            s = p[2];
            if (p[0].end - p[0].start <= T(0)) {
                if (p[1].delta_t == p[2].delta_t) {
                    s.start = p[1].start;
                    continue;
                }
                pieces[np++] = p[1];
            } else {
                pieces[np++] = p[0];
                if (p[1].delta_t == p[2].delta_t) {
                    s.start = p[1].start;
                    continue;
                }
                pieces[np++] = p[1];
            }
        }
        *end = i;
        if (s.end - s.start > T(0))
            pieces[np++] = s;
        return np;
    }

    DGMR_HD void put_by_pieces(Section<T> s)
    {
        if (s.end <= lo || s.start >= hi)
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
        Section<T> pieces[2 * MAX + 1], tail[MAX];
        unsigned end = last;
        const unsigned np = merge_pieces(s, first, last, pieces, &end);
        const unsigned nt = n - end;
        for (unsigned i = 0; i < nt; ++i)
            tail[i] = e[end + i];
        unsigned w = first;
        for (unsigned i = 0; i < np && w < MAX; ++i)
            e[w++] = pieces[i];
        for (unsigned i = 0; i < nt && w < MAX; ++i)
            e[w++] = tail[i];
        n = w;
        if (n == MAX)
            hi = min_f(hi, e[n - 1].end);
    }
};

// marching_steps.h:202-220: NS monotone sample positions (all zero for an empty set)
template <unsigned NS, unsigned MAX, class T>
DGMR_HD void sample_positions_n(const SectionSet<MAX, T>& d, T* out)
{
    if (d.n == 0) {
        for (unsigned i = 0; i < NS; ++i)
            out[i] = T(0);
        return;
    }
    out[0] = d.e[0].start;
    unsigned cur = 0;
    T prev = out[0];
    for (unsigned i = 1; i < NS; ++i) {
        const T v = min_f(d.e[cur].end, prev + d.e[cur].delta_t);
        out[i] = v;
        prev = v;
        if (cur < d.n - 1 && v == d.e[cur].end)
            ++cur;
    }
}

// The same positions, section by section: section j's samples are the chain
// v <- min(end_j, v + delta_j) from the previous section's end (from e[0].start
// for j = 0) until v reaches end_j -- sample_positions_n advances to the next
// section exactly there -- and the last section's chain continues to NS.  So
// each section's chain can run on its own lane, placed after the samples of
// the sections before it (the marcher's warps do that); this is the serial
// form, checked against sample_positions_n on random section sets.
// section_samples returns how many samples section j places (the last: its
// steps until v reaches its end; every count capped at NS - 1).
template <unsigned NS, unsigned MAX, class T>
DGMR_HD unsigned section_samples(const SectionSet<MAX, T>& d, unsigned j)
{
    const T end = d.e[j].end, dt = d.e[j].delta_t;
    T v = j == 0 ? d.e[0].start : d.e[j - 1].end;
    unsigned len = 0;
    while (len < NS - 1) {
        v = min_f(end, v + dt);
        ++len;
        if (v == end)
            break;
    }
    return len;
}

template <unsigned NS, unsigned MAX, class T>
DGMR_HD void sample_positions_by_sections(const SectionSet<MAX, T>& d, T* out)
{
    if (d.n == 0) {
        for (unsigned i = 0; i < NS; ++i)
            out[i] = T(0);
        return;
    }
    out[0] = d.e[0].start;
    unsigned off = 1;
    T v = out[0];
    for (unsigned j = 0; j < d.n && off < NS; ++j) {
        const T end = d.e[j].end, dt = d.e[j].delta_t;
        const unsigned len = section_samples<NS>(d, j);
        v = j == 0 ? d.e[0].start : d.e[j - 1].end;
        for (unsigned k = 0; k < len && off + k < NS; ++k) {
            v = min_f(end, v + dt);
            out[off + k] = v;
        }
        off += len;
    }
    // the last section's chain after it reached its end: min(end, end + dt) = end
    const T last = d.e[d.n - 1].end;
    for (unsigned i = off; i < NS; ++i)
        out[i] = last;
}


} // namespace dgmr
