// Exact 1D total variation on fibres: Condat's direct algorithm.
//
// L. Condat, "A direct algorithm for 1-D total variation denoising", IEEE
// Signal Processing Letters 20(11), 2013, generalised to a radius per edge:
// after a jump at edge e into a new segment starting at k, the bounds open at
// y_k + sigma r_e -+ r_k (sigma = +1 after a jump down, -1 after one up)
// instead of y_k and y_k +- 2 lambda. The end of the signal closes the last
// segment with a zero dual. The arithmetic is the reference's running-sum
// form of Condat's scan (src/ops/tv1d.cpp:72-83, 156-217), started at each
// segment's first sample (the reference's Short = 1 variant, :94-101), so
// that every step is the same few operations (CondatScan): the segment is
// tracked by the running sum s = sigma r_e + sum_{k0..k} (y_i - ref),
// ref = y_{k0}; the candidates ref + (s -+ r_k) / m bound its value, vmin is
// the running maximum of the lower ones and vmax the running minimum of the
// upper ones, and a jump down (up) is an upper (lower) candidate passing
// below vmin (above vmax). The reference runs the paper's bound updates in a
// segment's first three samples (Short = 3) and its end test in that form for
// segments of one sample, which rounds differently (the same exact prox).
// The scan computes in C: double (the reference's arithmetic) for double
// fibres, float for float fibres, whose inputs and outputs are float (the
// constant-mean case sums in double either way). 1/m comes from a table of
// correctly rounded reciprocals (the reference's RecipTable, the same values
// in double) or a division. Products are rounded on their own (__dmul_rn,
// __fmul_rn), never fused into the sums, as on the reference's x86-64 build. Unlike the reference, the scan never hands a row to the taut string:
// on ramps, where it rescans quadratically many steps (the reference's budget
// of 3n + 1024 rescans), it runs on to the same exact prox.
//
// The input is read through a functor in(i) (a fiber of a sum of arrays,
// say) and the output written through a sink: segment(k0, k1, v) sets entries
// k0..k1 to v, and finish(n) runs once at the end. EagerSink writes every
// entry through out(i, v) at once; a sink may also note the segment's end only
// and fill the entries in finish.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdint>

namespace fpb {

// The compute type's infinity and unfused product.
template <class C>
struct Num;
template <>
struct Num<double> {
    static __device__ __forceinline__ double inf() { return CUDART_INF; }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
};
template <>
struct Num<float> {
    static __device__ __forceinline__ float inf() { return CUDART_INF_F; }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
};

// 1/m by division.
template <class C>
struct DivRecip {
    __device__ __forceinline__ C operator()(int m) const { return C(1) / (C)m; }
};
// 1/m from a table t[m] = 1/m filled by DivRecip, m <= the fibre's length.
template <class C>
struct TableRecip {
    const C *t;
    __device__ __forceinline__ C operator()(int m) const { return t[m]; }
};

// The reference's min_nonan / max_nonan on NaN-free values (src/core/op.hpp:1198-1222).
template <class C>
__device__ __forceinline__ C min_nn(C a, C v) { return v < a ? v : a; }
template <class C>
__device__ __forceinline__ C max_nn(C a, C v) { return v > a ? v : a; }

template <class Out>
struct EagerSink {
    Out out;
    __device__ __forceinline__ void segment(int k0, int k1, double v) const {
        for (int i = k0; i <= k1; ++i) out(i, v);
    }
    __device__ __forceinline__ void finish(int) const {}
};

// One fibre's scan. k is the last sample taken (k0 - 1 while a segment
// opens), k0 the segment's first sample, km / kp the last samples where vmin /
// vmax were set and rkm / rkp their edges' radii (the radius a jump there
// opens the next segment with), ref = y_{k0} and s the running sum. Every step
// is the same arithmetic on one entry y and one radius r, read at next():
//  * opening a segment at k0 (after a jump at edge e, sigma = +1 down, -1 up):
//    ref = y, s = sigma r_e, and the candidates ref + (s -+ r) are the bounds;
//  * taking sample k + 1: s1 = s + (y - ref), candidates a, b = ref +
//    (s1 -+ r) / m; b below vmin is a jump down at km, a above vmax one up
//    at kp, else vmin = max(vmin, a), vmax = min(vmax, b);
//  * at the end (k = n - 1): the mean v = ref + s / m with the same tests.
template <class C>
struct CondatScan {
    int k, k0, km, kp;
    C vmin, vmax, ref, s, rkm, rkp;
    bool open;

    __device__ __forceinline__ void start() {
        k = -1;
        k0 = km = kp = 0;
        vmin = vmax = ref = s = rkm = rkp = C(0);
        open = true;
    }
    // Index of the entry the next step reads (n - 1 at the end test, where
    // the value read is not used).
    __device__ __forceinline__ int next(int n) const { return k + 1 < n ? k + 1 : n - 1; }
    // The segment length m of the next step (1 when it opens a segment).
    __device__ __forceinline__ int len(int n) const { return k == n - 1 ? k - k0 + 1 : k - k0 + 2; }

    // One step with yv = in(next(n)), rv = radius(next(n)) and rc = 1 /
    // len(n); true when the fibre is done.
    template <class Sink>
    __device__ __forceinline__ bool step(int n, C yv, C rv, C rc, const Sink &out) {
        const bool atend = k == n - 1;
        const C rf = open ? yv : ref;
        const C y = atend ? rf : yv;
        const C r = atend ? C(0) : rv;
        const C lo = open ? -Num<C>::inf() : vmin, hi = open ? Num<C>::inf() : vmax;
        const C s1 = s + (y - rf);
        const C a = rf + Num<C>::mul(s1 - r, rc), b = rf + Num<C>::mul(s1 + r, rc);
        const bool dn = b < lo, up = !dn && a > hi;
        if (!dn && !up) {
            if (atend) {
                out.segment(k0, n - 1, (double)a);
                return true;
            }
            ++k;
            s = s1;
            ref = rf;
            const bool cm = a >= lo, cp = b <= hi;
            km = cm ? k : km;
            rkm = cm ? r : rkm;
            vmin = max_nn(lo, a);
            kp = cp ? k : kp;
            rkp = cp ? r : rkp;
            vmax = min_nn(hi, b);
            open = false;
            return false;
        }
        const int e = dn ? km : kp;
        out.segment(k0, e, (double)(dn ? vmin : vmax));
        const C le = dn ? rkm : rkp;
        s = dn ? le : -le;
        k = e;
        k0 = e + 1;
        open = true;
        return false;
    }
};

// Condat's scan over a piece of m entries, radius(e) on edge (e, e + 1);
// radius(m - 1) is read but does not change the result.
template <class C, class In, class Sink, class R, class Rcp>
__device__ __forceinline__ void condat_piece(const In &in, const Sink &out, int m, const R &radius, const Rcp &rcp) {
    CondatScan<C> st;
    st.start();
    for (;;) {
        const int i = st.next(m);
        if (st.step(m, (C)in(i), radius(i), rcp(st.len(m)), out)) return;
    }
}

// Shifts a functor's index by an offset (a piece of a fiber).
template <class F>
struct Shifted {
    F f;
    int o;
    __device__ __forceinline__ auto operator()(int i) const { return f(i + o); }
};
template <class S>
struct ShiftedSink {
    const S &s;  // the sink itself (a sink may count what it is given)
    int o;
    __device__ __forceinline__ void segment(int k0, int k1, double v) const { s.segment(k0 + o, k1 + o, v); }
};

// Range (max - min) of a fibre, whether an edge has zero weight, and the
// largest edge weight.
template <class C, class In, class Wt>
__device__ __forceinline__ void fiber_range(const In &in, int n, bool has_w, const Wt &w, C &range, bool &cut,
                                            C &wmax) {
    C lo = (C)in(0), hi = lo;
    cut = false;
    wmax = C(0);
    for (int i = 1; i < n; ++i) {
        const C v = (C)in(i);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
        if (has_w) {
            const C we = (C)w(i - 1);
            cut = cut || we == C(0);
            wmax = we > wmax ? we : wmax;
        }
    }
    range = hi - lo;
}

// The constant mean (no edge can be active), summed in double.
template <class In, class Sink>
__device__ __forceinline__ void fiber_mean(const In &in, const Sink &out, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += (double)in(i);
    out.segment(0, n - 1, s / (double)n);
}

// prox of lam * sum_e w(e) |z_{e+1} - z_e| on one fiber of n entries, w(e)
// the edge weight functor (has_w = false for unit weights), computed in C.
// Zero-weight edges split the fiber into independent pieces; radii are
// clamped at 2 j range, a bound that an edge can never reach
// (src/ops/tv1d.cpp:238-246); no edge active past (n / 2) range gives the
// constant mean.
template <class C, class In, class Sink, class Wt, class Rcp>
__device__ __forceinline__ void tv1d_fiber_sink(const In &in, const Sink &out, int n, double lam_d, bool has_w,
                                                const Wt &w, const Rcp &rcp) {
    const C lam = (C)lam_d;
    C range, wmax;
    bool cut;
    fiber_range<C>(in, n, has_w, w, range, cut, wmax);
    if (n == 1 || lam == C(0) || range == C(0)) {
        for (int i = 0; i < n; ++i) out.segment(i, i, (double)in(i));
        out.finish(n);
        return;
    }
    if (!has_w) {
        if (lam >= (C)(n / 2) * range) {
            fiber_mean(in, out, n);
            out.finish(n);
            return;
        }
        const C cap = C(2) * (C)((n / 2) > 0 ? (n / 2) : 1) * range;
        const C l = lam < cap ? lam : cap;
        condat_piece<C>(in, out, n, [l](int) { return l; }, rcp);
        out.finish(n);
        return;
    }
    auto piece = [&](int s, int m) {
        auto rad = [&](int j) -> C {
            if (j >= m - 1) return C(0);
            const C r = lam * (C)w(s + j);
            const int jj = (j + 1 < m - 1 - j) ? j + 1 : m - 1 - j;
            const C cap = C(2) * (C)(jj > 0 ? jj : 1) * range;
            return r < cap ? r : cap;
        };
        condat_piece<C>(Shifted<In>{in, s}, ShiftedSink<Sink>{out, s}, m, rad, rcp);
    };
    if (!cut) {
        piece(0, n);
    } else {
        int s = 0;
        for (int e = 0; e < n; ++e) {
            if (e == n - 1 || (C)w(e) == C(0)) {
                piece(s, e - s + 1);
                s = e + 1;
            }
        }
    }
    out.finish(n);
}

// The same with the result written through out(i, v) as it is found.
template <class C, class In, class Out, class Wt, class Rcp>
__device__ void tv1d_fiber(const In &in, const Out &out, int n, double lam, bool has_w, const Wt &w, const Rcp &rcp) {
    tv1d_fiber_sink<C>(in, EagerSink<Out>{out}, n, lam, has_w, w, rcp);
}

struct NoWeight {
    __device__ __forceinline__ double operator()(int) const { return 1.0; }
};

constexpr int kScanUnroll = 4;  // scan steps per trip of tv1d_warp's loop

// tv1d_fiber_sink on the fibres of one warp at once: lane t scans fibre t when
// `act`, every lane of the warp calls it, and n is the same for all. COPY: a
// fibre that is its own prox is written through the sink too (every entry a
// segment of its own; without COPY the sink's storage is the input's). Run one
// lane per thread, the scans drift apart and a warp runs each lane's branches
// in turn; here the warp takes one CondatScan step of every live scan per trip
// of a loop that all its lanes share, and every step is the same arithmetic,
// so every instruction issued serves every live fibre (only a segment's write
// is a branch). The values are those of condat_piece, bit for bit. Fibres
// with zero-weight edges (pieces) run tv1d_fiber_sink after the loop. A scan
// takes at most 2 (n + 1)^2 steps (every jump moves the segment's start
// forward, and between jumps k only grows): the loop stops there.
template <class C, bool COPY = false, class In, class Sink, class Wt, class Rcp>
__device__ __forceinline__ void tv1d_warp(const In &in, const Sink &out, int n, double lam_d, bool has_w, const Wt &w,
                                          const Rcp &rcp, bool act) {
    const C lam = (C)lam_d;
    C range = C(0), wmax = C(0);
    bool cut = false;
    if (act) fiber_range<C>(in, n, has_w, w, range, cut, wmax);
    bool live = false, fill = false, serial = false;
    C l = lam;
    if (act && !(n == 1 || lam == C(0) || range == C(0))) {  // else the fibre is its own prox
        if (!has_w) {
            if (lam >= (C)(n / 2) * range) {
                fiber_mean(in, out, n);
                fill = true;
            } else {
                const C cap = C(2) * (C)((n / 2) > 0 ? (n / 2) : 1) * range;
                l = lam < cap ? lam : cap;
                live = fill = true;
            }
        } else if (!cut) {
            live = fill = true;
        } else {
            serial = true;
        }
    }
    // Below 2 range no radius reaches its clamp (2 max(j, 1) range), so the
    // clamp can be skipped when that holds for every live fibre of the warp.
    const bool clamp = has_w && __any_sync(0xffffffffu, live && lam * wmax > C(2) * range);
    CondatScan<C> st;
    st.start();
    // The loop, specialised on the radius form (warp-uniform: no weights, the
    // weights' radii, or those capped at the clamp), so that a step's radius
    // takes no branch, and four steps per trip (on 64 x 512^2 with edge weights
    // 195 images/s at one step per trip, 206 at two, 227 at four). A scan takes fewer than 2 (n + 1)^2 steps, which fits an
    // int for fibres of up to 32766 entries (a long counter beyond).
    auto scan = [&](auto rad, auto count) {
        using Cnt = decltype(count);
        const Cnt steps = (Cnt)2 * (Cnt)(n + 1) * (Cnt)(n + 1);
        // kScanUnroll steps of every live scan per trip (a lane whose scan ends
        // within a trip takes no further step), one vote per trip
        for (Cnt it = 0; it < steps && __any_sync(0xffffffffu, live); it += kScanUnroll) {
#pragma unroll
            for (int u = 0; u < kScanUnroll; ++u) {
                if (live) {
                    const int i = st.next(n);
                    live = !st.step(n, (C)in(i), rad(i), rcp(st.len(n)), out);
                }
            }
        }
    };
    auto run = [&](auto count) {
        if (!has_w) {
            scan([l](int) { return l; }, count);
        } else if (!clamp) {
            scan([&](int j) -> C { return j >= n - 1 ? C(0) : lam * (C)w(j); }, count);
        } else {
            scan(
                [&](int j) -> C {
                    if (j >= n - 1) return C(0);
                    const C r = lam * (C)w(j);
                    const int jj = (j + 1 < n - 1 - j) ? j + 1 : n - 1 - j;
                    const C cap = C(2) * (C)(jj > 0 ? jj : 1) * range;
                    return r < cap ? r : cap;
                },
                count);
        }
    };
    if (n <= 32766) run(0);
    else run(0ll);
    if (fill) out.finish(n);
    if (serial) tv1d_fiber_sink<C>(in, out, n, lam_d, true, w, rcp);
    if (COPY && act && !fill && !serial) {
        for (int i = 0; i < n; ++i) out.segment(i, i, (double)in(i));
        out.finish(n);
    }
}

}  // namespace fpb
