// Exact 1D total variation on one fiber, one thread per fiber.
//
// L. Condat, "A direct algorithm for 1-D total variation denoising", IEEE
// Signal Processing Letters 20(11), 2013, in its classic form (bounds vmin /
// vmax with running excesses umin / umax), generalised to a radius per edge:
// after a jump at edge e into a new segment starting at k, the bounds open at
// y_k +- (r_e -+ r_k) instead of y_k and y_k +- 2 lambda. The end of the
// signal closes the last segment with a zero dual. This is the method the
// reference runs for 1D TV steps (src/ops/tv1d.cpp:84-236), without its
// running-sum form and taut-string fallback, whose results are the same exact
// prox up to rounding. State is O(1) per fiber, so a thread needs no scratch;
// the worst case (long ramps) is quadratic.
//
// The input is read through a functor in(i) (a fiber of a sum of arrays,
// say) and the output written through a sink: segment(k0, k1, v) sets entries
// k0..k1 to v, and finish(n) runs once at the end. EagerSink writes every
// entry through out(i, v) at once; a sink may also note the segment's end only
// and fill the entries in finish, so that the threads of a warp do not wait
// on one another's long write loops at every jump.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fpb {

template <class Out>
struct EagerSink {
    Out out;
    __device__ __forceinline__ void segment(int k0, int k1, double v) const {
        for (int i = k0; i <= k1; ++i) out(i, v);
    }
    __device__ __forceinline__ void finish(int) const {}
};

// Condat's scan over a piece of m entries, radius(e) on edge (e, e + 1);
// radius(m - 1) is read but does not change the result.
template <class In, class Sink, class R>
__device__ void condat_piece(const In &in, const Sink &out, int m, const R &radius) {
    if (m == 1) {
        out.segment(0, 0, in(0));
        return;
    }
    int k = 0, k0 = 0, km = 0, kp = 0;
    double lk = radius(0);
    const double y0 = in(0);
    double vmin = y0 - lk, vmax = y0 + lk;
    double umin = lk, umax = -lk;
    auto jump_down = [&]() {  // closes [k0, km] at vmin; the edge km carries +radius
        out.segment(k0, km, vmin);
        const double le = radius(km);
        k = k0 = kp = km = km + 1;
        lk = radius(k);
        const double yk = in(k);
        vmin = yk + (le - lk);
        vmax = yk + (le + lk);
        umin = lk;
        umax = -lk;
    };
    auto jump_up = [&]() {  // closes [k0, kp] at vmax; the edge kp carries -radius
        out.segment(k0, kp, vmax);
        const double le = radius(kp);
        k = k0 = km = kp = kp + 1;
        lk = radius(k);
        const double yk = in(k);
        vmin = yk - (le + lk);
        vmax = yk - (le - lk);
        umin = lk;
        umax = -lk;
    };
    for (;;) {
        while (k < m - 1) {
            const double yn = in(k + 1);
            const double ln = radius(k + 1);
            const double len = (double)(k - k0 + 2);
            if (yn + umin < vmin - ln) {
                jump_down();
            } else if (yn + umax > vmax + ln) {
                jump_up();
            } else {
                ++k;
                umin += yn - vmin;
                umax += yn - vmax;
                if (umin >= ln) {
                    vmin += (umin - ln) / len;
                    umin = ln;
                    km = k;
                }
                if (umax <= -ln) {
                    vmax += (umax + ln) / len;
                    umax = -ln;
                    kp = k;
                }
            }
        }
        if (umin < 0.0) {
            jump_down();
        } else if (umax > 0.0) {
            jump_up();
        } else {
            const double v = vmin + umin / (double)(k - k0 + 1);
            out.segment(k0, m - 1, v);
            return;
        }
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
    S s;
    int o;
    __device__ __forceinline__ void segment(int k0, int k1, double v) const { s.segment(k0 + o, k1 + o, v); }
};

// prox of lam * sum_e w(e) |z_{e+1} - z_e| on one fiber of n entries, w(e)
// the edge weight functor (nullptr-like: has_w = false for unit weights).
// Zero-weight edges split the fiber into independent pieces; radii are
// clamped at 2 j range, a bound that an edge can never reach
// (src/ops/tv1d.cpp:238-246); no edge active past (n / 2) range gives the
// constant mean.
template <class In, class Sink, class Wt>
__device__ void tv1d_fiber_sink(const In &in, const Sink &out, int n, double lam, bool has_w, const Wt &w) {
    double lo = in(0), hi = lo;
    bool cut = false;  // a zero-weight edge
    for (int i = 1; i < n; ++i) {
        const double v = in(i);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
        if (has_w) cut = cut || w(i - 1) == 0.0;
    }
    const double range = hi - lo;
    if (n == 1 || lam == 0.0 || range == 0.0) {
        for (int i = 0; i < n; ++i) out.segment(i, i, in(i));
        out.finish(n);
        return;
    }
    if (!has_w) {
        if (lam >= (double)(n / 2) * range) {
            double s = 0.0;
            for (int i = 0; i < n; ++i) s += in(i);
            out.segment(0, n - 1, s / (double)n);
            out.finish(n);
            return;
        }
        const double cap = 2.0 * (double)((n / 2) > 0 ? (n / 2) : 1) * range;
        const double l = lam < cap ? lam : cap;
        condat_piece(in, out, n, [l](int) { return l; });
        out.finish(n);
        return;
    }
    auto piece = [&](int s, int m) {
        auto rad = [&](int j) -> double {
            if (j >= m - 1) return 0.0;
            const double r = lam * w(s + j);
            const int jj = (j + 1 < m - 1 - j) ? j + 1 : m - 1 - j;
            const double cap = 2.0 * (double)(jj > 0 ? jj : 1) * range;
            return r < cap ? r : cap;
        };
        condat_piece(Shifted<In>{in, s}, ShiftedSink<Sink>{out, s}, m, rad);
    };
    if (!cut) {
        piece(0, n);
    } else {
        int s = 0;
        for (int e = 0; e < n; ++e) {
            if (e == n - 1 || w(e) == 0.0) {
                piece(s, e - s + 1);
                s = e + 1;
            }
        }
    }
    out.finish(n);
}

// The same with the result written through out(i, v) as it is found.
template <class In, class Out, class Wt>
__device__ void tv1d_fiber(const In &in, const Out &out, int n, double lam, bool has_w, const Wt &w) {
    tv1d_fiber_sink(in, EagerSink<Out>{out}, n, lam, has_w, w);
}

struct NoWeight {
    __device__ __forceinline__ double operator()(int) const { return 1.0; }
};

}  // namespace fpb
