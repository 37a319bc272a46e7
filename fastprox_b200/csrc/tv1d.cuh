// Exact 1D total variation on one fiber, one thread per fiber.
//
// L. Condat, "A direct algorithm for 1-D total variation denoising", IEEE
// Signal Processing Letters 20(11), 2013, in its classic form (bounds vmin /
// vmax with running excesses umin / umax), generalised to a radius per edge:
// after a jump at edge e into a new segment starting at k, the bounds open at
// y_k +- (r_e -+ r_k) instead of y_k and y_k +- 2 lambda. The end of the
// signal closes the last segment with a zero dual. This is the method the
// reference runs for a single active axis (src/ops/tv1d.cpp:84-236, without
// its running-sum form and taut-string fallback, whose results are the same
// exact prox up to rounding). State is O(1) per fiber, so a thread needs no
// scratch; the worst case (long ramps) is quadratic.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fpb {

// Radius of edge e of a piece: the global lambda times the edge weight, or
// lambda; clamped at 2 j range (j = min(e + 1, m - 1 - e)), a bound that an
// edge of the piece can never reach (src/ops/tv1d.cpp:238-246), and 0 for the
// padding edge m - 1.
template <class T>
struct EdgeRadius {
    const T *w;
    int64_t ws;
    double lam, range;
    int64_t m;
    __device__ __forceinline__ double operator()(int64_t e) const {
        if (e >= m - 1) return 0.0;
        double r = w ? lam * (double)w[e * ws] : lam;
        const int64_t j = (e + 1 < m - 1 - e) ? e + 1 : m - 1 - e;
        const double cap = 2.0 * (double)(j > 0 ? j : 1) * range;
        return r < cap ? r : cap;
    }
};

// Condat's scan on y[0..m) (stride ys) into z (stride zs).
template <class T, class R>
__device__ void condat_piece(const T *y, int64_t ys, T *z, int64_t zs, int64_t m, const R &radius) {
    if (m == 1) {
        z[0] = y[0];
        return;
    }
    int64_t k = 0, k0 = 0, km = 0, kp = 0;
    double lk = radius(0);
    const double y0 = (double)y[0];
    double vmin = y0 - lk, vmax = y0 + lk;
    double umin = lk, umax = -lk;
    for (;;) {
        while (k < m - 1) {
            const double yn = (double)y[(k + 1) * ys];
            const double ln = radius(k + 1);
            const int64_t len = k - k0 + 2;
            if (yn + umin < vmin - ln) {  // a jump down closes [k0, km] at vmin
                const T v = (T)vmin;
                for (int64_t i = k0; i <= km; ++i) z[i * zs] = v;
                const double le = radius(km);
                k = k0 = kp = km = km + 1;
                lk = radius(k);
                const double yk = (double)y[k * ys];
                vmin = yk + (le - lk);
                vmax = yk + (le + lk);
                umin = lk;
                umax = -lk;
            } else if (yn + umax > vmax + ln) {  // a jump up closes [k0, kp] at vmax
                const T v = (T)vmax;
                for (int64_t i = k0; i <= kp; ++i) z[i * zs] = v;
                const double le = radius(kp);
                k = k0 = km = kp = kp + 1;
                lk = radius(k);
                const double yk = (double)y[k * ys];
                vmin = yk - (le + lk);
                vmax = yk - (le - lk);
                umin = lk;
                umax = -lk;
            } else {
                ++k;
                umin += yn - vmin;
                umax += yn - vmax;
                if (umin >= ln) {
                    vmin += (umin - ln) / (double)len;
                    umin = ln;
                    km = k;
                }
                if (umax <= -ln) {
                    vmax += (umax + ln) / (double)len;
                    umax = -ln;
                    kp = k;
                }
            }
        }
        const int64_t len = k - k0 + 1;
        if (umin < 0.0) {
            const T v = (T)vmin;
            for (int64_t i = k0; i <= km; ++i) z[i * zs] = v;
            const double le = radius(km);
            k = k0 = kp = km = km + 1;
            lk = radius(k);
            const double yk = (double)y[k * ys];
            vmin = yk + (le - lk);
            vmax = yk + (le + lk);
            umin = lk;
            umax = -lk;
        } else if (umax > 0.0) {
            const T v = (T)vmax;
            for (int64_t i = k0; i <= kp; ++i) z[i * zs] = v;
            const double le = radius(kp);
            k = k0 = km = kp = kp + 1;
            lk = radius(k);
            const double yk = (double)y[k * ys];
            vmin = yk - (le + lk);
            vmax = yk - (le - lk);
            umin = lk;
            umax = -lk;
        } else {
            const T v = (T)(vmin + umin / (double)len);
            for (int64_t i = k0; i < m; ++i) z[i * zs] = v;
            return;
        }
    }
}

// prox of lam * sum_e w_e |z_{e+1} - z_e| on one fiber of n entries (w null:
// unit weights). Zero-weight edges split the fiber into independent pieces.
template <class T>
__device__ void tv1d_fiber(const T *y, int64_t ys, T *z, int64_t zs, int64_t n, double lam, const T *w,
                           int64_t wst) {
    double lo = (double)y[0], hi = lo;
    for (int64_t i = 1; i < n; ++i) {
        const double v = (double)y[i * ys];
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    const double range = hi - lo;
    if (n == 1 || lam == 0.0 || range == 0.0) {
        for (int64_t i = 0; i < n; ++i) z[i * zs] = y[i * ys];
        return;
    }
    if (!w) {
        // No edge can be active past (n / 2) range: the constant mean.
        if (lam >= (double)(n / 2) * range) {
            double s = 0.0;
            for (int64_t i = 0; i < n; ++i) s += (double)y[i * ys];
            const T v = (T)(s / (double)n);
            for (int64_t i = 0; i < n; ++i) z[i * zs] = v;
            return;
        }
        // uniform radius: the clamp at 2 (n/2) range, the same for every edge
        const double cap = 2.0 * (double)((n / 2) > 0 ? (n / 2) : 1) * range;
        const double l = lam < cap ? lam : cap;
        struct Uni {
            double l;
            __device__ __forceinline__ double operator()(int64_t) const { return l; }
        } u{l};
        condat_piece<T>(y, ys, z, zs, n, u);
        return;
    }
    int64_t s = 0;
    for (int64_t e = 0; e < n; ++e) {
        if (e == n - 1 || (double)w[e * wst] == 0.0) {
            const int64_t m = e - s + 1;
            EdgeRadius<T> r{w + s * wst, wst, lam, range, m};
            condat_piece<T>(y + s * ys, ys, z + s * zs, zs, m, r);
            s = e + 1;
        }
    }
}

}  // namespace fpb
