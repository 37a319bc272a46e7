// The vector-Jacobian product of isotropic TV on sm_100a, by implicit
// differentiation at the point a prox call kept (keep_structure).
//
// The reference's TVIso::save / Sys / cg / vjp_img (src/ops/tv_iso.cpp:551-631,
// 672-934, 1000-1067), per image on the device:
//   * structure: a pixel is flat when it has no active forward neighbour, when
//     its gradient |(W D z)_p| is at the rounding level of the data, or when
//     its dual is strictly inside its ball (complementary slackness); flat
//     pixels join their forward neighbours into regions (union-find, each
//     region named by its smallest pixel index, its "root");
//   * the system (M^T (I + G_A^T H G_A) M) c = M^T g on the regions, with
//     H_p = r_p / max(|g_p|, mu) (I - n_p n_p^T) on the non-flat pixels, solved
//     by conjugate gradients preconditioned by its diagonal (Jacobi), each
//     image stopping at its own tolerance (the relative error of z that its gap
//     certifies, at least 1e-10, or the caller's);
//   * gx = M c (every pixel takes its region's value), and the step's gradient
//     -sum over non-flat pixels of alpha_p <(G gx)_p, n_p>.
// Region vectors live at the roots' slots of pixel-sized arrays, so nothing
// is compacted. Every region sum (the right-hand side, each product with the
// matrix, the diagonal) is accumulated in 128-bit fixed point with integer
// atomics: exact, so the result is the same bit for bit on every run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "vjp.h"

namespace fpb {
namespace {

constexpr int kT = 256;

__device__ __forceinline__ int uf_find_h(int *P, int i) {
    for (int n = 0; n < (1 << 30); ++n) {
        const int p = P[i];
        if (p == i) return i;
        const int q = P[p];
        if (q != p) P[i] = q;
        i = p;
    }
    return i;
}

__device__ __forceinline__ int uf_root_r(const int *P, int i) {
    for (int n = 0; n < (1 << 30); ++n) {
        const int p = P[i];
        if (p == i) return i;
        i = p;
    }
    return i;
}

// ---- 128-bit fixed point -------------------------------------------------

struct I128 {
    unsigned long long lo;
    long long hi;
};

// v 2^s as a 128-bit integer (|v 2^s| < 2^126)
__device__ __forceinline__ I128 to_fixed(double v, int s) {
    const double t = ldexp(v, s);
    const double h = floor(ldexp(t, -64));
    const double rem = t - ldexp(h, 64);  // in [0, 2^64)
    I128 r;
    r.hi = (long long)h;
    double rr = rint(rem);
    if (rr >= 18446744073709551616.0) {
        rr = 0.0;
        r.hi += 1;
    }
    r.lo = (unsigned long long)rr;
    return r;
}

__device__ __forceinline__ double from_fixed(unsigned long long lo, long long hi, int s) {
    return ldexp(ldexp((double)hi, 64) + (double)lo, -s);
}

__device__ __forceinline__ I128 add128(I128 a, I128 b) {
    I128 r;
    r.lo = a.lo + b.lo;
    r.hi = a.hi + b.hi + (r.lo < a.lo ? 1 : 0);
    return r;
}

// acc[2 slot] (lo) and acc[2 slot + 1] (hi) += v 2^s; a warp whose lanes all
// add to one slot sums first and adds once.
__device__ __forceinline__ void racc(unsigned long long *acc, int slot, double v, int s, bool active) {
    const unsigned mask = __activemask();
    I128 x = active ? to_fixed(v, s) : I128{0ull, 0ll};
    const int lead_slot = __shfl_sync(mask, active ? slot : -1, __ffs(mask) - 1);
    const bool uniform = __all_sync(mask, !active || slot == lead_slot) && lead_slot >= 0 && mask == 0xffffffffu;
    if (uniform) {
        for (int o = 16; o > 0; o >>= 1) {
            I128 y;
            y.lo = __shfl_down_sync(mask, x.lo, o);
            y.hi = __shfl_down_sync(mask, x.hi, o);
            if ((threadIdx.x & 31) + o < 32) x = add128(x, y);
        }
        if ((threadIdx.x & 31) == 0) {
            const unsigned long long old = atomicAdd(acc + 2 * (int64_t)lead_slot, x.lo);
            const unsigned long long carry = (old + x.lo < old) ? 1ull : 0ull;
            atomicAdd(acc + 2 * (int64_t)lead_slot + 1, (unsigned long long)x.hi + carry);
        }
        return;
    }
    if (!active) return;
    const unsigned long long old = atomicAdd(acc + 2 * (int64_t)slot, x.lo);
    const unsigned long long carry = (old + x.lo < old) ? 1ull : 0ull;
    atomicAdd(acc + 2 * (int64_t)slot + 1, (unsigned long long)x.hi + carry);
}

// the fixed-point exponent for values below 2^E in magnitude over N terms
__device__ __forceinline__ int fixed_exp(double maxabs, int64_t N) {
    if (!(maxabs > 0.0) || !isfinite(maxabs)) return 0;
    int lg = 0;
    while ((1LL << lg) <= N) ++lg;
    return 124 - lg - (ilogb(maxabs) + 1);
}

// ---- per-image bookkeeping --------------------------------------------------

__device__ __forceinline__ bool img_reduce(const VjpBuffers &bf, int b, unsigned blk, unsigned nblk, double a0,
                                           double a1, double *sh, int *flag, double &t0, double &t1, bool mx) {
    const double s0 = mx ? block_max(a0, sh) : block_sum(a0, sh);
    const double s1 = block_sum(a1, sh);
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[blk * 2 + 0] = s0;
        part[blk * 2 + 1] = s1;
    }
    if (!arrive_last(bf.ticket + b, nblk, flag)) return false;
    t0 = mx ? max_partials(part, nblk, 2, 0, sh) : sum_partials(part, nblk, 2, 0, sh);
    t1 = sum_partials(part, nblk, 2, 1, sh);
    if (threadIdx.x != 0) return false;
    bf.ticket[b] = 0;
    return true;
}

struct Px {  // a pixel's coordinates and its forward neighbours
    int64_t co[3];
    bool has[3];
};

__device__ __forceinline__ Px pix_of(const VjpGeom &g, int64_t p) {
    Px x;
    for (int a = 0; a < 3; ++a) {
        x.co[a] = a < g.k ? (p / g.S[a]) % g.L[a] : 0;
        x.has[a] = a < g.k && g.wa[a] != 0.0 && x.co[a] + 1 < g.L[a];
    }
    return x;
}

// z at the solved scale of image b at pixel q: from the dual of the solve
// (d - G^T u, tv_iso.cpp:251-270), or the stored z of a single-axis solve
template <class T>
__device__ __forceinline__ double z_at(const VjpGeom &g, const VjpBuffers &bf, int b, int64_t q) {
    const int mode = bf.img[b].mode;
    const int64_t N = g.N;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    if (mode == kModeTv1d) return (double)static_cast<const T *>(bf.U[0])[(int64_t)b * g.k * N + q];
    if (mode != kModeFdpg) return (double)D[q];
    const T *U = static_cast<const T *>(bf.U[bf.st[b].fin_par]) + (int64_t)b * g.k * N;
    double z = (double)D[q];
    for (int a = 0; a < g.k; ++a) {
        const double wh = g.wh[a];
        if (wh == 0.0) continue;
        const int64_t co = (q / g.S[a]) % g.L[a];
        const double cur = (double)U[a * N + q];
        const double prev = co > 0 ? (double)U[a * N + q - g.S[a]] : 0.0;
        z += wh * (cur - prev);
    }
    return z;
}

// ---- structure (tv_iso.cpp:551-631) ---------------------------------------------

template <class T>
__global__ void __launch_bounds__(kT) st_flat(VjpGeom g, VjpBuffers bf) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const VjpImage &vi = bf.vimg[b];
    const int mode = bf.img[b].mode;
    const bool from_dual = mode == kModeFdpg;
    const T *U = from_dual ? static_cast<const T *>(bf.U[bf.st[b].fin_par]) + (int64_t)b * g.k * N : nullptr;
    const T *AL = bf.alpha ? static_cast<const T *>(bf.alpha) + (int64_t)b * bf.alpha_stride : nullptr;
    double *GZ = bf.gz + (int64_t)b * g.k * N;
    uint8_t *F = bf.flat + (int64_t)b * N;
    int *P = bf.root + (int64_t)b * N;
    int *C = bf.cnt + (int64_t)b * N;
    unsigned long long *A = bf.acc + (int64_t)b * 2 * N;
    // an image with no active axis (gamma 0) has none here either: every
    // pixel flat and alone, G z = 0 (tv_iso.cpp:938-939)
    const bool ident = mode == kModeIdentity;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const Px x = pix_of(g, p);
        const double z0 = z_at<T>(g, bf, b, p);
        double nn = 0.0;
        bool any = false;
        for (int a = 0; a < g.k; ++a) {
            double gv = 0.0;
            if (x.has[a] && !ident) {
                gv = g.wa[a] * (z_at<T>(g, bf, b, p + g.S[a]) - z0);
                nn += gv * gv;
                any = true;
            }
            GZ[a * N + p] = gv;
        }
        bool fl = !any || sqrt(nn) <= vi.thr;
        if (from_dual && !fl) {
            double uu = 0.0;
            for (int a = 0; a < g.k; ++a) {
                const double ua = (double)U[a * N + p] / g.wmax;
                uu += ua * ua;
            }
            const double r = AL ? ((double)AL[p] == 0.0 ? 0.0 : vi.gs * (double)AL[p]) : vi.gs;
            fl = sqrt(uu) < r * (1.0 - g.eta);
        }
        F[p] = fl ? (any ? 1 : 3) : 0;  // bit 0: flat; bit 1: no active neighbour
        P[p] = (int)p;
        C[p] = 0;
        A[2 * p] = 0ull;
        A[2 * p + 1] = 0ull;
    }
}

// flat pixels with an active neighbour join it (tv_iso.cpp:601-608)
__global__ void st_union(VjpGeom g, VjpBuffers bf) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const uint8_t *F = bf.flat + (int64_t)b * N;
    int *P = bf.root + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        if (F[p] != 1) continue;
        const Px x = pix_of(g, p);
        for (int a = 0; a < g.k; ++a) {
            if (!x.has[a]) continue;
            int u = (int)p, v = (int)(p + g.S[a]);
            for (int tries = 0;; ++tries) {
                u = uf_find_h(P, u);
                v = uf_find_h(P, v);
                if (u == v) break;
                const int hi = u > v ? u : v, lo = u > v ? v : u;
                const int old = atomicCAS(P + hi, hi, lo);
                if (old == hi) break;
                u = old;
                v = lo;
                if (tries > (1 << 24)) {
                    atomicExch(bf.err, 2);
                    break;
                }
            }
        }
    }
}

// every pixel to its root (each thread writes its own entry); region sizes
__global__ void st_roots(VjpGeom g, VjpBuffers bf) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    int *P = bf.root + (int64_t)b * N;
    int *C = bf.cnt + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const int r = uf_root_r(P, (int)p);
        P[p] = r;
        atomicAdd(C + r, 1);
    }
}

// ---- region sums of pixel values: max pass, atomic pass, read-out ----------------

// pass 1 over the per-pixel values v_p (kind: 0 the cotangent g, 1 the product
// y = pix + G^T H G pix of the conjugate gradients, 3 a right-hand side
// already in y): the per-image maximum |v| sets the fixed-point exponent.
template <class T>
__device__ __forceinline__ double apply_y(const VjpGeom &g, const VjpBuffers &bf, int b, int64_t p) {
    // y_p = c[root p] - sum_a w_a (h_a[p] - h_a[p - e_a]) (tv_iso.cpp:870-884)
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N;
    const double *PV = bf.pv + (int64_t)b * N;
    const double *Hh = bf.h + (int64_t)b * g.k * N;
    double y = PV[R[p]];
    for (int a = 0; a < g.k; ++a) {
        if (g.wa[a] == 0.0) continue;
        const int64_t co = (p / g.S[a]) % g.L[a];
        const double prev = co > 0 ? Hh[a * N + p - g.S[a]] : 0.0;
        y -= g.wa[a] * (Hh[a * N + p] - prev);
    }
    return y;
}

template <class T>
__global__ void __launch_bounds__(kT) rs_max(VjpGeom g, VjpBuffers bf, int kind, const T *__restrict__ gin) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    if (kind == 1 && bf.cg[b].status != kCgLive) return;
    const int64_t N = g.N;
    double m = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        double v;
        if (kind == 0) v = (double)gin[(int64_t)b * N + p];
        else if (kind == 3) v = bf.y[(int64_t)b * N + p];
        else v = apply_y<T>(g, bf, b, p);
        if (kind == 1) bf.y[(int64_t)b * N + p] = v;
        m = fmax(m, fabs(v));
    }
    double mx, unused;
    if (!img_reduce(bf, b, blockIdx.x, gridDim.x, m, 0.0, sh, &flag, mx, unused, true)) return;
    bf.cg[b].fx = fixed_exp(mx, N);
}

template <class T>
__global__ void __launch_bounds__(kT) rs_add(VjpGeom g, VjpBuffers bf, int kind, const T *__restrict__ gin) {
    const int b = blockIdx.y;
    if (kind == 1 && bf.cg[b].status != kCgLive) return;
    const int64_t N = g.N;
    const int s = bf.cg[b].fx;
    const int *R = bf.root + (int64_t)b * N;
    unsigned long long *A = bf.acc + (int64_t)b * 2 * N;
    const int64_t n_pad = ((N + 31) / 32) * 32;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_pad; p += (int64_t)gridDim.x * blockDim.x) {
        const bool act = p < N;
        double v = 0.0;
        int slot = 0;
        if (act) {
            v = kind == 0 ? (double)gin[(int64_t)b * N + p] : bf.y[(int64_t)b * N + p];
            slot = R[p];
        }
        racc(A, slot, v, s, act);
    }
}

// read-out at the roots: out[C] = the sum, accumulators cleared
__global__ void rs_read(VjpGeom g, VjpBuffers bf, int kind, double *outv) {
    const int b = blockIdx.y;
    if (kind == 1 && bf.cg[b].status != kCgLive) return;
    const int64_t N = g.N;
    const int s = bf.cg[b].fx;
    const int *R = bf.root + (int64_t)b * N;
    unsigned long long *A = bf.acc + (int64_t)b * 2 * N;
    double *O = outv + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        if (R[p] != p) continue;
        O[p] = from_fixed(A[2 * p], (long long)A[2 * p + 1], s);
        A[2 * p] = 0ull;
        A[2 * p + 1] = 0ull;
    }
}

// ---- Jacobi diagonal ---------------------------------------------------------

template <class T>
__device__ __forceinline__ int jterms(const VjpGeom &g, const VjpBuffers &bf, int b, int64_t p, int *slot,
                                      double *val) {
    const int64_t N = g.N;
    if (bf.flat[(int64_t)b * N + p] & 1) return 0;
    const int *R = bf.root + (int64_t)b * N;
    const double *GZ = bf.gz + (int64_t)b * g.k * N;
    const VjpImage &vi = bf.vimg[b];
    const Px x = pix_of(g, p);
    double nn = 0.0;
    for (int a = 0; a < g.k; ++a) nn += GZ[a * N + p] * GZ[a * N + p];
    const double nr = sqrt(nn);
    double rp = vi.gs;
    if (bf.alpha) {
        const double al = (double)static_cast<const T *>(bf.alpha)[(int64_t)b * bf.alpha_stride + p];
        rp = al == 0.0 ? 0.0 : vi.gs * al;
    }
    const double hs = rp / fmax(nr, vi.mu);
    int lab[4];
    lab[0] = R[p];
    for (int a = 0; a < g.k; ++a) lab[a + 1] = x.has[a] ? R[p + g.S[a]] : -1;
    int n = 0;
    for (int c = 0; c <= g.k; ++c) {
        const int C = lab[c];
        if (C < 0) continue;
        bool seen = false;
        for (int e = 0; e < c; ++e) seen = seen || lab[e] == C;
        if (seen) continue;
        double hh = 0.0, nh = 0.0;
        for (int a = 0; a < g.k; ++a) {
            if (!x.has[a]) continue;
            const double h = g.wa[a] * ((lab[a + 1] == C ? 1.0 : 0.0) - (lab[0] == C ? 1.0 : 0.0));
            hh += h * h;
            nh += h * GZ[a * N + p] / nr;
        }
        slot[n] = C;
        val[n] = hs * (hh - nh * nh);
        ++n;
    }
    return n;
}

template <class T>
__global__ void __launch_bounds__(kT) jac_max(VjpGeom g, VjpBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int64_t N = g.N;
    double m = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        int slot[4];
        double val[4];
        const int n = jterms<T>(g, bf, b, p, slot, val);
        for (int i = 0; i < n; ++i) m = fmax(m, fabs(val[i]));
        if (bf.root[(int64_t)b * N + p] == p) m = fmax(m, (double)bf.cnt[(int64_t)b * N + p]);
    }
    double mx, unused;
    if (!img_reduce(bf, b, blockIdx.x, gridDim.x, m, 0.0, sh, &flag, mx, unused, true)) return;
    bf.cg[b].fx = fixed_exp(mx * 8.0, N);
}

template <class T>
__global__ void __launch_bounds__(kT) jac_add(VjpGeom g, VjpBuffers bf) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int s = bf.cg[b].fx;
    unsigned long long *A = bf.acc + (int64_t)b * 2 * N;
    const int64_t n_pad = ((N + 31) / 32) * 32;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_pad; p += (int64_t)gridDim.x * blockDim.x) {
        int slot[4] = {0, 0, 0, 0};
        double val[4] = {0.0, 0.0, 0.0, 0.0};
        int n = 0;
        if (p < N) {
            n = jterms<T>(g, bf, b, p, slot, val);
            if (bf.root[(int64_t)b * N + p] == p) {  // |C| at the root
                slot[n] = (int)p;
                val[n] = (double)bf.cnt[(int64_t)b * N + p];
                ++n;
            }
        }
        for (int i = 0; i < 5; ++i) {
            const bool act = i < n;
            racc(A, act ? slot[i] : 0, act ? val[i] : 0.0, s, act);
        }
    }
}

// ---- conjugate gradients (tv_iso.cpp:891-934) --------------------------------

// initial state: dinv = 1 / diag, bn = sum b^2 / |C|, x = 0, r = b, pv = r dinv, rz
__global__ void __launch_bounds__(kT) cg_init(VjpGeom g, VjpBuffers bf, double tol, int max_iter) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N;
    const int *C = bf.cnt + (int64_t)b * N;
    double *X = bf.x + (int64_t)b * N, *Rr = bf.r + (int64_t)b * N, *PV = bf.pv + (int64_t)b * N;
    double *DI = bf.dinv + (int64_t)b * N;
    const double *Bv = bf.b + (int64_t)b * N;
    double bn = 0.0, rz = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        if (R[p] != p) continue;
        const double di = 1.0 / DI[p];
        DI[p] = di;
        const double bv = Bv[p];
        X[p] = 0.0;
        Rr[p] = bv;
        PV[p] = bv * di;
        bn += bv * bv / (double)C[p];
        rz += bv * bv * di;
    }
    double tbn, trz;
    if (!img_reduce(bf, b, blockIdx.x, gridDim.x, bn, rz, sh, &flag, tbn, trz, false)) return;
    CgState &cs = bf.cg[b];
    cs.bn = tbn;
    cs.rz = trz;
    cs.res = 1.0;
    cs.it = 0;
    const double t = tol > 0.0 ? tol : fmax(1e-10, bf.vimg[b].rel);
    cs.tol = t;
    cs.status = (tbn == 0.0 || bf.img[b].mode == kModeNan) ? kCgDone : kCgLive;
    if (tbn == 0.0) cs.res = 0.0;
    if (cs.status == kCgLive) atomicAdd(bf.live, 1);
    cs.max_iter = max_iter;
}

// h = H G pix with pix = pv[root] (tv_iso.cpp:870-877, 809-827)
template <class T>
__global__ void __launch_bounds__(kT) cg_hg(VjpGeom g, VjpBuffers bf) {
    const int b = blockIdx.y;
    if (bf.cg[b].status != kCgLive) return;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N;
    const double *PV = bf.pv + (int64_t)b * N;
    const double *GZ = bf.gz + (int64_t)b * g.k * N;
    const uint8_t *F = bf.flat + (int64_t)b * N;
    double *Hh = bf.h + (int64_t)b * g.k * N;
    const VjpImage &vi = bf.vimg[b];
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const Px x = pix_of(g, p);
        if (F[p] & 1) {
            for (int a = 0; a < g.k; ++a) Hh[a * N + p] = 0.0;
            continue;
        }
        const double c0 = PV[R[p]];
        double y[3] = {0.0, 0.0, 0.0}, nn = 0.0, dot = 0.0;
        for (int a = 0; a < g.k; ++a) {
            y[a] = x.has[a] ? g.wa[a] * (PV[R[p + g.S[a]]] - c0) : 0.0;
            nn += GZ[a * N + p] * GZ[a * N + p];
        }
        const double nr = sqrt(nn);
        for (int a = 0; a < g.k; ++a) dot += GZ[a * N + p] * y[a];
        double rp = vi.gs;
        if (bf.alpha) {
            const double al = (double)static_cast<const T *>(bf.alpha)[(int64_t)b * bf.alpha_stride + p];
            rp = al == 0.0 ? 0.0 : vi.gs * al;
        }
        const double h = rp / fmax(nr, vi.mu);
        for (int a = 0; a < g.k; ++a) {
            const double na = GZ[a * N + p] / nr;
            Hh[a * N + p] = h * (y[a] - na * dot / nr);
        }
    }
}

// after qv = A pv: alpha = rz / <pv, qv>
__global__ void __launch_bounds__(kT) cg_alpha(VjpGeom g, VjpBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    if (bf.cg[b].status != kCgLive) return;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N;
    const double *PV = bf.pv + (int64_t)b * N, *QV = bf.qv + (int64_t)b * N;
    double pq = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
        if (R[p] == p) pq += PV[p] * QV[p];
    double t, unused;
    if (!img_reduce(bf, b, blockIdx.x, gridDim.x, pq, 0.0, sh, &flag, t, unused, false)) return;
    CgState &cs = bf.cg[b];
    if (!(t > 0.0)) {
        cs.status = kCgDone;
        atomicSub(bf.live, 1);
        return;
    }
    cs.alpha = cs.rz / t;
}

// x += alpha pv, r -= alpha qv; beta, the residual and the stopping test
__global__ void __launch_bounds__(kT) cg_step(VjpGeom g, VjpBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    if (bf.cg[b].status != kCgLive) return;
    const int64_t N = g.N;
    const double al = bf.cg[b].alpha;
    const int *R = bf.root + (int64_t)b * N;
    const int *C = bf.cnt + (int64_t)b * N;
    double *X = bf.x + (int64_t)b * N, *Rr = bf.r + (int64_t)b * N;
    const double *PV = bf.pv + (int64_t)b * N, *QV = bf.qv + (int64_t)b * N, *DI = bf.dinv + (int64_t)b * N;
    double rzn = 0.0, rn = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        if (R[p] != p) continue;
        X[p] += al * PV[p];
        const double r = Rr[p] - al * QV[p];
        Rr[p] = r;
        rzn += r * r * DI[p];
        rn += r * r / (double)C[p];
    }
    double t0, t1;
    if (!img_reduce(bf, b, blockIdx.x, gridDim.x, rzn, rn, sh, &flag, t0, t1, false)) return;
    CgState &cs = bf.cg[b];
    cs.beta = t0 / cs.rz;
    cs.rz = t0;
    cs.it += 1;
    cs.res = sqrt(t1 / cs.bn);
    if (!(cs.res > cs.tol) || cs.it >= cs.max_iter) {
        cs.status = kCgDone;
        atomicSub(bf.live, 1);
    }
}

__global__ void cg_pv(VjpGeom g, VjpBuffers bf) {
    const int b = blockIdx.y;
    if (bf.cg[b].status != kCgLive) return;
    const int64_t N = g.N;
    const double be = bf.cg[b].beta;
    const int *R = bf.root + (int64_t)b * N;
    double *PV = bf.pv + (int64_t)b * N;
    const double *Rr = bf.r + (int64_t)b * N, *DI = bf.dinv + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
        if (R[p] == p) PV[p] = Rr[p] * DI[p] + be * PV[p];
}

// ---- outputs (tv_iso.cpp:1014-1057) --------------------------------------------

// gx = M x; per image the step's gradient -sum_A alpha_p <(G v)_p, n_p>
template <class T>
__global__ void __launch_bounds__(kT) vjp_out(VjpGeom g, VjpBuffers bf, const T *__restrict__ gin, T *__restrict__ gx,
                                              int conj) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N;
    const double *X = bf.x + (int64_t)b * N;
    const double *GZ = bf.gz + (int64_t)b * g.k * N;
    const uint8_t *F = bf.flat + (int64_t)b * N;
    const bool nan = bf.img[b].mode == kModeNan;
    const bool empty = bf.cg[b].bn == 0.0;
    double gg = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const double v = empty ? 0.0 : X[R[p]];
        const double gi = (double)gin[(int64_t)b * N + p];
        double outv = nan ? (double)CUDART_NAN : v;
        if (conj) outv = gi - outv;
        gx[(int64_t)b * N + p] = (T)outv;
        if (nan || (F[p] & 1)) continue;
        const Px x = pix_of(g, p);
        double nn = 0.0, t = 0.0;
        for (int a = 0; a < g.k; ++a) nn += GZ[a * N + p] * GZ[a * N + p];
        const double nr = sqrt(nn);
        for (int a = 0; a < g.k; ++a) {
            const double gv = x.has[a] && !empty ? g.wa[a] * (X[R[p + g.S[a]]] - v) : 0.0;
            t += gv * GZ[a * N + p] / nr;
        }
        double al = 1.0;
        if (bf.alpha)
            al = (double)static_cast<const T *>(bf.alpha)[(int64_t)b * bf.alpha_stride + p];
        gg += al * t;
    }
    double tg, unused;
    if (!img_reduce(bf, b, blockIdx.x, gridDim.x, gg, 0.0, sh, &flag, tg, unused, false)) return;
    bf.ggam[b] = nan ? (double)CUDART_NAN : (conj ? 0.0 : -tg);
}

// ---- parameter gradients and the forward derivative (tv_iso.cpp:953-1057) -------

// The dual of an image solved as one 1D TV per fiber along its active axis
// (tv_iso.cpp:386-397): u[p] = -(1/w) sum_{i <= p} (d - z) along the fiber,
// 0 at its end; into out (B x N), for those images only.
template <class T>
__global__ void tv1d_dual(VjpGeom g, VjpBuffers bf, double *out) {
    const int b = blockIdx.y;
    if (bf.img[b].mode != kModeTv1d || g.act1 < 0) return;
    const int a = g.act1;
    const int64_t N = g.N, L = g.L[a], S = g.S[a];
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Z = static_cast<const T *>(bf.U[0]) + (int64_t)b * g.k * N;
    double *O = out + (int64_t)b * N;
    const double w = g.wa[a];
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < N / L; f += (int64_t)gridDim.x * blockDim.x) {
        const int64_t st = (f / S) * L * S + f % S;  // the fiber's first pixel
        double cs = 0.0;
        for (int64_t i = 0; i < L; ++i) {
            const int64_t o = st + i * S;
            cs += (double)D[o] - (double)Z[o];
            O[o] = i + 1 < L ? -cs / w : 0.0;
        }
    }
}

// u_a[q] of image b at the solved scale in the reference's form (z = d - G^T u)
template <class T>
__device__ __forceinline__ double u_at(const VjpGeom &g, const VjpBuffers &bf, int b, int a, int64_t q,
                                       const double *u1d) {
    const int mode = bf.img[b].mode;
    if (mode == kModeFdpg)
        return (double)static_cast<const T *>(bf.U[bf.st[b].fin_par])[((int64_t)b * g.k + a) * g.N + q] / g.wmax;
    if (mode == kModeTv1d && a == g.act1) return u1d[(int64_t)b * g.N + q];
    return 0.0;
}

// the radius gamma alpha_p at the solved scale
template <class T>
__device__ __forceinline__ double radius_at(const VjpBuffers &bf, int b, int64_t p) {
    const double gs = bf.vimg[b].gs;
    if (!bf.alpha) return gs;
    const double al = (double)static_cast<const T *>(bf.alpha)[(int64_t)b * bf.alpha_stride + p];
    return al == 0.0 ? 0.0 : gs * al;
}

// v = J^T g at a pixel: its region's value (NaN for a NaN image)
__device__ __forceinline__ double v_at(const VjpGeom &g, const VjpBuffers &bf, int b, int64_t q) {
    if (bf.img[b].mode == kModeNan) return (double)CUDART_NAN;
    if (bf.cg[b].bn == 0.0) return 0.0;
    return bf.x[(int64_t)b * g.N + bf.root[(int64_t)b * g.N + q]];
}

// Per pixel, the terms of the parameter gradients from v = J^T g
// (tv_iso.cpp:1020-1057), each times -2^e:
//   h_a[p] = (v[p + e_a] - v[p]) u_a[p] + [p non-flat] (H G v)_{a,p} (G z)_{a,p} / w_a
//   y[p]   = gamma alpha_p <(G v)_p, n_p> on non-flat pixels (alpha's gradient)
template <class T>
__global__ void __launch_bounds__(kT) vjp_params(VjpGeom g, VjpBuffers bf, const double *u1d) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int mode = bf.img[b].mode;
    const double sc = ldexp(1.0, bf.img[b].e);
    const double *GZ = bf.gz + (int64_t)b * g.k * N;
    const uint8_t *F = bf.flat + (int64_t)b * N;
    double *Hh = bf.h + (int64_t)b * g.k * N;
    double *Y = bf.y + (int64_t)b * N;
    const VjpImage &vi = bf.vimg[b];
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        double hv[3] = {0.0, 0.0, 0.0}, ay = 0.0;
        if (mode != kModeIdentity) {
            const Px x = pix_of(g, p);
            const double v0 = v_at(g, bf, b, p);
            double gv[3] = {0.0, 0.0, 0.0};
            for (int a = 0; a < g.k; ++a) {
                const bool next = g.L[a] > 1 && x.co[a] + 1 < g.L[a];
                const double vn = next ? v_at(g, bf, b, p + g.S[a]) : 0.0;
                if (next) hv[a] = (vn - v0) * u_at<T>(g, bf, b, a, p, u1d);
                if (x.has[a]) gv[a] = g.wa[a] * (vn - v0);
            }
            if (!(F[p] & 1)) {
                double nn = 0.0, dot = 0.0;
                for (int a = 0; a < g.k; ++a) {
                    nn += GZ[a * N + p] * GZ[a * N + p];
                    dot += GZ[a * N + p] * gv[a];
                }
                const double nr = sqrt(nn);
                const double h = radius_at<T>(bf, b, p) / fmax(nr, vi.mu);
                double t = 0.0;
                for (int a = 0; a < g.k; ++a) {
                    const double na = GZ[a * N + p] / nr;
                    const double hg = h * (gv[a] - na * dot / nr);
                    if (g.wa[a] != 0.0) hv[a] += hg * GZ[a * N + p] / g.wa[a];
                    t += gv[a] * na;
                }
                if (bf.alpha) ay = -(sc * vi.gs) * t;
            }
        }
        for (int a = 0; a < g.k; ++a) Hh[a * N + p] = -sc * hv[a];
        Y[p] = ay;
    }
}

// per image, the sums of h_a0 and h_a1 (a1 < 0: none) into gw[3 b + a]
__global__ void __launch_bounds__(kT) param_sums(VjpGeom g, VjpBuffers bf, int a0, int a1) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const double *H0 = bf.h + ((int64_t)b * g.k + a0) * N;
    const double *H1 = a1 >= 0 ? bf.h + ((int64_t)b * g.k + a1) * N : nullptr;
    double s0 = 0.0, s1 = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        s0 += H0[p];
        if (H1) s1 += H1[p];
    }
    double t0, t1;
    if (!img_reduce(bf, b, blockIdx.x, gridDim.x, s0, s1, sh, &flag, t0, t1, false)) return;
    bf.gw[3 * b + a0] = t0;
    if (a1 >= 0) bf.gw[3 * b + a1] = t1;
}

// alpha's gradient: out[p] = sum over the images, in order, of y[b][p]
__global__ void alpha_sum(VjpGeom g, VjpBuffers bf, double *out) {
    const int64_t N = g.N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int64_t b = 0; b < g.B; ++b) t += bf.y[b * N + p];
        out[p] = t;
    }
}

// The forward derivative's right-hand side before G^T (tv_iso.cpp:958-985):
//   y[p] = dx[p] + sum_a 2^e dw_a (u_a[p] - u_a[p - e_a]),
//   c_p  = H_p (2^e dW D z)_p + dr_p n_p on non-flat pixels (0 on flat ones),
//   dr_p = dgamma alpha_p + gamma 2^e dalpha_p  (dgamma without pixel weights),
// c into h.
template <class T>
__global__ void __launch_bounds__(kT) jvp_terms(VjpGeom g, VjpBuffers bf, const T *__restrict__ dx, double dgamma,
                                                JvpDir dir, const double *__restrict__ dalpha, const double *u1d) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int mode = bf.img[b].mode;
    const double sc = ldexp(1.0, bf.img[b].e);
    const double *GZ = bf.gz + (int64_t)b * g.k * N;
    const uint8_t *F = bf.flat + (int64_t)b * N;
    double *Hh = bf.h + (int64_t)b * g.k * N;
    double *Y = bf.y + (int64_t)b * N;
    const VjpImage &vi = bf.vimg[b];
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const Px x = pix_of(g, p);
        double rhs = dx ? (double)dx[(int64_t)b * N + p] : 0.0;
        double c[3] = {0.0, 0.0, 0.0};
        if (mode != kModeIdentity) {
            for (int a = 0; a < g.k; ++a) {
                if (dir.dw[a] == 0.0 || g.L[a] <= 1) continue;
                const double prev = x.co[a] > 0 ? u_at<T>(g, bf, b, a, p - g.S[a], u1d) : 0.0;
                rhs += sc * dir.dw[a] * (u_at<T>(g, bf, b, a, p, u1d) - prev);
            }
            if (!(F[p] & 1)) {
                double nn = 0.0, dot = 0.0;
                for (int a = 0; a < g.k; ++a) {
                    c[a] = g.wa[a] != 0.0 ? sc * dir.dw[a] * GZ[a * N + p] / g.wa[a] : 0.0;
                    nn += GZ[a * N + p] * GZ[a * N + p];
                    dot += GZ[a * N + p] * c[a];
                }
                const double nr = sqrt(nn);
                const double h = radius_at<T>(bf, b, p) / fmax(nr, vi.mu);
                double dr = dgamma;
                if (bf.alpha) {
                    const double al = (double)static_cast<const T *>(bf.alpha)[(int64_t)b * bf.alpha_stride + p];
                    dr = dgamma * al + (dalpha ? vi.gs * (sc * dalpha[p]) : 0.0);
                }
                for (int a = 0; a < g.k; ++a) {
                    const double na = GZ[a * N + p] / nr;
                    c[a] = h * (c[a] - na * dot / nr) + dr * na;
                }
            }
        }
        Y[p] = rhs;
        for (int a = 0; a < g.k; ++a) Hh[a * N + p] = c[a];
    }
}

// y -= G^T c, i.e. y[p] += sum_a w_a (c_a[p] - c_a[p - e_a]) (tv_iso.cpp:986)
__global__ void __launch_bounds__(kT) jvp_rhs(VjpGeom g, VjpBuffers bf) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const double *Hh = bf.h + (int64_t)b * g.k * N;
    double *Y = bf.y + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        double t = Y[p];
        for (int a = 0; a < g.k; ++a) {
            if (g.wa[a] == 0.0) continue;
            const int64_t co = (p / g.S[a]) % g.L[a];
            const double prev = co > 0 ? Hh[a * N + p - g.S[a]] : 0.0;
            t += g.wa[a] * (Hh[a * N + p] - prev);
        }
        Y[p] = t;
    }
}

// dz = M x (every pixel its region's value); the conjugate's dx - dz
template <class T>
__global__ void __launch_bounds__(kT) jvp_out(VjpGeom g, VjpBuffers bf, const T *__restrict__ dx, T *__restrict__ dz,
                                              int conj) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        double v = v_at(g, bf, b, p);
        if (conj) v = (dx ? (double)dx[(int64_t)b * N + p] : 0.0) - v;
        dz[(int64_t)b * N + p] = (T)v;
    }
}

// ---- anisotropic TV: structure and derivatives (tv_aniso.cpp:1012-1440) ----------

// z of image b at the solved scale: the input for an image without an active
// axis, NaN for a NaN image, else the solver's z (or its polished zp)
template <class T>
__device__ __forceinline__ double an_z(const VjpGeom &g, const VjpBuffers &bf, int b, int64_t q) {
    const int mode = bf.aimg[b].mode;
    const int64_t N = g.N;
    if (mode == kAnNan) return (double)CUDART_NAN;
    if (mode == kAnIdentity) return (double)static_cast<const T *>(bf.d)[(int64_t)b * N + q];
    const T *Z = static_cast<const T *>(bf.ast[b].zsel ? bf.zp : bf.U[1]) + (int64_t)b * N;
    return (double)Z[q];
}

// q_a of image b at the solved scale (the dual is kept at the input's scale)
template <class T>
__device__ __forceinline__ double an_q(const VjpGeom &g, const VjpBuffers &bf, int b, int a, int64_t q) {
    const AnImage &im = bf.aimg[b];
    const double v = (double)static_cast<const T *>(bf.qd)[((int64_t)a * g.B + b) * g.N + q];
    return im.e ? ldexp(v, -im.e) : v;
}

// lam_a of image b at the solved scale; a NaN image takes none (its
// components are single entries, tv_aniso.cpp:284-290)
__device__ __forceinline__ double an_lam(const VjpBuffers &bf, int b, int a) {
    const AnImage &im = bf.aimg[b];
    return im.mode == kAnNan ? 0.0 : im.lam[a];
}

template <class T>
__device__ __forceinline__ double an_beta(const VjpGeom &g, const VjpBuffers &bf, int a, int64_t i) {
    return bf.beta ? (double)static_cast<const T *>(bf.beta)[(int64_t)a * g.N + i] : 1.0;
}

// jump_bound (tv_aniso.cpp:1257-1300) per image: A = TV(z) + sum |z| |d - z|,
// the range of z and max |d|, summed and maxed in fixed trees, then tau and
// tau0; the structure's arrays are reset on the way.
template <class T>
__global__ void __launch_bounds__(kT) ad_bound(VjpGeom g, VjpBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    uint8_t *F = bf.flat + (int64_t)b * N, *Cd = bf.code + (int64_t)b * N;
    int *R = bf.root + (int64_t)b * N, *Cn = bf.cnt + (int64_t)b * N;
    unsigned long long *Ac = bf.acc + (int64_t)b * 2 * N;
    double lam[3];
    for (int a = 0; a < 3; ++a) lam[a] = a < g.k ? an_lam(bf, b, a) : 0.0;
    double A = 0.0, dm = 0.0, zhi = -DBL_MAX, nlo = -DBL_MAX;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const Px x = pix_of(g, p);
        const double z = an_z<T>(g, bf, b, p), d = (double)D[p];
        double tv = 0.0;
        for (int a = 0; a < g.k; ++a)
            if (lam[a] != 0.0 && x.co[a] + 1 < g.L[a])
                tv += lam[a] * an_beta<T>(g, bf, a, p) * fabs(an_z<T>(g, bf, b, p + g.S[a]) - z);
        A += tv + fabs(z) * fabs(d - z);
        dm = fmax(dm, fabs(d));
        zhi = fmax(zhi, z);
        nlo = fmax(nlo, -z);
        F[p] = 0;
        Cd[p] = 0;
        R[p] = (int)p;
        Cn[p] = 0;
        Ac[2 * p] = 0ull;
        Ac[2 * p + 1] = 0ull;
    }
    // four values per block: A (sum), max |d|, max z, max -z
    const double sA = block_sum(A, sh);
    const double sD = block_max(dm, sh);
    const double sZ = block_max(zhi, sh);
    const double sN = block_max(nlo, sh);
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[blockIdx.x * 4 + 0] = sA;
        part[blockIdx.x * 4 + 1] = sD;
        part[blockIdx.x * 4 + 2] = sZ;
        part[blockIdx.x * 4 + 3] = sN;
    }
    if (!arrive_last(bf.ticket + b, gridDim.x, &flag)) return;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    double tA = 0.0, tD = 0.0, tZ = -DBL_MAX, tN = -DBL_MAX;
    for (unsigned i = 0; i < gridDim.x; ++i) {
        tA += part[i * 4 + 0];
        tD = fmax(tD, part[i * 4 + 1]);
        tZ = fmax(tZ, part[i * 4 + 2]);
        tN = fmax(tN, part[i * 4 + 3]);
    }
    double lmax = 0.0;
    for (int a = 0; a < g.k; ++a)
        if (lam[a] != 0.0 && g.L[a] > 1) lmax += lam[a] * g.bmax[a];
    AnVjpImage &vi = bf.avimg[b];
    const double none = (double)CUDART_NAN;
    if (!(lmax > 0.0)) {
        vi.tau = vi.tau0 = none;
        return;
    }
    const double range = tZ + tN;
    const double tau0 = 64.0 * g.eps_t * (tD + 2.0 * lmax);
    vi.tau0 = tau0;
    const double gap = fmax(vi.gap, 0.0);
    if (!(2.0 * sqrt(2.0 * gap) < range)) {
        vi.tau = none;
        return;
    }
    const double M = (double)((g.k + 1) * N);
    const double gp = gap + (M + 4.0) * DBL_EPSILON * tA;
    const double tau = 2.0 * sqrt(2.0 * gp) + tau0;
    vi.tau = tau < range ? tau : none;
}

__device__ __forceinline__ uint8_t an_sgn(double v, int sh) {
    return (uint8_t)((((unsigned)(v > 0.0)) | ((unsigned)(v < 0.0) << 1)) << sh);
}

// edge_codes / code_chunk (tv_aniso.cpp:1095-1160) along axis a, one thread
// per fibre: the 1D dual p_e from the running sum of q_a; an edge with a bound
// is flat when its dual is strictly inside it (and its jump not certified) or
// its jump is within the rounding allowance; the others carry a sign, from the
// dual or, certified or without weight, from z's jump.
template <class T>
__global__ void __launch_bounds__(128) ad_codes(VjpGeom g, VjpBuffers bf, int a) {
    const int b = blockIdx.y;
    const int64_t N = g.N, L = g.L[a], s = g.S[a];
    if (L <= 1) return;
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= N / L) return;
    const int64_t base = (f / s) * L * s + f % s;
    uint8_t *F = bf.flat + (int64_t)b * N, *Cd = bf.code + (int64_t)b * N;
    const double lam = an_lam(bf, b, a);
    const AnVjpImage vi = bf.avimg[b];
    const bool cert = vi.tau == vi.tau;
    const int sh = 2 * a;
    const uint8_t bit = (uint8_t)(1u << a);
    double acc = 0.0;
    double zi = an_z<T>(g, bf, b, base);
    for (int64_t l = 0; l + 1 < L; ++l) {
        const int64_t i = base + l * s;
        const double zn = an_z<T>(g, bf, b, i + s);
        const uint8_t zc = an_sgn(zi - zn, sh);
        if (!(lam > 0.0)) {
            Cd[i] |= zc;
        } else {
            acc += an_q<T>(g, bf, b, a, i);
            const double pe = -acc;
            const double w = an_beta<T>(g, bf, a, i);
            const double le = lam * w;
            const double jump = fabs(zn - zi);
            const bool certified = cert && le > 0.0 && jump > vi.tau;
            bool flat = (fabs(pe) < le * (1.0 - g.eta) && !certified) || (le > 0.0 && jump <= vi.tau0);
            if (bf.side) {  // a branch override at a kink (tv_aniso.cpp:1150-1154)
                const int sd = bf.side[(int64_t)b * N + i];
                const bool kink = sd != 0 && le > 0.0 && jump <= g.stol && fabs(pe) >= le - g.stol;
                flat = kink ? sd < 0 : flat;
            }
            const bool from_z = certified || (bf.beta && w == 0.0);
            const uint8_t c = from_z ? zc : an_sgn(-pe, sh);
            if (flat) F[i] |= bit;
            else Cd[i] |= c;
        }
        zi = zn;
    }
}

// flat edges join their ends (union-find, roots at the smallest index)
__global__ void ad_union(VjpGeom g, VjpBuffers bf) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const uint8_t *F = bf.flat + (int64_t)b * N;
    int *P = bf.root + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t fl = F[p];
        if (!fl) continue;
        for (int a = 0; a < g.k; ++a) {
            if (!((fl >> a) & 1)) continue;
            int u = (int)p, v = (int)(p + g.S[a]);
            for (int tries = 0;; ++tries) {
                u = uf_find_h(P, u);
                v = uf_find_h(P, v);
                if (u == v) break;
                const int hi = u > v ? u : v, lo = u > v ? v : u;
                const int old = atomicCAS(P + hi, hi, lo);
                if (old == hi) break;
                u = old;
                v = lo;
                if (tries > (1 << 24)) {
                    atomicExch(bf.err, 2);
                    break;
                }
            }
        }
    }
}

// The sign of the edge (i, i + S[a]) between two components (1, -1), else 0.
__device__ __forceinline__ int an_edge_sign(const VjpGeom &g, const VjpBuffers &bf, int b, int a, int64_t i) {
    const int64_t N = g.N;
    const int cf = (bf.code[(int64_t)b * N + i] >> (2 * a)) & 3;
    if (cf == 0) return 0;
    const int *R = bf.root + (int64_t)b * N;
    if (R[i + g.S[a]] == R[i]) return 0;
    return cf == 1 ? 1 : -1;
}

// y = the term of entry i in S_{C(i),a}: its edge (i, i + e_a) to another
// component minus the edge (i - e_a, i) from one, each sign_e beta_e
// (tv_aniso.cpp:1187-1255)
template <class T>
__global__ void __launch_bounds__(kT) ad_term(VjpGeom g, VjpBuffers bf, int a) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    double *Y = bf.y + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        double e = 0.0;
        if (g.L[a] > 1) {
            const int64_t co = (p / g.S[a]) % g.L[a];
            if (co + 1 < g.L[a]) {
                const int sf = an_edge_sign(g, bf, b, a, p);
                if (sf) e += sf * an_beta<T>(g, bf, a, p);
            }
            if (co > 0) {
                const int sb = an_edge_sign(g, bf, b, a, p - g.S[a]);
                if (sb) e -= sb * an_beta<T>(g, bf, a, p - g.S[a]);
            }
        }
        Y[p] = e;
    }
}

// the component averages of the cotangent G_C = sum_C g / |C| at the roots
// (from the region sums in b); gx = G_C(i) (the conjugate's g - G); per root
// the products S_{C,a} G_C into h for the parameter sums
template <class T>
__global__ void __launch_bounds__(kT) ad_vjp_out(VjpGeom g, VjpBuffers bf, const T *__restrict__ gin,
                                                  T *__restrict__ gx, int conj) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N, *Cn = bf.cnt + (int64_t)b * N;
    const double *Bv = bf.b + (int64_t)b * N;
    double *X = bf.x + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const int r = R[p];
        const double G = Bv[r] / (double)Cn[r];
        double o = G;
        if (conj) o = (double)gin[(int64_t)b * N + p] - G;
        gx[(int64_t)b * N + p] = (T)o;
        if (r == p) X[p] = G;
        for (int a = 0; a < g.k; ++a)
            bf.h[((int64_t)b * g.k + a) * N + p] = r == p ? bf.gz[((int64_t)b * g.k + a) * N + p] * G : 0.0;
    }
}

// the edge weights' gradient along axis a, per image:
// -gamma w_a sign_e (G_C(i) - G_C(i + e_a)) at the edge's first entry
template <class T>
__global__ void __launch_bounds__(kT) ad_vjp_beta(VjpGeom g, VjpBuffers bf, int a) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N;
    const double *X = bf.x + (int64_t)b * N;
    const double gam = bf.avimg[b].gamma;
    double *Y = bf.y + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
        if (g.L[a] > 1 && (p / g.S[a]) % g.L[a] + 1 < g.L[a]) {
            const int sg = an_edge_sign(g, bf, b, a, p);
            if (sg) v = -gam * g.w[a] * sg * (X[R[p]] - X[R[p + g.S[a]]]);
        }
        Y[p] = v;
    }
}

// The forward derivative's per-entry terms (tv_aniso.cpp:1362-1395):
// dx_i, minus gamma w_a dbeta_e sign_e for the edge leaving i, plus it for the
// edge entering i, summed per component afterwards.
template <class T>
__global__ void __launch_bounds__(kT) ad_jvp_terms(VjpGeom g, VjpBuffers bf, const T *__restrict__ dx,
                                                    const double *__restrict__ dbeta) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const double gam = bf.avimg[b].gamma;
    double *Y = bf.y + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        double t = dx ? (double)dx[(int64_t)b * N + p] : 0.0;
        if (dbeta)
            for (int a = 0; a < g.k; ++a) {
                if (g.L[a] <= 1) continue;
                const int64_t co = (p / g.S[a]) % g.L[a];
                if (co + 1 < g.L[a]) {
                    const int sf = an_edge_sign(g, bf, b, a, p);
                    if (sf) t -= gam * g.w[a] * dbeta[(int64_t)a * N + p] * sf;
                }
                if (co > 0) {
                    const int sb = an_edge_sign(g, bf, b, a, p - g.S[a]);
                    if (sb) t += gam * g.w[a] * dbeta[(int64_t)a * N + p - g.S[a]] * sb;
                }
            }
        Y[p] = t;
    }
}

// dz_C = (sum_C t - sum_a (dgamma w_a + gamma dw_a) S_{C,a}) / |C|, every
// entry its component's; the conjugate's dx - dz
template <class T>
__global__ void __launch_bounds__(kT) ad_jvp_out(VjpGeom g, VjpBuffers bf, const T *__restrict__ dx,
                                                  T *__restrict__ dz, double dgamma, JvpDir dir, int conj) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N, *Cn = bf.cnt + (int64_t)b * N;
    const double *Bv = bf.b + (int64_t)b * N;
    const double gam = bf.avimg[b].gamma;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const int r = R[p];
        double t = Bv[r];
        for (int a = 0; a < g.k; ++a)
            t -= (dgamma * g.w[a] + gam * dir.dw[a]) * bf.gz[((int64_t)b * g.k + a) * N + r];
        double v = t / (double)Cn[r];
        if (conj) v = (dx ? (double)dx[(int64_t)b * N + p] : 0.0) - v;
        dz[(int64_t)b * N + p] = (T)v;
    }
}

// ---- structure queries ----------------------------------------------------------

__device__ __forceinline__ bool q_nan(const VjpBuffers &bf, bool aniso, int b) {
    return aniso ? bf.aimg[b].mode == kAnNan : bf.img[b].mode == kModeNan;
}

// Labels in order of each region's first entry (its root, the smallest
// index): one block per image scans the roots in order; every other entry
// then takes its root's label.
__global__ void __launch_bounds__(1024) q_label_roots(VjpGeom g, VjpBuffers bf, bool aniso, int32_t *labels,
                                                      double *nreg) {
    __shared__ int wsum[32];
    __shared__ int base;
    const int b = blockIdx.x;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N;
    int32_t *Lb = labels + (int64_t)b * N;
    if (q_nan(bf, aniso, b)) {
        if (threadIdx.x == 0) nreg[b] = -1.0;
        return;
    }
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t c0 = 0; c0 < N; c0 += blockDim.x) {
        const int64_t i = c0 + threadIdx.x;
        const int f = (i < N && R[i] == i) ? 1 : 0;
        int x = f;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        if (f) Lb[i] = base + (wid > 0 ? wsum[wid - 1] : 0) + x - 1;
        __syncthreads();
        if (threadIdx.x == 0) base += wsum[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) nreg[b] = (double)base;
}

__global__ void __launch_bounds__(kT) q_label_rest(VjpGeom g, VjpBuffers bf, bool aniso, int32_t *labels) {
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const int *R = bf.root + (int64_t)b * N;
    int32_t *Lb = labels + (int64_t)b * N;
    const bool nan = q_nan(bf, aniso, b);
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        if (nan) Lb[p] = -1;
        else if (R[p] != p) Lb[p] = Lb[R[p]];
    }
}

// kink_image of isotropic TV (tv_iso.cpp:654-678): 1 where |(W D z)_p| <= tol
// and |u_p| >= gamma alpha_p - tol, for pixels of positive radius
template <class T>
__global__ void __launch_bounds__(kT) q_kinks_iso(VjpGeom g, VjpBuffers bf, const double *gam, double tol,
                                                  int8_t *mask) {
    const int b = blockIdx.y;
    const int64_t N = g.N, B = g.B;
    const int e = bf.img[b].e;
    const T *Q = static_cast<const T *>(bf.qd);
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const Px x = pix_of(g, p);
        const double z0 = ldexp(z_at<T>(g, bf, b, p), e);
        double gg = 0.0, uu = 0.0;
        for (int a = 0; a < g.k; ++a) {
            if (g.w[a] > 0.0 && x.co[a] + 1 < g.L[a]) {
                const double t = g.w[a] * (ldexp(z_at<T>(g, bf, b, p + g.S[a]), e) - z0);
                gg += t * t;
            }
            const double u = (double)Q[((int64_t)a * B + b) * N + p];
            uu += u * u;
        }
        double r = gam[b];
        if (bf.alpha) r *= (double)static_cast<const T *>(bf.alpha)[(int64_t)b * bf.alpha_stride + p];
        mask[(int64_t)b * N + p] = (int8_t)(r > 0.0 && sqrt(gg) <= tol && sqrt(uu) >= r - tol);
    }
}

// kink_image of anisotropic TV (tv_aniso.cpp:1318-1348) along axis a: bit a
// at the edge's first entry when its jump is within tol of 0 and its 1D dual
// within tol of its bound gamma w_a beta_e (edges of zero bound are free)
template <class T>
__global__ void __launch_bounds__(128) q_kinks_aniso(VjpGeom g, VjpBuffers bf, const double *gam, double tol, int a,
                                                     int8_t *mask) {
    const int b = blockIdx.y;
    const int64_t N = g.N, B = g.B, L = g.L[a], s = g.S[a];
    const double lam = gam[b] * g.w[a];
    if (!(lam > 0.0) || L == 1 || bf.aimg[b].mode == kAnNan) return;
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= N / L) return;
    const int64_t base = (f / s) * L * s + f % s;
    const int e = bf.aimg[b].e;
    const T *Q = static_cast<const T *>(bf.qd) + ((int64_t)a * B + b) * N;
    double acc = 0.0;
    double zi = ldexp(an_z<T>(g, bf, b, base), e);
    for (int64_t l = 0; l + 1 < L; ++l) {
        const int64_t i = base + l * s;
        acc += (double)Q[i];
        const double zn = ldexp(an_z<T>(g, bf, b, i + s), e);
        const double r = bf.beta ? lam * an_beta<T>(g, bf, a, i) : lam;
        if (r > 0.0 && fabs(zn - zi) <= tol && fabs(acc) >= r - tol)
            mask[(int64_t)b * N + i] = (int8_t)(mask[(int64_t)b * N + i] | (1 << a));
        zi = zn;
    }
}

struct ScatterDesc {
    int ndim;
    int64_t shape[8], st[8];
};

__global__ void scatter_kernel(const unsigned char *src, size_t esize, ScatterDesc d, int64_t n, unsigned char *dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = i, o = 0;
        for (int k = d.ndim - 1; k >= 0; --k) {
            o += (r % d.shape[k]) * d.st[k];
            r /= d.shape[k];
        }
        for (size_t j = 0; j < esize; ++j) dst[o * (int64_t)esize + (int64_t)j] = src[i * (int64_t)esize + (int64_t)j];
    }
}

int pblocks(const VjpGeom &g) {
    int64_t nb = (g.N + kT * 4 - 1) / (kT * 4);
    return (int)std::max<int64_t>(1, std::min<int64_t>(nb, 512));
}

template <class T>
cudaError_t structure_t(const VjpGeom &g, const VjpBuffers &bf, cudaStream_t s) {
    const dim3 grid(pblocks(g), (unsigned)g.B);
    st_flat<T><<<grid, kT, 0, s>>>(g, bf);
    st_union<<<grid, kT, 0, s>>>(g, bf);
    st_roots<<<grid, kT, 0, s>>>(g, bf);
    return cudaGetLastError();
}

// The system on the regions for a right-hand side (kind 0: the pixel vector
// gin; 3: the one in y): region sums, the Jacobi diagonal, and conjugate
// gradients in chunks of 8 iterations until every image has stopped.
template <class T>
cudaError_t solve_system(const VjpGeom &g, const VjpBuffers &bf, int kind, const T *gin, double tol, int max_iter,
                         cudaStream_t s, int *h_live, cudaEvent_t ev, int64_t &nl) {
    const dim3 grid(pblocks(g), (unsigned)g.B);
    rs_max<T><<<grid, kT, 0, s>>>(g, bf, kind, gin);
    rs_add<T><<<grid, kT, 0, s>>>(g, bf, kind, gin);
    rs_read<<<grid, kT, 0, s>>>(g, bf, kind, bf.b);
    jac_max<T><<<grid, kT, 0, s>>>(g, bf);
    jac_add<T><<<grid, kT, 0, s>>>(g, bf);
    rs_read<<<grid, kT, 0, s>>>(g, bf, 0, bf.dinv);
    cudaMemsetAsync(bf.live, 0, sizeof(int), s);
    cg_init<<<grid, kT, 0, s>>>(g, bf, tol, max_iter);
    nl += 7;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int chunk = 8;
    for (int it = 0; it < max_iter + chunk; it += chunk) {
        for (int j = 0; j < chunk; ++j) {
            cg_hg<T><<<grid, kT, 0, s>>>(g, bf);
            rs_max<T><<<grid, kT, 0, s>>>(g, bf, 1, gin);
            rs_add<T><<<grid, kT, 0, s>>>(g, bf, 1, gin);
            rs_read<<<grid, kT, 0, s>>>(g, bf, 1, bf.qv);
            cg_alpha<<<grid, kT, 0, s>>>(g, bf);
            cg_step<<<grid, kT, 0, s>>>(g, bf);
            cg_pv<<<grid, kT, 0, s>>>(g, bf);
            nl += 7;
        }
        e = cudaMemcpyAsync(h_live, bf.live, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaEventRecord(ev, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev);
        if (e != cudaSuccess) return e;
        if (*h_live == 0) break;
    }
    return cudaSuccess;
}

template <class T>
cudaError_t vjp_t(const VjpGeom &g, const VjpBuffers &bf, const void *gin, void *gx, double tol, int max_iter, int conj,
                  bool params, cudaStream_t s, int *h_live, cudaEvent_t ev, int64_t *launches) {
    const dim3 grid(pblocks(g), (unsigned)g.B);
    const T *gi = static_cast<const T *>(gin);
    int64_t nl = 0;
    cudaError_t e = solve_system<T>(g, bf, 0, gi, tol, max_iter, s, h_live, ev, nl);
    if (e != cudaSuccess) return e;
    vjp_out<T><<<grid, kT, 0, s>>>(g, bf, gi, static_cast<T *>(gx), conj);
    ++nl;
    if (params) {
        // r, y, h and qv are free once the gradients are solved
        tv1d_dual<T><<<grid, kT, 0, s>>>(g, bf, bf.r);
        vjp_params<T><<<grid, kT, 0, s>>>(g, bf, bf.r);
        param_sums<<<grid, kT, 0, s>>>(g, bf, 0, g.k > 1 ? 1 : -1);
        nl += 3;
        if (g.k > 2) {
            param_sums<<<grid, kT, 0, s>>>(g, bf, 2, -1);
            ++nl;
        }
        if (bf.alpha) {
            alpha_sum<<<pblocks(g), kT, 0, s>>>(g, bf, bf.qv);
            ++nl;
        }
    }
    if (launches) *launches = nl;
    return cudaGetLastError();
}

template <class T>
cudaError_t jvp_t(const VjpGeom &g, const VjpBuffers &bf, const void *dx, void *dz, double dgamma, const JvpDir &dir,
                  const double *dalpha, double tol, int max_iter, int conj, cudaStream_t s, int *h_live,
                  cudaEvent_t ev, int64_t *launches) {
    const dim3 grid(pblocks(g), (unsigned)g.B);
    const T *dxi = static_cast<const T *>(dx);
    int64_t nl = 0;
    // the single-axis duals into r, which the solve then overwrites
    tv1d_dual<T><<<grid, kT, 0, s>>>(g, bf, bf.r);
    jvp_terms<T><<<grid, kT, 0, s>>>(g, bf, dxi, dgamma, dir, dalpha, bf.r);
    jvp_rhs<<<grid, kT, 0, s>>>(g, bf);
    nl += 3;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = solve_system<T>(g, bf, 3, static_cast<const T *>(nullptr), tol, max_iter, s, h_live, ev, nl);
    if (e != cudaSuccess) return e;
    jvp_out<T><<<grid, kT, 0, s>>>(g, bf, dxi, static_cast<T *>(dz), conj);
    ++nl;
    if (launches) *launches = nl;
    return cudaGetLastError();
}

template <class T>
cudaError_t an_structure_t(const VjpGeom &g, const VjpBuffers &bf, cudaStream_t s) {
    const dim3 grid(pblocks(g), (unsigned)g.B);
    ad_bound<T><<<grid, kT, 0, s>>>(g, bf);
    for (int a = 0; a < g.k; ++a) {
        const int64_t nf = g.N / g.L[a];
        ad_codes<T><<<dim3((unsigned)((nf + 127) / 128), (unsigned)g.B), 128, 0, s>>>(g, bf, a);
    }
    ad_union<<<grid, kT, 0, s>>>(g, bf);
    st_roots<<<grid, kT, 0, s>>>(g, bf);
    // S_{C,a}: exact region sums of the edge terms, into gz at the roots
    for (int a = 0; a < g.k; ++a) {
        ad_term<T><<<grid, kT, 0, s>>>(g, bf, a);
        rs_max<T><<<grid, kT, 0, s>>>(g, bf, 3, static_cast<const T *>(nullptr));
        rs_add<T><<<grid, kT, 0, s>>>(g, bf, 3, static_cast<const T *>(nullptr));
        // read-out into a B x N slice, then to image-major k x N
        rs_read<<<grid, kT, 0, s>>>(g, bf, 3, bf.r);
        cudaError_t e = cudaMemcpy2DAsync(bf.gz + (int64_t)a * g.N, (size_t)g.k * g.N * sizeof(double), bf.r,
                                          (size_t)g.N * sizeof(double), (size_t)g.N * sizeof(double), (size_t)g.B,
                                          cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

template <class T>
cudaError_t an_vjp_t(const VjpGeom &g, const VjpBuffers &bf, const void *gin, void *gx, int conj, bool params,
                     double *gb, cudaStream_t s, int64_t *launches) {
    const dim3 grid(pblocks(g), (unsigned)g.B);
    const T *gi = static_cast<const T *>(gin);
    int64_t nl = 0;
    rs_max<T><<<grid, kT, 0, s>>>(g, bf, 0, gi);
    rs_add<T><<<grid, kT, 0, s>>>(g, bf, 0, gi);
    rs_read<<<grid, kT, 0, s>>>(g, bf, 0, bf.b);
    ad_vjp_out<T><<<grid, kT, 0, s>>>(g, bf, gi, static_cast<T *>(gx), conj);
    nl += 4;
    if (params) {
        param_sums<<<grid, kT, 0, s>>>(g, bf, 0, g.k > 1 ? 1 : -1);
        ++nl;
        if (g.k > 2) {
            param_sums<<<grid, kT, 0, s>>>(g, bf, 2, -1);
            ++nl;
        }
        if (bf.beta && gb) {
            for (int a = 0; a < g.k; ++a) {
                ad_vjp_beta<T><<<grid, kT, 0, s>>>(g, bf, a);
                alpha_sum<<<pblocks(g), kT, 0, s>>>(g, bf, bf.qv);
                nl += 2;
                cudaError_t e = cudaMemcpyAsync(gb + (int64_t)a * g.N, bf.qv, (size_t)g.N * sizeof(double),
                                                cudaMemcpyDeviceToHost, s);
                if (e != cudaSuccess) return e;
            }
        }
    }
    if (launches) *launches = nl;
    return cudaGetLastError();
}

template <class T>
cudaError_t an_jvp_t(const VjpGeom &g, const VjpBuffers &bf, const void *dx, void *dz, double dgamma,
                     const JvpDir &dir, const double *dbeta, int conj, cudaStream_t s, int64_t *launches) {
    const dim3 grid(pblocks(g), (unsigned)g.B);
    const T *dxi = static_cast<const T *>(dx);
    ad_jvp_terms<T><<<grid, kT, 0, s>>>(g, bf, dxi, dbeta);
    rs_max<T><<<grid, kT, 0, s>>>(g, bf, 3, static_cast<const T *>(nullptr));
    rs_add<T><<<grid, kT, 0, s>>>(g, bf, 3, static_cast<const T *>(nullptr));
    rs_read<<<grid, kT, 0, s>>>(g, bf, 3, bf.b);
    ad_jvp_out<T><<<grid, kT, 0, s>>>(g, bf, dxi, static_cast<T *>(dz), dgamma, dir, conj);
    if (launches) *launches = 5;
    return cudaGetLastError();
}

}  // namespace

cudaError_t vjp_structure(int dtype, const VjpGeom &g, const VjpBuffers &bf, cudaStream_t s) {
    return dtype == 1 ? structure_t<float>(g, bf, s) : structure_t<double>(g, bf, s);
}

cudaError_t vjp_solve(int dtype, const VjpGeom &g, const VjpBuffers &bf, const void *gin, void *gx, double tol,
                      int max_iter, int conj, bool params, cudaStream_t s, int *h_live, cudaEvent_t ev,
                      int64_t *launches) {
    return dtype == 1 ? vjp_t<float>(g, bf, gin, gx, tol, max_iter, conj, params, s, h_live, ev, launches)
                      : vjp_t<double>(g, bf, gin, gx, tol, max_iter, conj, params, s, h_live, ev, launches);
}

cudaError_t jvp_solve(int dtype, const VjpGeom &g, const VjpBuffers &bf, const void *dx, void *dz, double dgamma,
                      const JvpDir &dir, const double *dalpha, double tol, int max_iter, int conj, cudaStream_t s,
                      int *h_live, cudaEvent_t ev, int64_t *launches) {
    return dtype == 1 ? jvp_t<float>(g, bf, dx, dz, dgamma, dir, dalpha, tol, max_iter, conj, s, h_live, ev, launches)
                      : jvp_t<double>(g, bf, dx, dz, dgamma, dir, dalpha, tol, max_iter, conj, s, h_live, ev,
                                      launches);
}

}  // namespace fpb

namespace fpb {

cudaError_t an_vjp_structure(int dtype, const VjpGeom &g, const VjpBuffers &bf, cudaStream_t s) {
    return dtype == 1 ? an_structure_t<float>(g, bf, s) : an_structure_t<double>(g, bf, s);
}

cudaError_t an_vjp_solve(int dtype, const VjpGeom &g, const VjpBuffers &bf, const void *gin, void *gx, int conj,
                         bool params, double *gb, cudaStream_t s, int64_t *launches) {
    return dtype == 1 ? an_vjp_t<float>(g, bf, gin, gx, conj, params, gb, s, launches)
                      : an_vjp_t<double>(g, bf, gin, gx, conj, params, gb, s, launches);
}

cudaError_t an_jvp_solve(int dtype, const VjpGeom &g, const VjpBuffers &bf, const void *dx, void *dz, double dgamma,
                         const JvpDir &dir, const double *dbeta, int conj, cudaStream_t s, int64_t *launches) {
    return dtype == 1 ? an_jvp_t<float>(g, bf, dx, dz, dgamma, dir, dbeta, conj, s, launches)
                      : an_jvp_t<double>(g, bf, dx, dz, dgamma, dir, dbeta, conj, s, launches);
}

}  // namespace fpb

namespace fpb {

cudaError_t query_labels(bool aniso, const VjpGeom &g, const VjpBuffers &bf, int32_t *labels, double *nreg,
                         cudaStream_t s) {
    q_label_roots<<<(unsigned)g.B, 1024, 0, s>>>(g, bf, aniso, labels, nreg);
    q_label_rest<<<dim3(pblocks(g), (unsigned)g.B), kT, 0, s>>>(g, bf, aniso, labels);
    return cudaGetLastError();
}

cudaError_t query_kinks(int dtype, bool aniso, const VjpGeom &g, const VjpBuffers &bf, const double *gam,
                        double tol, int8_t *mask, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(mask, 0, (size_t)g.B * (size_t)g.N, s);
    if (e != cudaSuccess) return e;
    if (!aniso) {
        const dim3 grid(pblocks(g), (unsigned)g.B);
        if (dtype == 1) q_kinks_iso<float><<<grid, kT, 0, s>>>(g, bf, gam, tol, mask);
        else q_kinks_iso<double><<<grid, kT, 0, s>>>(g, bf, gam, tol, mask);
    } else {
        for (int a = 0; a < g.k; ++a) {
            const int64_t nf = g.N / g.L[a];
            const dim3 grid((unsigned)((nf + 127) / 128), (unsigned)g.B);
            if (dtype == 1) q_kinks_aniso<float><<<grid, 128, 0, s>>>(g, bf, gam, tol, a, mask);
            else q_kinks_aniso<double><<<grid, 128, 0, s>>>(g, bf, gam, tol, a, mask);
        }
    }
    return cudaGetLastError();
}

cudaError_t scatter_elements(const void *src, size_t esize, int ndim, const int64_t *shape, const int64_t *strides,
                             void *dst, cudaStream_t s) {
    if (ndim > 8) return cudaErrorInvalidValue;
    ScatterDesc d{};
    d.ndim = ndim;
    int64_t n = 1;
    for (int k = 0; k < ndim; ++k) {
        d.shape[k] = shape[k];
        d.st[k] = strides[k];
        n *= shape[k];
    }
    if (n == 0) return cudaSuccess;
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 4096);
    scatter_kernel<<<grid, 256, 0, s>>>(static_cast<const unsigned char *>(src), esize, d, n,
                                        static_cast<unsigned char *>(dst));
    return cudaGetLastError();
}

}  // namespace fpb
