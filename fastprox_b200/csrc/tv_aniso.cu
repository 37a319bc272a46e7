// Anisotropic image TV on sm_100a: the reference's own method, replayed per
// image on the device.
//
// Two active axes: the accelerated dual block proximal gradient method
// (ADBPG) of TVAniso::adbpg (src/ops/tv_aniso.cpp:429-530): per iteration an
// exact 1D TV prox of every fibre along the axis of smaller stride (a1) and
// then along the other (a2), the dual update with extrapolation, the gradient
// restart every 4 iterations (Restart, :357-367), gap checks on the adaptive
// CheckSchedule (:396-414), and the polish on the PolishSchedule (:382-391)
// that reads the flat regions off the dual and solves on them exactly
// (try_polish, :886-953). Three active axes: FDPG for three terms
// (TVAniso::fdpg3, :534-616). One active axis: a single exact pass.
//
// Each image carries a stage (iterate, check, polish, final, done); every
// kernel acts only on the images in its stage, and the last block of an
// image (a ticket per image) advances the stage with the scalar logic of the
// reference in FP64. The host issues the same round of launches until no
// image is live. The 1D steps are Condat's algorithm, one thread per fibre
// (tv1d.cuh). Components of the polish are found by union-find with atomic
// hooking of the larger root to the smaller (so every root is the smallest
// index of its component, whatever the order), and region sums use 64-bit
// fixed point, so every result is the same bit for bit on every run.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdlib>

#include "aniso.h"
#include "common.cuh"
#include "tv1d.cuh"

namespace fpb {
namespace {

constexpr int kCheck = 4;               // tv_aniso.cpp:76
constexpr double kPolishDrop = 0.1;     // :78
constexpr double kPolishEta = 1e-9;     // :81, for FP64 duals
// FP32 duals carry rounding near 1e-7 of the bound: the margin of the
// reference's own device path for float32, max(1e-9, 64 eps)
// (bindings/python/fastprox/_tv_torch.py dual_eta).
template <class T>
__device__ __forceinline__ double polish_eta() {
    return sizeof(T) == 4 ? 64.0 * 1.1920928955078125e-07 : kPolishEta;
}
constexpr double kPolishRatio = 0.01;   // :86
constexpr int kThreads = 256;

template <class T>
__device__ __forceinline__ T ldexp_t(T v, int e);
template <>
__device__ __forceinline__ float ldexp_t<float>(float v, int e) { return ldexpf(v, e); }
template <>
__device__ __forceinline__ double ldexp_t<double>(double v, int e) { return ldexp(v, e); }

struct Fib {
    int64_t s, L, nfib;
    __device__ __forceinline__ int64_t base(int64_t f) const { return (f / s) * L * s + (f % s); }
};

__device__ __forceinline__ Fib fibers(const AnGeom &g, int a) {
    Fib f;
    f.s = g.S[a];
    f.L = g.L[a];
    f.nfib = g.N / g.L[a];
    return f;
}

// The image of launch slot z in a round (-1: none, the live list is shorter).
__device__ __forceinline__ int round_image(const AnBuffers &bf, unsigned z) {
    if (!bf.lmap) return (int)z;
    return (int)z < *bf.lcnt ? bf.lmap[z] : -1;
}

// The live images in order (one block).
__global__ void __launch_bounds__(1024) an_live_list(const AnState *st, int64_t B, int *lmap, int *lcnt) {
    __shared__ int wsum[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t c0 = 0; c0 < B; c0 += blockDim.x) {
        const int64_t i = c0 + threadIdx.x;
        const int f = (i < B && st[i].status == kLive) ? 1 : 0;
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
        const int before = base + (wid > 0 ? wsum[wid - 1] : 0) + x - f;
        if (f) lmap[before] = (int)i;
        __syncthreads();
        if (threadIdx.x == 0) base += wsum[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) *lcnt = base;
}

__device__ __forceinline__ double *img_part(const AnBuffers &bf, int b) { return bf.part + (int64_t)b * bf.max_part * 2; }

// Ends a per-image reduction: block partial (two sums) to part, and in the
// last block of the image the totals. Returns true in thread 0 of that block.
__device__ __forceinline__ bool reduce2(const AnBuffers &bf, int b, unsigned blk, unsigned nblk, double a0,
                                        double a1, double *sh, int *flag, double &t0, double &t1) {
    const double s0 = block_sum(a0, sh);
    const double s1 = block_sum(a1, sh);
    double *part = img_part(bf, b);
    if (threadIdx.x == 0) {
        part[blk * 2 + 0] = s0;
        part[blk * 2 + 1] = s1;
    }
    if (!arrive_last(bf.ticket + b, nblk, flag)) return false;
    t0 = sum_partials(part, nblk, 2, 0, sh);
    t1 = sum_partials(part, nblk, 2, 1, sh);
    if (threadIdx.x != 0) return false;
    bf.ticket[b] = 0;
    return true;
}

// ---------------------------------------------------------------------------
// Set-up (tv_aniso.cpp:260-340)
// ---------------------------------------------------------------------------

template <class T>
__global__ void __launch_bounds__(kThreads) an_scan1(const T *__restrict__ x, AnGeom g, AnCall c, AnBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const T *xb = x + (int64_t)b * N;
    T *db = static_cast<T *>(bf.d) + (int64_t)b * N;
    double m = 0.0;
    int fl = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const T v = xb[i];
        if (xb != db) db[i] = v;
        const double a = fabs((double)v);
        if (isnan(a)) fl |= 1;
        else if (isinf(a)) fl |= 2;
        else m = fmax(m, a);
    }
    const double mb = block_max(m, sh);
    const double f1 = block_max((double)(fl & 1), sh);
    const double f2 = block_max((double)((fl >> 1) & 1), sh);
    double *part = img_part(bf, b);
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2 + 0] = mb;
        part[blockIdx.x * 2 + 1] = f1 + 2.0 * f2;
    }
    if (!arrive_last(bf.ticket + b, gridDim.x, &flag)) return;
    const double mx = max_partials(part, gridDim.x, 2, 0, sh);
    double o1 = 0.0, o2 = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
        const int code = (int)__ldcg(part + i * 2 + 1);
        o1 = fmax(o1, (double)(code & 1));
        o2 = fmax(o2, (double)((code >> 1) & 1));
    }
    o1 = block_max(o1, sh);
    o2 = block_max(o2, sh);
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    AnImage im{};
    im.gamma_in = bf.gammas[b];
    im.maxabs = mx;
    im.flags = (o1 > 0.0 ? 1 : 0) | (o2 > 0.0 ? 2 : 0);
    int na = 0;
    for (int a = 0; a < 3; ++a) {
        im.lam[a] = 0.0;
        if (a < g.k) {
            const double l = im.gamma_in * c.w[a];
            if (l > 0.0 && g.L[a] > 1) {
                im.lam[a] = l;
                ++na;
            }
        }
    }
    im.na = na;
    if (im.flags & 2) im.mode = kAnInf;
    else if (im.flags & 1) im.mode = kAnNan;
    else if (na == 0) im.mode = kAnIdentity;
    else if (na == 1) im.mode = kAnSingle;
    else im.mode = na == 2 ? kAnAdbpg : kAnFdpg3;
    int e = 0;
    if (na > 0 && mx > 0.0) {  // rescale_exponent (src/ops/image_util.hpp:56-65)
        const double gamma = im.gamma_in;
        e = ilogb(mx);
        if (e >= -64 && e <= 64) {
            e = 0;
        } else {
            const double top = fmax(gamma, gamma * c.step_scale);
            if (e < 0 && top > 0.0) e = min(0, max(e, ilogb(top) + 1 - 960));
        }
        for (int a = 0; a < 3 && e; ++a)
            if (im.lam[a] > 0.0 && !(ldexp(im.lam[a], -e) > 0.0)) e = 0;
    }
    im.e = e;
    for (int a = 0; a < 3; ++a) im.lam[a] = e ? ldexp(im.lam[a], -e) : im.lam[a];
    // the active axes of ADBPG: a1 of the smaller stride (tv_aniso.cpp:432-433)
    int act[3], n = 0;
    for (int a = 0; a < g.k; ++a)
        if (im.lam[a] > 0.0) act[n++] = a;
    im.a1 = n >= 2 ? (g.S[act[0]] < g.S[act[1]] ? act[0] : act[1]) : (n ? act[0] : 0);
    im.a2 = n >= 2 ? (im.a1 == act[0] ? act[1] : act[0]) : 0;
    // the fixed-point scale of the polish's region sums: |zp| <= max|d| + 2 k lam_max beta_max
    double lmax = 0.0;
    for (int a = 0; a < 3; ++a) lmax = fmax(lmax, im.lam[a]);
    const double zb = ldexp(mx, -e) + 2.0 * g.k * lmax * c.beta_max + 1e-300;
    int lgN = 0;
    while ((1LL << lgN) <= g.N) ++lgN;
    im.fx_shift = 61 - lgN - (ilogb(zb) + 1);
    bf.img[b] = im;
    AnState st{};
    st.status = (im.mode == kAnAdbpg || im.mode == kAnFdpg3) ? kLive : kFinished;
    st.stage = kStIter;
    st.tn = fista_t(1.0);
    st.beta = 0.0;
    st.gp = CUDART_INF;
    st.chk_next = 1;
    st.chk_prev_it = -1;
    st.pol_next = CUDART_INF;
    bf.st[b] = st;
    if (st.status == kLive) atomicAdd(bf.live, 1);
}

// d *= 2^-e, |d|^2 -> target (tv_aniso.cpp:329-337)
template <class T>
__global__ void __launch_bounds__(kThreads) an_scan2(AnGeom g, AnCall c, AnBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int mode = bf.img[b].mode;
    if (mode == kAnNan || mode == kAnInf) return;
    const int e = bf.img[b].e;
    T *db = static_cast<T *>(bf.d) + (int64_t)b * g.N;
    double s2 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.N; i += (int64_t)gridDim.x * blockDim.x) {
        T v = db[i];
        if (e) {
            v = ldexp_t(v, -e);
            db[i] = v;
        }
        s2 += (double)v * (double)v;
    }
    double t0, t1;
    if (!reduce2(bf, b, blockIdx.x, gridDim.x, s2, 0.0, sh, &flag, t0, t1)) return;
    bf.img[b].dd = t0;
    bf.img[b].target = c.tol * 0.5 * t0;
}

// ---------------------------------------------------------------------------
// Fibre passes of the iteration
// ---------------------------------------------------------------------------

// Edge weight of the edge (o, o + S[a]) times nothing (beta), or 1.
template <class T>
struct BetaW {
    const T *p;
    int64_t s;
    __device__ __forceinline__ double operator()(int64_t i) const { return (double)p[i * s]; }
};

// One exact 1D TV prox on fibre f of axis a of image b: in(i) -> out(i, v).
template <class T, class In, class Out>
__device__ __forceinline__ void fibre_prox(const AnCall &c, const AnBuffers &bf, int a, int64_t base, const Fib &fb,
                                           double lam, const In &in, const Out &out) {
    if (c.has_beta) {
        const T *bw = static_cast<const T *>(bf.beta) + (int64_t)a * c.N + base;
        tv1d_fiber<T>(in, out, (int)fb.L, lam, true, BetaW<T>{bw, fb.s}, DivRecip<T>{});
    } else {
        tv1d_fiber<T>(in, out, (int)fb.L, lam, false, NoWeight{}, DivRecip<T>{});
    }
}

// ADBPG first block step: u = prox_{g1}(d + w) along a1 (tv_aniso.cpp:459-460).
template <class T>
__global__ void __launch_bounds__(128) an_pass1(AnGeom g, AnCall c, AnBuffers bf) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || (st.stage != kStIter && st.stage != kStWarm)) return;
    const AnImage &im = bf.img[b];
    if (im.mode != kAnAdbpg) return;
    const int a = im.a1;
    const Fib fb = fibers(g, a);
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= fb.nfib) return;
    const int64_t N = g.N, base = fb.base(f), s = fb.s;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N + base;
    const T *Wv = static_cast<const T *>(bf.wv) + (int64_t)b * g.k * N + base;
    T *U = static_cast<T *>(bf.u) + (int64_t)b * N + base;
    auto in = [D, Wv, s](int64_t i) -> double { return (double)(D[i * s] + Wv[i * s]); };
    auto out = [U, s](int64_t i, double v) { U[i * s] = (T)v; };
    fibre_prox<T>(c, bf, a, base, fb, im.lam[a], in, out);
}

// ADBPG second block step along a2 with the dual update and extrapolation
// (tv_aniso.cpp:461-80); the last block runs the restart test, advances the
// iteration and decides whether a gap check is due.
template <class T>
__global__ void __launch_bounds__(128) an_pass2(AnGeom g, AnCall c, AnBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState st = bf.st[b];
    if (st.status != kLive || st.stage != kStIter) return;
    const AnImage &im = bf.img[b];
    if (im.mode != kAnAdbpg) return;
    const int a = im.a2;
    const Fib fb = fibers(g, a);
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t N = g.N;
    const bool test = st.it % kCheck == 0;
    const T beta = (T)st.beta;
    double up = 0.0;
    if (f < fb.nfib) {
        const int64_t base = fb.base(f), s = fb.s;
        const T *U = static_cast<const T *>(bf.u) + (int64_t)b * N + base;
        T *Wv = static_cast<T *>(bf.wv) + (int64_t)b * g.k * N + base;
        T *Y = static_cast<T *>(bf.y) + (int64_t)b * g.k * N + base;
        T *Z = static_cast<T *>(bf.z) + (int64_t)b * N + base;
        auto in = [U, Wv, s](int64_t i) -> double { return (double)(U[i * s] - Wv[i * s]); };
        auto out = [Z, s](int64_t i, double v) { Z[i * s] = (T)v; };
        fibre_prox<T>(c, bf, a, base, fb, im.lam[a], in, out);
        for (int64_t i = 0; i < fb.L; ++i) {
            const int64_t o = i * s;
            const T v = U[o] - Wv[o];
            const T yn = Z[o] - v;
            const T y = Y[o], w = Wv[o];
            if (test) up += (double)((w - yn) * (yn - y));
            Wv[o] = yn + beta * (yn - y);
            Y[o] = yn;
        }
    }
    double dot, unused;
    if (!reduce2(bf, b, blockIdx.x, gridDim.x, test ? up : 0.0, 0.0, sh, &flag, dot, unused)) return;
    AnState s2 = st;
    // Restart (tv_aniso.cpp:357-367): ++since; restart when test && up > 0 && since >= last
    s2.since += 1;
    double t = s2.tn;
    if (test && dot > 0.0 && s2.since >= s2.last) {
        s2.last = s2.since;
        s2.since = 0;
        s2.restart = 1;
        t = 1.0;
    } else {
        s2.restart = 0;
    }
    s2.it += 1;
    const double tn = fista_t(t);
    s2.beta = (t - 1.0) / tn;
    s2.tn = tn;
    if (s2.it == s2.chk_next || s2.it == c.max_iter) s2.stage = kStCheck;
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// Fibre tiles in shared memory
// ---------------------------------------------------------------------------
//
// A thread walking one fibre through global memory waits a memory latency at
// every step of Condat's scan (each step depends on the last), and a batch has
// only as many fibres as rows or columns: the passes above run latency-bound
// at a few percent of the memory bandwidth. The tiled passes copy the inputs of
// fb fibres (and their edge weights) into shared memory first, with loads
// that do not depend on one another and are coalesced (along the fibre when
// fibres are contiguous, across fibres otherwise), run the scans out of shared
// memory (the result overwrites the input: Condat never reads back an entry it
// has written), and store the results the same way. A tile is L x (fb + 1)
// entries (the odd row length keeps both copy directions free of bank
// conflicts; thread t of the scan always reads bank t + i mod 32). The values
// and their order of operations are those of the untiled passes.

struct TileCfg {
    int fb[3];  // fibres per block along each axis (0: the axis does not fit)
};

template <class T>
struct TileIn {
    const T *s;
    int P, t;
    __device__ __forceinline__ T operator()(int i) const { return s[i * P + t]; }
};
// A segment writes its value at its last entry and marks it (one bit per
// entry, word i / 32 of the fibre's column); finish fills each segment's
// other entries from its end, backwards, and clears the marks.
template <class T>
struct TileSink {
    T *s;
    unsigned *m;
    int P, t;
    __device__ __forceinline__ void segment(int, int k1, double v) const {
        s[k1 * P + t] = (T)v;
        m[(k1 >> 5) * P + t] |= 1u << (k1 & 31);
    }
    __device__ __forceinline__ void finish(int n) const {
        T v = T(0);
        for (int w = (n - 1) >> 5; w >= 0; --w) {
            const unsigned bits = m[w * P + t];
            m[w * P + t] = 0u;
            const int top = (w << 5) + 31 < n - 1 ? (w << 5) + 31 : n - 1;
            for (int i = top; i >= (w << 5); --i) {
                const int j = i * P + t;
                if (bits & (1u << (i & 31))) v = s[j];
                else s[j] = v;
            }
        }
    }
};

// tile[i][r] = ld(o) for the block's nv fibres, o the entry's offset in the image
template <class T, class Ld>
__device__ __forceinline__ void tile_load(T *tile, int P, const Fib &fb, int64_t f0, int nv, const Ld &ld) {
    const int L = (int)fb.L, n = nv * L;
    if (fb.s == 1) {
        for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
            const int r = idx / L, i = idx - r * L;
            tile[i * P + r] = ld(fb.base(f0 + r) + i);
        }
    } else {
        for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
            const int i = idx / nv, r = idx - i * nv;
            tile[i * P + r] = ld(fb.base(f0 + r) + (int64_t)i * fb.s);
        }
    }
}

// st(o, tile[i][r]) for the block's nv fibres, in the order of tile_load
template <class T, class St>
__device__ __forceinline__ void tile_store(const T *tile, int P, const Fib &fb, int64_t f0, int nv, const St &st) {
    const int L = (int)fb.L, n = nv * L;
    if (fb.s == 1) {
        for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
            const int r = idx / L, i = idx - r * L;
            st(fb.base(f0 + r) + i, tile[i * P + r]);
        }
    } else {
        for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
            const int i = idx / nv, r = idx - i * nv;
            st(fb.base(f0 + r) + (int64_t)i * fb.s, tile[i * P + r]);
        }
    }
}

// The tiles of a block in shared memory: the fibres' inputs (then results),
// their edge weights when there are any, one mark bit per entry, and the
// reciprocals 1/m (m <= L) of the scans.
template <class T>
struct Tiles {
    T *in, *w, *rc;
    unsigned *mk;
    __device__ __forceinline__ Tiles(unsigned char *smem, const AnCall &c, int L, int P) {
        in = reinterpret_cast<T *>(smem);
        w = in + L * P;
        mk = reinterpret_cast<unsigned *>(in + (c.has_beta ? 2 : 1) * L * P);
        const int nw = ((L + 31) >> 5) * P;
        rc = reinterpret_cast<T *>(mk + ((nw + 1) & ~1));
        for (int i = threadIdx.x; i < nw; i += blockDim.x) mk[i] = 0u;
        const DivRecip<T> div;
        for (int m = threadIdx.x; m <= L; m += blockDim.x) rc[m] = m ? div(m) : T(0);
    }
};

// Shared-memory bytes of a tile of fb fibres of L entries.
__host__ __device__ __forceinline__ size_t tile_bytes(int L, int fb, int nbuf, size_t tsize) {
    const size_t P = (size_t)fb + 1;
    const size_t nw = (((size_t)L + 31) / 32) * P;
    return (size_t)nbuf * tsize * (size_t)L * P + 4 * ((nw + 1) & ~(size_t)1) + tsize * ((size_t)L + 1);
}

// The scans of a loaded tile (edge weights in the second tile when present),
// by the block's first warp, lane t on fibre t, in lockstep (tv1d_warp).
template <class T>
__device__ __forceinline__ void tile_scan(const AnCall &c, const Tiles<T> &tl, int P, int nv, int L, double lam) {
    const int t = threadIdx.x;
    if (t >= 32) return;
    const TileIn<T> in{tl.in, P, t};
    const TileSink<T> out{tl.in, tl.mk, P, t};
    if (c.has_beta) tv1d_warp<T>(in, out, L, lam, true, TileIn<T>{tl.w, P, t}, TableRecip<T>{tl.rc}, t < nv);
    else tv1d_warp<T>(in, out, L, lam, false, NoWeight{}, TableRecip<T>{tl.rc}, t < nv);
}

// Threads of a tile block: all copy the tiles in and out, the first warp scans.
constexpr int kTileThreads = 128;

// an_pass1 on tiles
template <class T>
__global__ void __launch_bounds__(kTileThreads) an_pass1_tile(AnGeom g, AnCall c, AnBuffers bf, TileCfg tc) {
    extern __shared__ __align__(16) unsigned char an_smem[];
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || (st.stage != kStIter && st.stage != kStWarm)) return;
    const AnImage &im = bf.img[b];
    if (im.mode != kAnAdbpg) return;
    const int a = im.a1;
    const Fib fb = fibers(g, a);
    const int FB = tc.fb[a];
    const int64_t f0 = (int64_t)blockIdx.x * FB;
    if (f0 >= fb.nfib) return;
    const int nv = (int)(fb.nfib - f0 < FB ? fb.nfib - f0 : FB), P = FB + 1;
    const Tiles<T> tl(an_smem, c, (int)fb.L, P);
    const int64_t N = g.N;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Wv = static_cast<const T *>(bf.wv) + (int64_t)b * g.k * N;
    tile_load(tl.in, P, fb, f0, nv, [D, Wv](int64_t o) { return (T)(D[o] + Wv[o]); });
    if (c.has_beta) {
        const T *bw = static_cast<const T *>(bf.beta) + (int64_t)a * c.N;
        tile_load(tl.w, P, fb, f0, nv, [bw](int64_t o) { return bw[o]; });
    }
    __syncthreads();
    tile_scan(c, tl, P, nv, (int)fb.L, im.lam[a]);
    __syncthreads();
    T *U = static_cast<T *>(bf.u) + (int64_t)b * N;
    tile_store(tl.in, P, fb, f0, nv, [U](int64_t o, T v) { U[o] = v; });
}

// an_pass2 on tiles, with the dual update, the extrapolation and the restart
// logic of an_pass2
template <class T>
__global__ void __launch_bounds__(kTileThreads) an_pass2_tile(AnGeom g, AnCall c, AnBuffers bf, TileCfg tc) {
    extern __shared__ __align__(16) unsigned char an_smem[];
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState st = bf.st[b];
    if (st.status != kLive || st.stage != kStIter) return;
    const AnImage &im = bf.img[b];
    if (im.mode != kAnAdbpg) return;
    const int a = im.a2;
    const Fib fb = fibers(g, a);
    const int FB = tc.fb[a];
    const int64_t f0 = (int64_t)blockIdx.x * FB;
    const int64_t N = g.N;
    const bool test = st.it % kCheck == 0;
    const T beta = (T)st.beta;
    double up = 0.0;
    if (f0 < fb.nfib) {
        const int nv = (int)(fb.nfib - f0 < FB ? fb.nfib - f0 : FB), P = FB + 1;
        const Tiles<T> tl(an_smem, c, (int)fb.L, P);
        const T *U = static_cast<const T *>(bf.u) + (int64_t)b * N;
        T *Wv = static_cast<T *>(bf.wv) + (int64_t)b * g.k * N;
        T *Y = static_cast<T *>(bf.y) + (int64_t)b * g.k * N;
        T *Z = static_cast<T *>(bf.z) + (int64_t)b * N;
        tile_load(tl.in, P, fb, f0, nv, [U, Wv](int64_t o) { return (T)(U[o] - Wv[o]); });
        if (c.has_beta) {
            const T *bw = static_cast<const T *>(bf.beta) + (int64_t)a * c.N;
            tile_load(tl.w, P, fb, f0, nv, [bw](int64_t o) { return bw[o]; });
        }
        __syncthreads();
        tile_scan(c, tl, P, nv, (int)fb.L, im.lam[a]);
        __syncthreads();
        tile_store(tl.in, P, fb, f0, nv, [&](int64_t o, T z) {
            const T v = U[o] - Wv[o];
            const T yn = z - v;
            const T y = Y[o], w = Wv[o];
            if (test) up += (double)((w - yn) * (yn - y));
            Wv[o] = yn + beta * (yn - y);
            Y[o] = yn;
            Z[o] = z;
        });
    }
    double dot, unused;
    if (!reduce2(bf, b, blockIdx.x, gridDim.x, test ? up : 0.0, 0.0, sh, &flag, dot, unused)) return;
    AnState s2 = st;
    s2.since += 1;
    double t = s2.tn;
    if (test && dot > 0.0 && s2.since >= s2.last) {
        s2.last = s2.since;
        s2.since = 0;
        s2.restart = 1;
        t = 1.0;
    } else {
        s2.restart = 0;
    }
    s2.it += 1;
    const double tn = fista_t(t);
    s2.beta = (t - 1.0) / tn;
    s2.tn = tn;
    if (s2.it == s2.chk_next || s2.it == c.max_iter) s2.stage = kStCheck;
    bf.st[b] = s2;
}

// an_fdpg3_pass on tiles (blockIdx.y = axis)
template <class T>
__global__ void __launch_bounds__(kTileThreads) an_fdpg3_tile(AnGeom g, AnCall c, AnBuffers bf, TileCfg tc) {
    extern __shared__ __align__(16) unsigned char an_smem[];
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = round_image(bf, blockIdx.z);
    if (b < 0) return;
    const AnState st = bf.st[b];
    if (st.status != kLive || st.stage != kStIter) return;
    const AnImage &im = bf.img[b];
    if (im.mode != kAnFdpg3) return;
    const int64_t N = g.N;
    const bool test = st.it % kCheck == 0;
    const T beta = (T)st.beta;
    double up = 0.0;
    const int a = blockIdx.y;
    const Fib fb = fibers(g, a);
    const int FB = tc.fb[a];
    const int64_t f0 = (int64_t)blockIdx.x * FB;
    if (f0 < fb.nfib) {
        const int nv = (int)(fb.nfib - f0 < FB ? fb.nfib - f0 : FB), P = FB + 1;
        const Tiles<T> tl(an_smem, c, (int)fb.L, P);
        const T *U = static_cast<const T *>(bf.u) + (int64_t)b * N;
        T *Wa = static_cast<T *>(bf.wv) + ((int64_t)b * 3 + a) * N;
        T *Ya = static_cast<T *>(bf.y) + ((int64_t)b * 3 + a) * N;
        // the three axes write disjoint scratch: zp (a = 0), z (a = 1), dual slot (a = 2)
        T *Za = static_cast<T *>(bf.zp) + (int64_t)b * N;
        if (a == 1) Za = static_cast<T *>(bf.z) + (int64_t)b * N;
        if (a == 2) Za = static_cast<T *>(bf.scratch) + (int64_t)b * N;
        tile_load(tl.in, P, fb, f0, nv, [U, Wa](int64_t o) { return (T)(U[o] - T(3) * Wa[o]); });
        if (c.has_beta) {
            const T *bw = static_cast<const T *>(bf.beta) + (int64_t)a * c.N;
            tile_load(tl.w, P, fb, f0, nv, [bw](int64_t o) { return bw[o]; });
        }
        __syncthreads();
        tile_scan(c, tl, P, nv, (int)fb.L, 3.0 * im.lam[a]);
        __syncthreads();
        tile_store(tl.in, P, fb, f0, nv, [&](int64_t o, T z) {
            const T v = U[o] - T(3) * Wa[o];
            const T yn = (z - v) / T(3);
            const T y = Ya[o], w = Wa[o];
            if (test) up += (double)((w - yn) * (yn - y));
            Wa[o] = yn + beta * (yn - y);
            Ya[o] = yn;
            Za[o] = z;
        });
    }
    double dot, unused;
    const unsigned nblk = gridDim.x * gridDim.y;
    const unsigned blk = blockIdx.y * gridDim.x + blockIdx.x;
    if (!reduce2(bf, b, blk, nblk, test ? up : 0.0, 0.0, sh, &flag, dot, unused)) return;
    AnState s2 = st;
    s2.since += 1;
    double t = s2.tn;
    if (test && dot > 0.0 && s2.since >= s2.last) {
        s2.last = s2.since;
        s2.since = 0;
        s2.restart = 1;
        t = 1.0;
    } else {
        s2.restart = 0;
    }
    s2.it += 1;
    const double tn = fista_t(t);
    s2.beta = (t - 1.0) / tn;
    s2.tn = tn;
    if (s2.it % kCheck == 0 || s2.it == c.max_iter) s2.stage = kStCheck;
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// Fibre-major passes
// ---------------------------------------------------------------------------
//
// The fibre scans are long serial chains (each step of Condat's scan depends on
// the last), so a pass is bound by how many fibres an SM keeps in flight. The
// tiles above hold a block's fibres in shared memory, which caps an SM at a few
// dozen fibres. These passes keep every fibre of the launch in flight at once
// (a lane per fibre, 32 fibres a warp, in lockstep) and read the fibres through
// the L1 cache from a fibre-major copy, where each fibre's entries are
// contiguous: a lane's reads walk its own few cache lines. A pass is:
//  * stage: y of every fibre of the axis into ys, fibre-major (entry i of fibre
//    f at f L + i), through 32 x 32 tiles of shared memory (coalesced both
//    ways); a contiguous axis (stride 1) is fibre-major already, and its scan
//    reads the image arrays directly;
//  * scan: Condat's scan of every fibre (tv1d_warp); each segment's last entry
//    and value go to a list in the order the scan emits them (segk, segv);
//    after the scan each lane fills its fibre's entries from the list, into ys
//    in place (or, for the first pass over a contiguous axis, straight into u);
//  * unstage: the results back into the image's layout with the pass's
//    epilogue (the dual update and the restart test's sums for the second
//    pass), through the same tiles.
// The arithmetic of every step is the tiled passes'. The restart test's FP64
// sums are formed per tile block in a fixed order (its tiles, then the blocks),
// a partition that depends on the image's shape only.
// Edge weights along a strided axis are read from a fibre-major copy made once
// per workspace (an_weights_fm).

// The segments of a fibre's scan as a list in the order the scan emits them,
// which is their order along the fibre (a segment, once emitted, is final:
// the scan goes on from the entry after its end): entry q of the list holds
// the q-th segment's last entry and value. finish walks the list forwards and
// fills the fibre's entries; each segment's list entry is read one segment
// ahead, so the reads do not wait on one another.
template <class T>
struct SegSink {
    T *val;
    int *end;
    T *out;
    int *err;
    mutable int cnt = 0;  // segments emitted
    __device__ __forceinline__ void segment(int, int k1, double v) const {
        val[cnt] = (T)v;
        end[cnt] = k1;
        ++cnt;
    }
    __device__ __forceinline__ void finish(int n) const {
        int prev = -1;
        int e = cnt > 0 ? end[0] : -1;
        T v = cnt > 0 ? val[0] : T(0);
        for (int q = 0; q < cnt; ++q) {
            const int en = q + 1 < cnt ? end[q + 1] : -1;
            const T vn = q + 1 < cnt ? val[q + 1] : T(0);
            if (e <= prev || e >= n) break;  // not in order: a broken scan, flagged below
            for (int i = prev + 1; i <= e; ++i) out[i] = v;
            prev = e;
            e = en;
            v = vn;
        }
        if (prev != n - 1) atomicExch(err, 4);
        cnt = 0;
    }
};

// Entry i of a fibre-major fibre.
template <class T>
struct FmIn {
    const T *p;
    __device__ __forceinline__ T operator()(int i) const { return p[i]; }
};
// d + w (the first pass) or u - w (the second) of a contiguous fibre.
template <class T, int PASS>
struct SumIn {
    const T *a, *w;
    __device__ __forceinline__ T operator()(int i) const { return PASS == 1 ? (T)(a[i] + w[i]) : (T)(a[i] - w[i]); }
};

// Whether pass PASS of a round acts on image b (the stages of an_pass1 / an_pass2).
template <int PASS>
__device__ __forceinline__ bool fm_active(const AnState &st, const AnImage &im) {
    if (st.status != kLive || im.mode != kAnAdbpg) return false;
    return PASS == 1 ? (st.stage == kStIter || st.stage == kStWarm) : st.stage == kStIter;
}

constexpr int kFmTile = 32;     // tile of 32 fibres x 32 entries
constexpr int kFmThreads = 256; // 32 x 8 threads per tile block
constexpr int kFmScan = 128;    // threads per scan block
constexpr int kFmLanes = 8;     // fibres per warp of a scan block (its other lanes idle)

__host__ __device__ __forceinline__ int64_t fm_tiles(int64_t nfib, int64_t L) {
    return ((nfib + kFmTile - 1) / kFmTile) * ((L + kFmTile - 1) / kFmTile);
}

// ys = y of axis a's fibres, fibre-major (PASS 1: d + w along a1; 2: u - w along a2).
template <class T, int PASS>
__global__ void __launch_bounds__(kFmThreads) an_fm_stage(AnGeom g, AnCall c, AnBuffers bf) {
    __shared__ T tile[kFmTile][kFmTile + 1];
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnImage &im = bf.img[b];
    if (!fm_active<PASS>(bf.st[b], im)) return;
    const int a = PASS == 1 ? im.a1 : im.a2;
    const Fib fb = fibers(g, a);
    const int64_t N = g.N, L = fb.L;
    const T *P0 = static_cast<const T *>(PASS == 1 ? bf.d : bf.u) + (int64_t)b * N;
    const T *Wv = static_cast<const T *>(bf.wv) + (int64_t)b * g.k * N;
    T *Y = static_cast<T *>(bf.ys) + (int64_t)b * N;
    auto src = [&](int64_t o) -> T { return PASS == 1 ? (T)(P0[o] + Wv[o]) : (T)(P0[o] - Wv[o]); };
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int64_t neg = (L + kFmTile - 1) / kFmTile, nt = fm_tiles(fb.nfib, L);
    for (int64_t t = blockIdx.x; t < nt; t += gridDim.x) {
        const int64_t f0 = (t / neg) * kFmTile, i0 = (t % neg) * kFmTile;
#pragma unroll
        for (int r = 0; r < kFmTile; r += 8) {  // along the fibres (adjacent fibres are adjacent in memory)
            const int64_t f = f0 + tx, i = i0 + ty + r;
            tile[ty + r][tx] = (f < fb.nfib && i < L) ? src(fb.base(f) + i * fb.s) : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kFmTile; r += 8) {  // along each fibre
            const int64_t f = f0 + ty + r, i = i0 + tx;
            if (f < fb.nfib && i < L) Y[f * L + i] = tile[tx][ty + r];
        }
        __syncthreads();
    }
}

// Condat's scan of every fibre of the pass's axis, a lane per fibre.
// DIRECT: the axis is contiguous and the scan reads the image arrays (d + w,
// or u - w); the first pass then fills u, the second ys.
template <class T, int PASS, bool DIRECT>
__global__ void __launch_bounds__(kFmScan) an_fm_scan(AnGeom g, AnCall c, AnBuffers bf) {
    extern __shared__ __align__(16) unsigned char an_fm_smem[];
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnImage &im = bf.img[b];
    if (!fm_active<PASS>(bf.st[b], im)) return;
    const int a = PASS == 1 ? im.a1 : im.a2;
    const Fib fb = fibers(g, a);
    const int L = (int)fb.L;
    T *rc = reinterpret_cast<T *>(an_fm_smem);  // 1/m, m <= L
    {
        const DivRecip<T> div;
        for (int m = threadIdx.x; m <= L; m += blockDim.x) rc[m] = m ? div(m) : T(0);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t f = ((int64_t)blockIdx.x * (kFmScan / 32) + (threadIdx.x >> 5)) * kFmLanes + lane;
    const bool act = lane < kFmLanes && f < fb.nfib;
    const int64_t N = g.N, fo = act ? f * L : 0;  // fibre-major offset (the image offset when DIRECT)
    T *Y = static_cast<T *>(bf.ys) + (int64_t)b * N + fo;
    T *out = (DIRECT && PASS == 1) ? static_cast<T *>(bf.u) + (int64_t)b * N + fo : Y;
    const SegSink<T> sink{static_cast<T *>(bf.segv) + (int64_t)b * N + fo, bf.segk + (int64_t)b * N + fo, out, bf.err};
    const double lam = im.lam[a];
    const TableRecip<T> rcp{rc};
    auto run = [&](const auto &in) {
        if (c.has_beta) {
            const T *bw = static_cast<const T *>(fb.s == 1 ? bf.beta : bf.wt) + (int64_t)a * c.N + fo;
            tv1d_warp<T, true>(in, sink, L, lam, true, FmIn<T>{bw}, rcp, act);
        } else {
            tv1d_warp<T, true>(in, sink, L, lam, false, NoWeight{}, rcp, act);
        }
    };
    if (DIRECT) {
        const T *P0 = static_cast<const T *>(PASS == 1 ? bf.d : bf.u) + (int64_t)b * N + fo;
        const T *Wv = static_cast<const T *>(bf.wv) + (int64_t)b * g.k * N + fo;
        run(SumIn<T, PASS>{P0, Wv});
    } else {
        run(FmIn<T>{Y});
    }
}

// The scan's results back into the image's layout. PASS 1: u = z. PASS 2:
// z, and the dual update with the extrapolation (an_pass2's); the last block
// of the image runs the restart test and advances the iteration.
template <class T, int PASS>
__global__ void __launch_bounds__(kFmThreads) an_fm_unstage(AnGeom g, AnCall c, AnBuffers bf) {
    __shared__ T tile[kFmTile][kFmTile + 1];
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState st = bf.st[b];
    const AnImage &im = bf.img[b];
    if (!fm_active<PASS>(st, im)) return;
    const int a = PASS == 1 ? im.a1 : im.a2;
    const Fib fb = fibers(g, a);
    const int64_t N = g.N, L = fb.L;
    const T *Y = static_cast<const T *>(bf.ys) + (int64_t)b * N;
    T *U = static_cast<T *>(bf.u) + (int64_t)b * N;
    T *Wv = static_cast<T *>(bf.wv) + (int64_t)b * g.k * N;
    T *Yd = static_cast<T *>(bf.y) + (int64_t)b * g.k * N;
    T *Z = static_cast<T *>(bf.z) + (int64_t)b * N;
    const bool test = st.it % kCheck == 0;
    const T beta = (T)st.beta;
    double up = 0.0;
    auto put = [&](int64_t o, T z) {
        if (PASS == 1) {
            U[o] = z;
        } else {
            const T v = U[o] - Wv[o];
            const T yn = z - v;
            const T y = Yd[o], w = Wv[o];
            if (test) up += (double)((w - yn) * (yn - y));
            Wv[o] = yn + beta * (yn - y);
            Yd[o] = yn;
            Z[o] = z;
        }
    };
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    if (fb.s == 1) {  // fibre-major is the image's layout
        for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x)
            put(p, Y[p]);
    } else {
        const int64_t neg = (L + kFmTile - 1) / kFmTile, nt = fm_tiles(fb.nfib, L);
        for (int64_t t = blockIdx.x; t < nt; t += gridDim.x) {
            const int64_t f0 = (t / neg) * kFmTile, i0 = (t % neg) * kFmTile;
#pragma unroll
            for (int r = 0; r < kFmTile; r += 8) {  // along each fibre
                const int64_t f = f0 + ty + r, i = i0 + tx;
                tile[ty + r][tx] = (f < fb.nfib && i < L) ? Y[f * L + i] : T(0);
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < kFmTile; r += 8) {  // along the fibres
                const int64_t f = f0 + tx, i = i0 + ty + r;
                if (f < fb.nfib && i < L) put(fb.base(f) + i * fb.s, tile[tx][ty + r]);
            }
            __syncthreads();
        }
    }
    if (PASS == 1) return;
    double dot, unused;
    if (!reduce2(bf, b, blockIdx.x, gridDim.x, test ? up : 0.0, 0.0, sh, &flag, dot, unused)) return;
    AnState s2 = st;
    s2.since += 1;
    double t = s2.tn;
    if (test && dot > 0.0 && s2.since >= s2.last) {
        s2.last = s2.since;
        s2.since = 0;
        s2.restart = 1;
        t = 1.0;
    } else {
        s2.restart = 0;
    }
    s2.it += 1;
    const double tn = fista_t(t);
    s2.beta = (t - 1.0) / tn;
    s2.tn = tn;
    if (s2.it == s2.chk_next || s2.it == c.max_iter) s2.stage = kStCheck;
    bf.st[b] = s2;
}

// The edge weights of every strided axis, fibre-major (once per workspace).
template <class T>
__global__ void __launch_bounds__(kFmThreads) an_weights_fm(AnGeom g, const T *__restrict__ beta, T *__restrict__ wt) {
    __shared__ T tile[kFmTile][kFmTile + 1];
    const int a = blockIdx.y;
    const Fib fb = fibers(g, a);
    if (fb.s == 1) return;
    const int64_t N = g.N, L = fb.L;
    const T *Bw = beta + (int64_t)a * N;
    T *Wt = wt + (int64_t)a * N;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int64_t neg = (L + kFmTile - 1) / kFmTile, nt = fm_tiles(fb.nfib, L);
    for (int64_t t = blockIdx.x; t < nt; t += gridDim.x) {
        const int64_t f0 = (t / neg) * kFmTile, i0 = (t % neg) * kFmTile;
#pragma unroll
        for (int r = 0; r < kFmTile; r += 8) {
            const int64_t f = f0 + tx, i = i0 + ty + r;
            tile[ty + r][tx] = (f < fb.nfib && i < L) ? Bw[fb.base(f) + i * fb.s] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kFmTile; r += 8) {
            const int64_t f = f0 + ty + r, i = i0 + tx;
            if (f < fb.nfib && i < L) Wt[f * L + i] = tile[tx][ty + r];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Warm starts (tv_aniso.cpp:316-320, 436-486, 539-543, 630-684)
// ---------------------------------------------------------------------------

// feasible_dual along axis a, one thread per fibre: q_a at the solved scale
// (zero on an inactive axis); a fibre whose running sums -p_e stay within
// their bounds and end at 0 up to rounding is kept, any other rebuilt from
// its running sums clipped to [-lam_e, lam_e] (non-finite ones 0).
template <class T>
__global__ void __launch_bounds__(128) an_warm_feasible(AnGeom g, AnCall c, AnBuffers bf, int a) {
    const int b = blockIdx.y;
    const AnImage &im = bf.img[b];
    if (bf.st[b].status != kLive || (im.mode != kAnAdbpg && im.mode != kAnFdpg3)) return;
    const Fib fb = fibers(g, a);
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= fb.nfib) return;
    const int64_t N = g.N, B = g.B, base = fb.base(f), s = fb.s, L = fb.L;
    T *Q = static_cast<T *>(bf.dual) + ((int64_t)a * B + b) * N + base;
    const double lam = im.lam[a];
    const T *bw = c.has_beta ? static_cast<const T *>(bf.beta) + (int64_t)a * c.N + base : nullptr;
    if (!(lam > 0.0)) {
        for (int64_t l = 0; l < L; ++l) Q[l * s] = T(0);
        return;
    }
    double acc = 0.0, mass = 0.0, peak = -lam;
    for (int64_t l = 0; l < L; ++l) {
        const double q = im.e ? ldexp((double)Q[l * s], -im.e) : (double)Q[l * s];
        Q[l * s] = (T)q;
        acc += q;
        mass += fabs(q);
        const double e = l + 1 < L ? fabs(acc) - (bw ? lam * (double)bw[l * s] : lam) : -lam;
        peak = (e > peak || e != e) ? e : peak;
    }
    const double eps = sizeof(T) == 4 ? 1.1920928955078125e-07 : DBL_EPSILON;
    const double tol = 1e-10 * lam + 16.0 * eps * mass;
    if (isfinite(mass) && peak <= tol && fabs(acc) <= tol) return;
    double run = 0.0, prev = 0.0;
    for (int64_t l = 0; l < L; ++l) {
        const double qi = (double)Q[l * s];
        run += qi;
        double pe = 0.0;
        const double lb = (l + 1 < L && bw) ? lam * (double)bw[l * s] : lam;
        if (l + 1 < L && isfinite(run)) pe = fmin(fmax(-run, -lb), lb);
        Q[l * s] = (T)(prev - pe);
        prev = pe;
    }
}

// y = -q2 and z = d - q1 - q2 (ADBPG), y_a = -q_a (FDPG-3); w = y
template <class T>
__global__ void an_warm_init(AnGeom g, AnBuffers bf) {
    const int b = blockIdx.y;
    const AnImage &im = bf.img[b];
    if (bf.st[b].status != kLive || (im.mode != kAnAdbpg && im.mode != kAnFdpg3)) return;
    const int64_t N = g.N, B = g.B;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Q = static_cast<const T *>(bf.dual);
    T *Y = static_cast<T *>(bf.y) + (int64_t)b * g.k * N;
    T *Wv = static_cast<T *>(bf.wv) + (int64_t)b * g.k * N;
    T *Z = static_cast<T *>(bf.z) + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        if (im.mode == kAnAdbpg) {
            const T q1 = Q[((int64_t)im.a1 * B + b) * N + p], q2 = Q[((int64_t)im.a2 * B + b) * N + p];
            Y[p] = -q2;
            Wv[p] = -q2;
            Z[p] = D[p] - q1 - q2;
        } else {
            for (int a = 0; a < 3; ++a) {
                const T q = Q[((int64_t)a * B + b) * N + p];
                Y[(int64_t)a * N + p] = -q;
                Wv[(int64_t)a * N + p] = -q;
            }
        }
    }
}

// the first check at iteration 0
__global__ void an_warm_state(AnGeom g, AnBuffers bf) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.B) return;
    AnState &st = bf.st[b];
    const int mode = bf.img[b].mode;
    if (st.status != kLive || (mode != kAnAdbpg && mode != kAnFdpg3)) return;
    st.warm = 1;
    st.stage = kStCheck;
    st.wphase = mode == kAnAdbpg ? 1 : 0;
}

// The warm pass's dual (tv_aniso.cpp:443-449): q1 = d + y - u, q2 = -y and
// z = d - q1 - q2, for the second check.
template <class T>
__global__ void an_warm_z(AnGeom g, AnBuffers bf) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || st.stage != kStWarm) return;
    const int64_t N = g.N;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Y = static_cast<const T *>(bf.y) + (int64_t)b * g.k * N;
    const T *U = static_cast<const T *>(bf.u) + (int64_t)b * N;
    T *Z = static_cast<T *>(bf.z) + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const T q1 = D[p] + Y[p] - U[p], q2 = -Y[p];
        Z[p] = D[p] - q1 - q2;
    }
}

__global__ void an_warm_next(AnGeom g, AnBuffers bf) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.B) return;
    AnState &st = bf.st[b];
    if (st.status == kLive && st.stage == kStWarm) st.stage = kStCheck;
}

// After a restart the extrapolated dual restarts from y (tv_aniso.cpp:474-477).
template <class T>
__global__ void an_restart_copy(AnGeom g, AnBuffers bf) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || !st.restart) return;
    const int64_t n = (int64_t)g.k * g.N;
    const T *Y = static_cast<const T *>(bf.y) + (int64_t)b * n;
    T *Wv = static_cast<T *>(bf.wv) + (int64_t)b * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        Wv[i] = Y[i];
}

// FDPG-3 (tv_aniso.cpp:534-616): u = d + w0 + w1 + w2, then for each axis a
// y_a+ = (prox_{3 g_a}(u - 3 w_a) - (u - 3 w_a)) / 3 and the extrapolation.
template <class T>
__global__ void an_fdpg3_u(AnGeom g, AnBuffers bf) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || st.stage != kStIter || bf.img[b].mode != kAnFdpg3) return;
    const int64_t N = g.N;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Wv = static_cast<const T *>(bf.wv) + (int64_t)b * 3 * N;
    T *U = static_cast<T *>(bf.u) + (int64_t)b * N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        U[i] = D[i] + Wv[i] + Wv[N + i] + Wv[2 * N + i];
}

template <class T>
__global__ void __launch_bounds__(128) an_fdpg3_pass(AnGeom g, AnCall c, AnBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = round_image(bf, blockIdx.z);
    if (b < 0) return;
    const AnState st = bf.st[b];
    if (st.status != kLive || st.stage != kStIter) return;
    const AnImage &im = bf.img[b];
    if (im.mode != kAnFdpg3) return;
    const int64_t N = g.N;
    const bool test = st.it % kCheck == 0;
    const T beta = (T)st.beta;
    double up = 0.0;
    // blockIdx.y = axis; the fibres of all three axes in one launch
    const int a = blockIdx.y;
    const Fib fb = fibers(g, a);
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f < fb.nfib) {
        const int64_t base = fb.base(f), s = fb.s;
        const T *U = static_cast<const T *>(bf.u) + (int64_t)b * N + base;
        T *Wa = static_cast<T *>(bf.wv) + ((int64_t)b * 3 + a) * N + base;
        T *Ya = static_cast<T *>(bf.y) + ((int64_t)b * 3 + a) * N + base;
        T *Zs = static_cast<T *>(bf.zp) + (int64_t)b * N;  // scratch: z of this axis' fibres
        T *Za = Zs + base;
        // the three axes write disjoint scratch: zp (a = 0), z (a = 1), dual slot (a = 2)
        if (a == 1) Za = static_cast<T *>(bf.z) + (int64_t)b * N + base;
        if (a == 2) Za = static_cast<T *>(bf.scratch) + (int64_t)b * N + base;
        auto in = [U, Wa, s](int64_t i) -> double { return (double)(U[i * s] - T(3) * Wa[i * s]); };
        auto out = [Za, s](int64_t i, double v) { Za[i * s] = (T)v; };
        fibre_prox<T>(c, bf, a, base, fb, 3.0 * im.lam[a], in, out);
        for (int64_t i = 0; i < fb.L; ++i) {
            const int64_t o = i * s;
            const T v = U[o] - T(3) * Wa[o];
            const T yn = (Za[o] - v) / T(3);
            const T y = Ya[o], w = Wa[o];
            if (test) up += (double)((w - yn) * (yn - y));
            Wa[o] = yn + beta * (yn - y);
            Ya[o] = yn;
        }
    }
    double dot, unused;
    const unsigned nblk = gridDim.x * gridDim.y;
    const unsigned blk = blockIdx.y * gridDim.x + blockIdx.x;
    if (!reduce2(bf, b, blk, nblk, test ? up : 0.0, 0.0, sh, &flag, dot, unused)) return;
    AnState s2 = st;
    s2.since += 1;
    double t = s2.tn;
    if (test && dot > 0.0 && s2.since >= s2.last) {
        s2.last = s2.since;
        s2.since = 0;
        s2.restart = 1;
        t = 1.0;
    } else {
        s2.restart = 0;
    }
    s2.it += 1;
    const double tn = fista_t(t);
    s2.beta = (t - 1.0) / tn;
    s2.tn = tn;
    if (s2.it % kCheck == 0 || s2.it == c.max_iter) s2.stage = kStCheck;
    bf.st[b] = s2;
}

// FDPG-3's primal at a check: z = prox_{g_c}(d + y_0 + y_1) along the
// contiguous axis c = 2 (tv_aniso.cpp:118-123).
template <class T>
__global__ void __launch_bounds__(128) an_fdpg3_primal(AnGeom g, AnCall c, AnBuffers bf, int stage) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || st.stage != stage) return;
    const AnImage &im = bf.img[b];
    if (im.mode != kAnFdpg3) return;
    const Fib fb = fibers(g, 2);
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= fb.nfib) return;
    const int64_t N = g.N, base = fb.base(f), s = fb.s;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N + base;
    const T *Y0 = static_cast<const T *>(bf.y) + (int64_t)b * 3 * N + base;
    const T *Y1 = Y0 + N;
    T *Z = static_cast<T *>(bf.z) + (int64_t)b * N + base;
    auto in = [D, Y0, Y1, s](int64_t i) -> double { return (double)(D[i * s] + Y0[i * s] + Y1[i * s]); };
    auto out = [Z, s](int64_t i, double v) { Z[i * s] = (T)v; };
    fibre_prox<T>(c, bf, 2, base, fb, im.lam[2], in, out);
}

// ---------------------------------------------------------------------------
// The gap of a point: sum_a lam_e |z_j - z_i| - <z, d - z> (tv_aniso.cpp:192-226)
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ double tv_at(const AnGeom &g, const AnCall &c, const AnBuffers &bf, const AnImage &im,
                                        const T *Z, int64_t p, int64_t Nimg) {
    double s = 0.0;
    for (int a = 0; a < g.k; ++a) {
        const double l = im.lam[a];
        if (l == 0.0) continue;
        const int64_t co = (p / g.S[a]) % g.L[a];
        if (co + 1 >= g.L[a]) continue;
        double le = l;
        if (c.has_beta) le = l * (double)static_cast<const T *>(bf.beta)[(int64_t)a * Nimg + p];
        s += le * fabs((double)Z[p + g.S[a]] - (double)Z[p]);
    }
    return s;
}

// The stage after a check (and its polish, if any) that left the image
// unconverged. In the loop: CheckSchedule::done for ADBPG, then iterate (or
// finish at max_iter). A warm start's first check is followed by its pass
// (ADBPG) and second check, which take no part in the schedule
// (tv_aniso.cpp:473-486).
__device__ __forceinline__ void after_check(AnState &s2, const AnImage &im, bool last) {
    if (s2.wphase == 1 && im.mode == kAnAdbpg) {
        s2.wphase = 2;
        s2.stage = kStWarm;
        return;
    }
    if (s2.wphase != 0) {
        s2.wphase = 0;
    } else if (im.mode == kAnAdbpg) {
        check_done(s2, s2.gp, im.target);
    }
    s2.stage = last ? kStFinal : kStIter;
}

// stage kStCheck: the gap of z; kStFinal: the gap of zp (the final rebuild).
template <class T>
__global__ void __launch_bounds__(kThreads) an_gap(AnGeom g, AnCall c, AnBuffers bf, int stage) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState st = bf.st[b];
    if (st.status != kLive || st.stage != stage) return;
    if (stage == kStFinal && (st.polished || st.it == 0 || bf.img[b].mode != kAnAdbpg)) return;
    const AnImage im = bf.img[b];
    const int64_t N = g.N;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Z = static_cast<const T *>(stage == kStCheck ? bf.z : bf.zp) + (int64_t)b * N;
    double acc = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const double z = (double)Z[p];
        acc += tv_at<T>(g, c, bf, im, Z, p, N) - z * ((double)D[p] - z);
    }
    double gz, unused;
    if (!reduce2(bf, b, blockIdx.x, gridDim.x, acc, 0.0, sh, &flag, gz, unused)) return;
    AnState s2 = st;
    if (stage == kStFinal) {
        // d - q1 - q2 in place of the iterate, unless rounding alone takes its
        // gap over the target (tv_aniso.cpp:87-96)
        if (gz <= im.target || !(s2.gp <= im.target)) {
            s2.zsel = 1;
            s2.gp = gz;
        }
        s2.stage = kStDone;
        bf.st[b] = s2;
        return;
    }
    const bool last = s2.it == c.max_iter;
    s2.gz = gz;
    if (gz <= im.target) {
        s2.gp = gz;
        s2.stage = kStFinal;
    } else if (last ? !s2.polished
                    : (im.mode == kAnAdbpg ? ((s2.warm || s2.it >= kCheck) && gz <= s2.pol_next) : gz <= s2.pol_next)) {
        s2.accept = last ? gz : im.target;
        s2.stage = kStPolish;
    } else {
        s2.gp = gz;
        after_check(s2, im, last);
    }
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// The polish (tv_aniso.cpp:630-953)
// ---------------------------------------------------------------------------

// dual(z) (tv_aniso.cpp:443-449, 124-131) into the dual, and the polish's
// scratch reset: zp = d, flags 0, parent = self, sums 0.
// stage kStPolish: for a polish; kStFinal: the final rebuild zp = d - q1 - q2.
template <class T>
__global__ void an_dual(AnGeom g, AnBuffers bf, int stage) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || st.stage != stage) return;
    if (stage == kStFinal && (st.polished || st.it == 0)) return;
    const AnImage &im = bf.img[b];
    const int64_t N = g.N, B = g.B;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Z = static_cast<const T *>(bf.z) + (int64_t)b * N;
    const T *Y = static_cast<const T *>(bf.y) + (int64_t)b * g.k * N;
    T *Q = static_cast<T *>(bf.dual);
    T *ZP = static_cast<T *>(bf.zp) + (int64_t)b * N;
    uint8_t *F = bf.flag + (int64_t)b * N;
    int *P = bf.parent + (int64_t)b * N;
    unsigned long long *S = bf.sum + (int64_t)b * N;
    int *C = bf.cnt + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        T q[3] = {T(0), T(0), T(0)};
        if (im.mode == kAnAdbpg) {
            q[im.a1] = D[p] + Y[p] - Z[p];
            q[im.a2] = -Y[p];
        } else {
            q[0] = -Y[p];
            q[1] = -Y[N + p];
            q[2] = D[p] + Y[p] + Y[N + p] - Z[p];
        }
        for (int a = 0; a < g.k; ++a) Q[((int64_t)a * B + b) * N + p] = q[a];
        if (stage == kStFinal) {
            if (im.mode == kAnAdbpg) {
                T s = T(0);
                for (int a = 0; a < g.k; ++a) s += q[a];
                ZP[p] = D[p] - s;
            }
        } else {
            ZP[p] = D[p];
            F[p] = 0;
            P[p] = (int)p;
            S[p] = 0ull;
            C[p] = 0;
        }
    }
}

// mark_edges (tv_aniso.cpp:256-297) along axis a: the 1D dual of each edge
// from the running sum of q_a along its fibre; an edge strictly inside its
// bound is flat (bit a), the others move lam_e sign(p_e) from j to i in zp.
template <class T>
__global__ void __launch_bounds__(128) an_mark(AnGeom g, AnCall c, AnBuffers bf, int a) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || st.stage != kStPolish) return;
    const AnImage &im = bf.img[b];
    const double lam = im.lam[a];
    if (lam == 0.0) return;
    const Fib fb = fibers(g, a);
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= fb.nfib) return;
    const int64_t N = g.N, base = fb.base(f), s = fb.s;
    const T *Q = static_cast<const T *>(bf.dual) + ((int64_t)a * g.B + b) * N + base;
    const T *Bw = c.has_beta ? static_cast<const T *>(bf.beta) + (int64_t)a * N + base : nullptr;
    T *ZP = static_cast<T *>(bf.zp) + (int64_t)b * N + base;
    uint8_t *F = bf.flag + (int64_t)b * N + base;
    const uint8_t bit = (uint8_t)(1u << a);
    double acc = 0.0;
    // zp of the edge's first entry is carried in a register from the last
    // edge (which may have changed it), so no step waits on its own store
    T zc = ZP[0];
    for (int64_t l = 0; l + 1 < fb.L; ++l) {
        const int64_t o = l * s;
        T zn = ZP[o + s];
        acc += (double)Q[o];
        const double pe = -acc;
        const double lb = Bw ? lam * (double)Bw[o] : lam;
        const bool inside = fabs(pe) < lb * (1.0 - polish_eta<T>());
        if (inside) {
            F[o] |= bit;
        } else {
            const double ls = copysign(lb, pe);
            zc = (T)((double)zc + ls);
            zn = (T)((double)zn - ls);
        }
        ZP[o] = zc;
        zc = zn;
    }
    ZP[(fb.L - 1) * s] = zc;
}

__device__ __forceinline__ int uf_find(int *P, int i) {
    // parents point to smaller indices, so the walk ends; path halving
    for (int n = 0; n < (1 << 30); ++n) {
        const int p = P[i];
        if (p == i) return i;
        const int q = P[p];
        if (q != p) P[i] = q;
        i = p;
    }
    return i;
}

// components (tv_aniso.cpp:324-439) by union-find: the flat edges join
// their ends, the larger root hooked under the smaller by compare-and-swap,
// so each root is the smallest index of its component.
__global__ void an_union(AnGeom g, AnBuffers bf) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || st.stage != kStPolish) return;
    const int64_t N = g.N;
    const uint8_t *F = bf.flag + (int64_t)b * N;
    int *P = bf.parent + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t fl = F[p];
        if (!fl) continue;
        for (int a = 0; a < g.k; ++a) {
            if (!(fl & (1u << a))) continue;
            int x = (int)p, y = (int)(p + g.S[a]);
            int tries = 0;
            for (;;) {
                x = uf_find(P, x);
                y = uf_find(P, y);
                if (x == y) break;
                const int hi = x > y ? x : y, lo = x > y ? y : x;
                const int old = atomicCAS(P + hi, hi, lo);
                if (old == hi) break;
                x = old;  // hi was hooked meanwhile: retry from there
                y = lo;
                if (++tries > (1 << 24)) {
                    atomicExch(bf.err, 2);
                    break;
                }
            }
        }
    }
}

// The root of i by a walk that writes nothing (parents point to smaller
// indices, so it ends). After the unions, each thread stores its own
// entry's root only: a halving write here could put a stale, non-root
// ancestor over an entry whose root another thread has already stored.
__device__ __forceinline__ int uf_root(const int *P, int i) {
    for (int n = 0; n < (1 << 30); ++n) {
        const int p = P[i];
        if (p == i) return i;
        i = p;
    }
    return i;
}

// every entry to its root; the region sums of zp (64-bit fixed point) and sizes
template <class T>
__global__ void an_region_sum(AnGeom g, AnBuffers bf) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || st.stage != kStPolish) return;
    const int64_t N = g.N;
    const int sh = bf.img[b].fx_shift;
    int *P = bf.parent + (int64_t)b * N;
    const T *ZP = static_cast<const T *>(bf.zp) + (int64_t)b * N;
    unsigned long long *S = bf.sum + (int64_t)b * N;
    int *C = bf.cnt + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const int r = uf_root(P, (int)p);
        P[p] = r;
        const long long fx = llrint(ldexp((double)ZP[p], sh));
        atomicAdd(S + r, (unsigned long long)fx);
        atomicAdd(C + r, 1);
    }
}

// zp = the region means; the polished gap P(zp) - D(q) (tv_aniso.cpp:504-523);
// the last block accepts or schedules the next attempt (:520-523, :382-391).
template <class T>
__global__ void __launch_bounds__(kThreads) an_polish_gap(AnGeom g, AnCall c, AnBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState st = bf.st[b];
    if (st.status != kLive || st.stage != kStPolish) return;
    const AnImage im = bf.img[b];
    const int64_t N = g.N, B = g.B;
    const int shf = im.fx_shift;
    const int *P = bf.parent + (int64_t)b * N;
    const unsigned long long *S = bf.sum + (int64_t)b * N;
    const int *C = bf.cnt + (int64_t)b * N;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Q = static_cast<const T *>(bf.dual);
    T *ZP = static_cast<T *>(bf.zp) + (int64_t)b * N;
    auto mean = [&](int64_t p) -> double {
        const int r = P[p];
        return ldexp((double)(long long)S[r], -shf) / (double)C[r];
    };
    double acc = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const double zp = mean(p);
        const double d = (double)D[p];
        const double e = zp - d;
        double sj = 0.0;
        for (int a = 0; a < g.k; ++a) sj += (double)Q[((int64_t)a * B + b) * N + p];
        double tv = 0.0;
        for (int a = 0; a < g.k; ++a) {
            const double l = im.lam[a];
            if (l == 0.0) continue;
            const int64_t co = (p / g.S[a]) % g.L[a];
            if (co + 1 >= g.L[a]) continue;
            double le = l;
            if (c.has_beta) le = l * (double)static_cast<const T *>(bf.beta)[(int64_t)a * N + p];
            tv += le * fabs(mean(p + g.S[a]) - zp);
        }
        acc += 0.5 * e * e - (d * sj - 0.5 * sj * sj) + tv;
    }
    // write the means after every block of this image has read them: the
    // last block does it (below); here only the gap
    double pz, unused;
    if (!reduce2(bf, b, blockIdx.x, gridDim.x, acc, 0.0, sh, &flag, pz, unused)) return;
    (void)ZP;
    AnState s2 = st;
    const double gz = s2.gz;
    const bool last = s2.it == c.max_iter;
    if (pz <= s2.accept && pz <= kPolishRatio * gz) {
        s2.polished = 1;
        s2.zsel = 1;
        s2.gp = pz;
        s2.pol_accept = 1;
    } else {
        // PolishSchedule::done (tv_aniso.cpp:386-390)
        const bool eager = im.mode == kAnFdpg3;
        double next = gz * kPolishDrop;
        if (pz > 0.0 && pz < (eager ? 1.0 : kPolishRatio) * gz) next = fmax(next, im.target * gz / pz);
        s2.pol_next = next;
        s2.gp = gz;
        s2.pol_accept = 0;
    }
    if (s2.gp <= im.target) s2.stage = kStFinal;
    else after_check(s2, im, last);
    bf.st[b] = s2;
}

// the accepted candidate: zp = region means
template <class T>
__global__ void an_polish_write(AnGeom g, AnBuffers bf) {
    const int b = round_image(bf, blockIdx.y);
    if (b < 0) return;
    const AnState &st = bf.st[b];
    if (st.status != kLive || !st.pol_accept) return;
    const int64_t N = g.N;
    const int shf = bf.img[b].fx_shift;
    const int *P = bf.parent + (int64_t)b * N;
    const unsigned long long *S = bf.sum + (int64_t)b * N;
    const int *C = bf.cnt + (int64_t)b * N;
    T *ZP = static_cast<T *>(bf.zp) + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const int r = P[p];
        ZP[p] = (T)(ldexp((double)(long long)S[r], -shf) / (double)C[r]);
    }
}

// images whose stage is done leave the live set
__global__ void an_retire(AnGeom g, AnBuffers bf) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.B) return;
    AnState &st = bf.st[b];
    st.pol_accept = 0;
    if (st.status == kLive && (st.stage == kStDone || (st.stage == kStFinal && bf.img[b].mode == kAnFdpg3))) {
        st.status = st.gp <= bf.img[b].target ? kConverged : kNotConv;
        atomicSub(bf.live, 1);
    }
}

// a final rebuild is not needed after a polish or at it = 0: done
__global__ void an_final_skip(AnGeom g, AnBuffers bf) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.B) return;
    AnState &st = bf.st[b];
    if (st.status == kLive && st.stage == kStFinal && (st.polished || st.it == 0)) st.stage = kStDone;
}

// ---------------------------------------------------------------------------
// Single active axis, identity, NaN; the output at the input's scale
// ---------------------------------------------------------------------------

template <class T>
__global__ void __launch_bounds__(128) an_single(AnGeom g, AnCall c, AnBuffers bf) {
    const int b = blockIdx.y;
    const AnImage &im = bf.img[b];
    if (im.mode != kAnSingle) return;
    int a = 0;
    for (int x = 0; x < g.k; ++x)
        if (im.lam[x] > 0.0) a = x;
    const Fib fb = fibers(g, a);
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= fb.nfib) return;
    const int64_t N = g.N, base = fb.base(f), s = fb.s;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N + base;
    T *Z = static_cast<T *>(bf.z) + (int64_t)b * N + base;
    auto in = [D, s](int64_t i) -> double { return (double)D[i * s]; };
    auto out = [Z, s](int64_t i, double v) { Z[i * s] = (T)v; };
    fibre_prox<T>(c, bf, a, base, fb, im.lam[a], in, out);
}

template <class T>
__global__ void an_output(AnGeom g, AnBuffers bf, T *__restrict__ out) {
    const int b = blockIdx.y;
    const AnImage im = bf.img[b];
    if (im.mode == kAnInf) return;
    const AnState st = bf.st[b];
    const int64_t N = g.N, B = g.B;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *Z = static_cast<const T *>(st.zsel ? bf.zp : bf.z) + (int64_t)b * N;
    T *Q = static_cast<T *>(bf.dual);
    T *O = out + (int64_t)b * N;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        if (im.mode == kAnNan) {
            O[p] = (T)CUDART_NAN;
            for (int a = 0; a < g.k; ++a) Q[((int64_t)a * B + b) * N + p] = (T)CUDART_NAN;
        } else if (im.mode == kAnIdentity) {
            O[p] = D[p];
            for (int a = 0; a < g.k; ++a) Q[((int64_t)a * B + b) * N + p] = T(0);
        } else if (im.mode == kAnSingle) {
            const T z = Z[p];
            O[p] = im.e ? ldexp_t(z, im.e) : z;
            for (int a = 0; a < g.k; ++a) {
                T q = im.lam[a] > 0.0 ? D[p] - z : T(0);  // q_a = v - z (tv_aniso.cpp:321-323)
                Q[((int64_t)a * B + b) * N + p] = im.e ? ldexp_t(q, im.e) : q;
            }
        } else {
            const T z = Z[p];
            O[p] = im.e ? ldexp_t(z, im.e) : z;
            if (im.e)
                for (int a = 0; a < g.k; ++a) {
                    T &q = Q[((int64_t)a * B + b) * N + p];
                    q = ldexp_t(q, im.e);
                }
        }
    }
}


template <class T>
cudaError_t setup_t(const AnGeom &g, const AnCall &c, const AnBuffers &bf, const void *x, cudaStream_t s) {
    const int nb = (int)std::min<int64_t>(128, std::max<int64_t>(1, (g.N + kThreads * 8 - 1) / (kThreads * 8)));
    const dim3 grid(nb, (unsigned)g.B);
    an_scan1<T><<<grid, kThreads, 0, s>>>(static_cast<const T *>(x), g, c, bf);
    an_scan2<T><<<grid, kThreads, 0, s>>>(g, c, bf);
    // single-axis images are solved here
    int64_t nfmax = 0;
    for (int a = 0; a < g.k; ++a) nfmax = std::max<int64_t>(nfmax, g.N / g.L[a]);
    an_single<T><<<dim3((unsigned)((nfmax + 127) / 128), (unsigned)g.B), 128, 0, s>>>(g, c, bf);
    return cudaGetLastError();
}

// Fibres per tile along each axis. A block scans its tile with one warp, so
// an SM scans as many fibres at once as the tiles of its resident blocks hold
// (shared memory, registers and threads bound how many blocks it holds): fb
// makes that number largest, up to 8 fibres (a warp's step takes longer the
// more lanes it carries, and more warps hide more of its latency: on 64 x
// 512^2 with edge weights 8 per block ran 3% faster than 16 and 8% faster than
// 26), among tiles of at most budget bytes (default
// kTileSmemMax) and while the launch still gives every SM a block; the larger
// fb on ties, so that fewer warps issue the same steps. fb is 1 or even (the
// tile's row length fb + 1 odd). 0 when one fibre does not fit: the untiled
// pass then runs.
constexpr int kTileSmemMax = 200 * 1024;
constexpr size_t kSmemPerSM = 228 * 1024;  // shared memory of an SM (sm_100)
constexpr size_t kSmemReserve = 1024 + 512;  // per block: the system's and the kernels' static arrays
constexpr int kSMs = 148;

// The tiled kernels may take up to kTileSmemMax of dynamic shared memory. Set
// once per kernel, before any launch: the attribute is per function, and
// threads launching with different sizes must not lower it under one another.
template <class T>
void tile_attributes() {
    static std::atomic<unsigned long long> done{0};  // one bit per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    const unsigned long long bit = 1ull << dev;
    if (done.load() & bit) return;
    cudaFuncSetAttribute(an_pass1_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemMax);
    cudaFuncSetAttribute(an_pass2_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemMax);
    cudaFuncSetAttribute(an_fdpg3_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemMax);
    done.fetch_or(bit);
}

// Blocks of the tiled kernels an SM holds by registers and threads (their
// largest register count, allocated per warp in units of 256).
template <class T>
int tile_blocks_by_regs() {
    static const int n = [] {
        int regs = 0;
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, an_pass1_tile<T>) == cudaSuccess) regs = std::max(regs, fa.numRegs);
        if (cudaFuncGetAttributes(&fa, an_pass2_tile<T>) == cudaSuccess) regs = std::max(regs, fa.numRegs);
        if (cudaFuncGetAttributes(&fa, an_fdpg3_tile<T>) == cudaSuccess) regs = std::max(regs, fa.numRegs);
        const int per_warp = ((std::max(regs, 1) * 32 + 255) / 256) * 256;
        const int warps = kTileThreads / 32;
        return std::max(1, std::min(2048 / kTileThreads, 65536 / (per_warp * warps)));
    }();
    return n;
}

template <class T>
TileCfg tile_cfg(const AnGeom &g, const AnCall &c, int64_t nimg, size_t &smem) {
    // tuning hints: FASTPROX_B200_TILE_FB caps fb, FASTPROX_B200_TILE_KB the
    // tile; FASTPROX_B200_TILES=0 runs the untiled passes (for comparison)
    static const bool off = [] {
        const char *v = std::getenv("FASTPROX_B200_TILES");
        return v && v[0] == '0' && v[1] == 0;
    }();
    static const int fb_max = [] {
        const char *v = std::getenv("FASTPROX_B200_TILE_FB");
        const int f = v ? std::atoi(v) : 0;
        return (f >= 1 && f <= 32) ? f : 8;
    }();
    static const size_t budget = [] {
        const char *v = std::getenv("FASTPROX_B200_TILE_KB");
        const int k = v ? std::atoi(v) : 0;
        return (size_t)((k >= 8 && k <= 200) ? k : 200) * 1024;
    }();
    const int by_regs = tile_blocks_by_regs<T>();
    TileCfg tc{{0, 0, 0}};
    smem = 0;
    const int nbuf = c.has_beta ? 2 : 1;
    for (int a = 0; a < g.k && !off; ++a) {
        const int L = (int)g.L[a];
        const int64_t fibres = nimg * (g.N / std::max<int64_t>(g.L[a], 1));
        int best = 0;
        double best_waves = 0.0;
        for (int fb = 1; fb <= fb_max; fb += (fb == 1 ? 1 : 2)) {
            const size_t by = tile_bytes(L, fb, nbuf, sizeof(T));
            if (by > budget || by > (size_t)kTileSmemMax) break;
            const int per_sm = std::min<int>(by_regs, (int)(kSmemPerSM / (by + kSmemReserve)));
            if (per_sm < 1) break;
            const int64_t blocks = (fibres + fb - 1) / fb;
            if (fb > 1 && blocks < kSMs) break;
            const double waves = std::max(1.0, (double)blocks / ((double)per_sm * kSMs));
            if (best == 0 || waves <= best_waves) {
                best = fb;
                best_waves = waves;
            }
        }
        tc.fb[a] = best;
        if (best) smem = std::max(smem, tile_bytes(L, best, nbuf, sizeof(T)));
    }
    return tc;
}

// The fibre-major scan keeps its table of 1/m (m <= L) in the default 48 KB
// of shared memory.
template <class T>
bool fm_fits(const AnGeom &g) {
    for (int a = 0; a < g.k; ++a)
        if ((size_t)(g.L[a] + 1) * sizeof(T) > 48 * 1024) return false;
    return true;
}

template <class T>
cudaError_t round_t(const AnGeom &g, const AnCall &c, const AnBuffers &bf, int64_t nimg, cudaStream_t s,
                   int64_t *launches) {
    if (nimg <= 0) return cudaSuccess;
    const unsigned B = (unsigned)nimg;
    int64_t nl = 0;
    const int pb = an_pixel_blocks(g);
    const dim3 pg(pb, B);
    // the iteration: ADBPG's two passes, or FDPG-3's three
    int64_t nf[3] = {1, 1, 1};
    for (int a = 0; a < g.k; ++a) nf[a] = g.N / g.L[a];
    int64_t nfmax = 0;
    for (int a = 0; a < g.k; ++a) nfmax = std::max(nfmax, nf[a]);
    const unsigned fbk = (unsigned)((nfmax + 127) / 128);
    if (c.has_adbpg && aniso_fm_enabled() && fm_fits<T>(g)) {
        // the fibre-major passes: the active axes (the same for every image of
        // the call), a1 the one of smaller stride
        int act[3], n = 0;
        for (int a = 0; a < g.k; ++a)
            if (c.w[a] > 0.0 && g.L[a] > 1) act[n++] = a;
        const int a1 = g.S[act[0]] < g.S[act[1]] ? act[0] : act[1], a2 = a1 == act[0] ? act[1] : act[0];
        auto tiles_grid = [&](int a) {
            if (g.S[a] == 1) return (unsigned)std::min<int64_t>((g.N + kFmThreads - 1) / kFmThreads, 1024);
            return (unsigned)std::min<int64_t>(fm_tiles(nf[a], g.L[a]), 1024);
        };
        constexpr int per = kFmScan / 32 * kFmLanes;  // fibres per scan block
        auto scan_grid = [&](int a) { return dim3((unsigned)((nf[a] + per - 1) / per), B); };
        auto scan_smem = [&](int a) { return (size_t)(g.L[a] + 1) * sizeof(T); };
        if (g.S[a1] == 1) {
            an_fm_scan<T, 1, true><<<scan_grid(a1), kFmScan, scan_smem(a1), s>>>(g, c, bf);
            nl += 1;
        } else {
            an_fm_stage<T, 1><<<dim3(tiles_grid(a1), B), kFmThreads, 0, s>>>(g, c, bf);
            an_fm_scan<T, 1, false><<<scan_grid(a1), kFmScan, scan_smem(a1), s>>>(g, c, bf);
            an_fm_unstage<T, 1><<<dim3(tiles_grid(a1), B), kFmThreads, 0, s>>>(g, c, bf);
            nl += 3;
        }
        if (g.S[a2] == 1) {
            an_fm_scan<T, 2, true><<<scan_grid(a2), kFmScan, scan_smem(a2), s>>>(g, c, bf);
            nl += 1;
        } else {
            an_fm_stage<T, 2><<<dim3(tiles_grid(a2), B), kFmThreads, 0, s>>>(g, c, bf);
            an_fm_scan<T, 2, false><<<scan_grid(a2), kFmScan, scan_smem(a2), s>>>(g, c, bf);
            nl += 2;
        }
        an_fm_unstage<T, 2><<<dim3(tiles_grid(a2), B), kFmThreads, 0, s>>>(g, c, bf);
        nl += 1;
    } else if (c.has_adbpg) {
        size_t smem = 0;
        const TileCfg tc = tile_cfg<T>(g, c, nimg, smem);
        bool tiled = true;
        int64_t tblk = 0;
        for (int a = 0; a < g.k; ++a) {
            if (g.L[a] > 1 && tc.fb[a] == 0) tiled = false;
            if (tc.fb[a]) tblk = std::max<int64_t>(tblk, (nf[a] + tc.fb[a] - 1) / tc.fb[a]);
        }
        if (tiled && tblk > 0 && tblk <= bf.max_part) {
            tile_attributes<T>();
            an_pass1_tile<T><<<dim3((unsigned)tblk, B), kTileThreads, smem, s>>>(g, c, bf, tc);
            an_pass2_tile<T><<<dim3((unsigned)tblk, B), kTileThreads, smem, s>>>(g, c, bf, tc);
        } else {
            an_pass1<T><<<dim3(fbk, B), 128, 0, s>>>(g, c, bf);
            an_pass2<T><<<dim3(fbk, B), 128, 0, s>>>(g, c, bf);
        }
        nl += 2;
    }
    if (c.has_fdpg3) {
        an_fdpg3_u<T><<<pg, kThreads, 0, s>>>(g, bf);
        size_t smem = 0;
        const TileCfg tc = tile_cfg<T>(g, c, nimg, smem);
        int64_t tblk = 0;
        bool tiled = g.k == 3;
        for (int a = 0; a < g.k; ++a) {
            if (tc.fb[a] == 0) tiled = false;
            else tblk = std::max<int64_t>(tblk, (nf[a] + tc.fb[a] - 1) / tc.fb[a]);
        }
        if (tiled && tblk > 0 && 3 * tblk <= bf.max_part) {
            tile_attributes<T>();
            an_fdpg3_tile<T><<<dim3((unsigned)tblk, 3, B), kTileThreads, smem, s>>>(g, c, bf, tc);
        } else {
            an_fdpg3_pass<T><<<dim3(fbk, 3, B), 128, 0, s>>>(g, c, bf);
        }
        nl += 2;
    }
    an_restart_copy<T><<<pg, kThreads, 0, s>>>(g, bf);
    ++nl;
    if (c.warm && c.has_adbpg) {
        // a warm start's pass (run by the first pass above) and its dual
        an_warm_z<T><<<pg, kThreads, 0, s>>>(g, bf);
        an_warm_next<<<((unsigned)g.B + 127) / 128, 128, 0, s>>>(g, bf);
        nl += 2;
    }
    // gap check (FDPG-3 forms its primal first)
    if (c.has_fdpg3) {
        an_fdpg3_primal<T><<<dim3((unsigned)((nf[2] + 127) / 128), B), 128, 0, s>>>(g, c, bf, kStCheck);
        ++nl;
    }
    an_gap<T><<<pg, kThreads, 0, s>>>(g, c, bf, kStCheck);
    ++nl;
    // polish
    an_dual<T><<<pg, kThreads, 0, s>>>(g, bf, kStPolish);
    for (int a = 0; a < g.k; ++a) an_mark<T><<<dim3((unsigned)((nf[a] + 127) / 128), B), 128, 0, s>>>(g, c, bf, a);
    an_union<<<pg, kThreads, 0, s>>>(g, bf);
    an_region_sum<T><<<pg, kThreads, 0, s>>>(g, bf);
    an_polish_gap<T><<<pg, kThreads, 0, s>>>(g, c, bf);
    an_polish_write<T><<<pg, kThreads, 0, s>>>(g, bf);
    nl += 5 + g.k;
    // final rebuild, then retirement (over every image)
    const unsigned BA = (unsigned)g.B;
    an_final_skip<<<(BA + 127) / 128, 128, 0, s>>>(g, bf);
    an_dual<T><<<pg, kThreads, 0, s>>>(g, bf, kStFinal);
    an_gap<T><<<pg, kThreads, 0, s>>>(g, c, bf, kStFinal);
    an_retire<<<(BA + 127) / 128, 128, 0, s>>>(g, bf);
    nl += 4;
    if (launches) *launches += nl;
    return cudaGetLastError();
}

template <class T>
cudaError_t warm_t(const AnGeom &g, const AnCall &c, const AnBuffers &bf, cudaStream_t s) {
    for (int a = 0; a < g.k; ++a) {
        const int64_t nf = g.N / g.L[a];
        an_warm_feasible<T><<<dim3((unsigned)((nf + 127) / 128), (unsigned)g.B), 128, 0, s>>>(g, c, bf, a);
    }
    an_warm_init<T><<<dim3(an_pixel_blocks(g), (unsigned)g.B), kThreads, 0, s>>>(g, bf);
    an_warm_state<<<((unsigned)g.B + 127) / 128, 128, 0, s>>>(g, bf);
    return cudaGetLastError();
}

template <class T>
cudaError_t output_t(const AnGeom &g, const AnBuffers &bf, void *out, cudaStream_t s) {
    an_output<T><<<dim3(an_pixel_blocks(g), (unsigned)g.B), kThreads, 0, s>>>(g, bf, static_cast<T *>(out));
    return cudaGetLastError();
}

}  // namespace

bool aniso_fm_enabled() {
    static const bool on = [] {  // tuning hint FASTPROX_B200_AN_FIB=0: the tiled passes
        const char *v = std::getenv("FASTPROX_B200_AN_FIB");
        return !(v && v[0] == '0' && v[1] == 0);
    }();
    return on;
}

cudaError_t aniso_weights_fm(int dtype, const AnGeom &g, const void *beta, void *wt, cudaStream_t s) {
    int64_t nt = 1;
    for (int a = 0; a < g.k; ++a) nt = std::max<int64_t>(nt, fm_tiles(g.N / g.L[a], g.L[a]));
    const dim3 grid((unsigned)std::min<int64_t>(nt, 4096), (unsigned)g.k);
    if (dtype == 1)
        an_weights_fm<float><<<grid, kFmThreads, 0, s>>>(g, static_cast<const float *>(beta), static_cast<float *>(wt));
    else
        an_weights_fm<double>
            <<<grid, kFmThreads, 0, s>>>(g, static_cast<const double *>(beta), static_cast<double *>(wt));
    return cudaGetLastError();
}

int an_pixel_blocks(const AnGeom &g) {
    int64_t nb = (g.N + kThreads * 4 - 1) / (kThreads * 4);
    return (int)std::max<int64_t>(1, std::min<int64_t>(nb, 256));
}

cudaError_t aniso_setup(int dtype, const AnGeom &g, const AnCall &c, const AnBuffers &bf, const void *x,
                        cudaStream_t s) {
    return dtype == 1 ? setup_t<float>(g, c, bf, x, s) : setup_t<double>(g, c, bf, x, s);
}

cudaError_t aniso_warm(int dtype, const AnGeom &g, const AnCall &c, const AnBuffers &bf, cudaStream_t s) {
    return dtype == 1 ? warm_t<float>(g, c, bf, s) : warm_t<double>(g, c, bf, s);
}

void aniso_prepare(int dtype) {
    if (dtype == 1) tile_attributes<float>();
    else tile_attributes<double>();
}

cudaError_t aniso_round(int dtype, const AnGeom &g, const AnCall &c, const AnBuffers &bf, int64_t nimg,
                        cudaStream_t s, int64_t *launches) {
    return dtype == 1 ? round_t<float>(g, c, bf, nimg, s, launches) : round_t<double>(g, c, bf, nimg, s, launches);
}

cudaError_t aniso_live_list(const AnState *st, int64_t B, int *lmap, int *lcnt, cudaStream_t s) {
    an_live_list<<<1, 1024, 0, s>>>(st, B, lmap, lcnt);
    return cudaGetLastError();
}

cudaError_t aniso_output(int dtype, const AnGeom &g, const AnBuffers &bf, void *out, cudaStream_t s) {
    return dtype == 1 ? output_t<float>(g, bf, out, s) : output_t<double>(g, bf, out, s);
}

}  // namespace fpb
