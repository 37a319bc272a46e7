// Isotropic image TV by dual FISTA on sm_100a: the set-up scans, the fused
// iteration, the per-image stopping and restart logic, and the finalisation.
//
// The schedule is the reference's TVIso::fdpg (src/ops/tv_iso.cpp:424-543),
// replayed per image on the device: the restart test of O'Donoghue and
// Candes at every iteration it with it % 4 == 0 (tv_iso.cpp:498, 528-534),
// the duality gap after every fourth iteration and at max_iter
// (tv_iso.cpp:536), with FP64 accumulation of the gap and of the restart
// dot. Iterates are kept in the array's dtype (FP32 for float32 input).
//
// One launch is one iteration of every live image. The gap of the state an
// iteration starts from is evaluated in that same launch (its stencil reads
// the same rows), and the last block of each image decides: converged (the
// launch's update is dropped: it wrote the other ping-pong buffer), max_iter
// reached, or go on, with the restart folded into the next launch's reads
// (v = u) instead of a copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <type_traits>
#include <cfloat>
#include <cmath>
#include <cstdlib>

#include "common.cuh"
#include "launch.h"

namespace fpb {
namespace {

constexpr int kScanThreads = 256;
#define FP_MAX_NDIM_DEV 32
constexpr double kMaxScaledStepLog2 = 960.0;  // the reference's kMaxScaledStep = 2^960 (core/op.hpp:48)

template <class T>
__device__ __forceinline__ T ldexp_t(T v, int e);
template <>
__device__ __forceinline__ float ldexp_t<float>(float v, int e) { return ldexpf(v, e); }
template <>
__device__ __forceinline__ double ldexp_t<double>(double v, int e) { return ldexp(v, e); }

__device__ __forceinline__ float sqrt_t(float v) { return sqrtf(v); }
__device__ __forceinline__ double sqrt_t(double v) { return sqrt(v); }

// ---------------------------------------------------------------------------
// Set-up scans (tv_iso.cpp:342-366, 369-377, 435-452, 479-483)
// ---------------------------------------------------------------------------

// Pass 1: copy x into d (unless it is already there), max |x|, NaN and Inf
// flags; the last block picks the rescaling exponent and the image's mode.
template <class T>
__global__ void __launch_bounds__(kScanThreads) scan1_kernel(const T *__restrict__ x, T *__restrict__ d, Geometry g,
                                                             IsoCall c, IsoBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int64_t N = g.N;
    const T *xb = x + (int64_t)b * N;
    T *db = d + (int64_t)b * N;
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
    // the two flag bits are reduced apart: a max cannot OR them
    const double mb = block_max(m, sh);
    const double f1 = block_max((double)(fl & 1), sh);
    const double f2 = block_max((double)((fl >> 1) & 1), sh);
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2 + 0] = mb;
        part[blockIdx.x * 2 + 1] = f1 + 2.0 * f2;
    }
    if (!arrive_last(bf.ticket + b, gridDim.x, &flag)) return;
    const double mx = max_partials(part, gridDim.x, 2, 0, sh);
    // OR of the flag codes: max over bit 0 and bit 1 separately
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
    IsoImage im;
    im.gamma_in = bf.gammas[b];
    im.maxabs = mx;
    im.flags = (o1 > 0.0 ? 1 : 0) | (o2 > 0.0 ? 2 : 0);
    im.mean = 0.0;
    im.dd = 0.0;
    im.target = 0.0;
    im.bound = 0.0;
    im.radius = 0.0;
    im.pad = 0;
    int e = 0;
    const bool act = im.gamma_in > 0.0 && c.na > 0;
    if (im.flags & 2) im.mode = kModeInf;
    else if (im.flags & 1) im.mode = kModeNan;
    else if (!act) im.mode = kModeIdentity;
    else im.mode = (c.na == 1 && !c.has_alpha && !c.huber) ? kModeTv1d : kModeFdpg;
    if (im.mode == kModeFdpg || im.mode == kModeTv1d) {
        // rescale_exponent (src/ops/image_util.hpp:56-65)
        const double gamma = im.gamma_in;
        if (mx > 0.0) {
            e = ilogb(mx);
            if (e >= -64 && e <= 64) {
                e = 0;
            } else {
                const double top = fmax(gamma, gamma * c.step_scale);
                if (e < 0 && top > 0.0) e = min(0, max(e, ilogb(top) + 1 - (int)kMaxScaledStepLog2));
            }
        }
        // unless an active step would underflow there (tv_iso.cpp:371-372)
        for (int a = 0; a < g.k && e; ++a) {
            const double wa = c.wh[a] * c.wmax;
            if (wa > 0.0 && !(ldexp(gamma * wa, -e) > 0.0)) e = 0;
        }
    }
    im.e = e;
    bf.img[b] = im;
    IsoState st;
    st.it = 0;
    st.since = 0;
    st.last = 0;
    st.status = kFinished;
    st.vsel = 0;
    st.zero_in = 1;
    st.warm = 0;
    st.fin_par = 0;
    st.redo = 0;
    st.redo_vsel = 0;
    st.tn = fista_t(1.0);
    st.beta = 0.0;
    st.gp = CUDART_INF;
    st.dot = 0.0;
    bf.st[b] = st;
}

// Pass 2: d *= 2^-e, sum d and sum d^2 (mean and the stopping target).
template <class T>
__global__ void __launch_bounds__(kScanThreads) scan2_kernel(T *__restrict__ d, Geometry g, IsoCall c, IsoBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    const int mode = bf.img[b].mode;
    if (mode == kModeNan || mode == kModeInf) return;
    const int e = bf.img[b].e;  // 0 unless the image is solved (fdpg, tv1d)
    const int64_t N = g.N;
    T *db = d + (int64_t)b * N;
    double s = 0.0, s2 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        T v = db[i];
        if (e) {
            v = ldexp_t(v, -e);
            db[i] = v;
        }
        const double dv = (double)v;
        s += dv;
        s2 += dv * dv;
    }
    const double sb = block_sum(s, sh);
    const double s2b = block_sum(s2, sh);
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2 + 0] = sb;
        part[blockIdx.x * 2 + 1] = s2b;
    }
    if (!arrive_last(bf.ticket + b, gridDim.x, &flag)) return;
    const double tot = sum_partials(part, gridDim.x, 2, 0, sh);
    const double tot2 = sum_partials(part, gridDim.x, 2, 1, sh);
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    bf.img[b].mean = tot / (double)N;
    bf.img[b].dd = tot2;
    bf.img[b].target = c.tol * 0.5 * tot2;
}

// Pass 3: the imbalance sum |d - mean| -> bound and radius; state set-up.
template <class T>
__global__ void __launch_bounds__(kScanThreads) scan3_kernel(const T *__restrict__ d, Geometry g, IsoCall c,
                                                             IsoBuffers bf, int warm) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = blockIdx.y;
    if (bf.img[b].mode != kModeFdpg) return;
    const double mean = bf.img[b].mean;
    const int64_t N = g.N;
    const T *db = d + (int64_t)b * N;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        s += fabs((double)db[i] - mean);
    const double sb = block_sum(s, sh);
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) part[blockIdx.x * 2 + 0] = sb;
    if (!arrive_last(bf.ticket + b, gridDim.x, &flag)) return;
    const double imb = sum_partials(part, gridDim.x, 2, 0, sh);
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoImage &im = bf.img[b];
    const double gamma_s = ldexp(im.gamma_in, -im.e);
    double gamma = gamma_s * c.wmax;  // tv_iso.cpp:445-447
    const double bound = 2.0 * imb / c.whmin + DBL_MIN;
    if (!(gamma <= bound) && !c.has_alpha && !c.huber) gamma = bound;  // (no such cap for Huber-smoothed TV)
    im.bound = bound;
    im.radius = gamma;
    IsoState &st = bf.st[b];
    st.status = kLive;
    st.zero_in = warm ? 0 : 1;
    st.warm = warm ? 1 : 0;
    atomicAdd(bf.live, 1);
}

// The radius of pixel p: gamma alpha_p capped at bound, 0 where alpha_p = 0
// (tv_iso.cpp:180-185); gamma itself without pixel weights.
template <class T, bool ALPHA>
__device__ __forceinline__ T pixel_radius(T rad, T bnd, const T *al, int64_t p) {
    if (!ALPHA) return rad;
    const T a = al[p];
    if (a == T(0)) return T(0);
    const T r = rad * a;
    return r <= bnd ? r : bnd;
}

// Warm start: u = q 2^-e wmax, zero on inactive axes, at the last entry
// along each axis and where not finite, projected onto the balls
// (tv_iso.cpp:456-478); v = u.
template <class T, bool ALPHA>
__global__ void warm_kernel(Geometry g, IsoCall c, IsoBuffers bf, int par) {
    const int b = blockIdx.y;
    const IsoImage &im = bf.img[b];
    if (im.mode != kModeFdpg) return;
    const int64_t N = g.N, B = g.B;
    const T *q = static_cast<const T *>(bf.dual);
    T *U = static_cast<T *>(bf.U[par]) + (int64_t)b * g.k * N;
    T *V = static_cast<T *>(bf.V[par]) + (int64_t)b * g.k * N;
    const T *al = ALPHA ? static_cast<const T *>(bf.alpha) + (int64_t)b * c.alpha_stride : nullptr;
    const T rad = (T)im.radius, bnd = (T)im.bound;
    int64_t S[3];
    S[g.k - 1] = 1;
    for (int a = g.k - 2; a >= 0; --a) S[a] = S[a + 1] * g.L[a + 1];
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        T u[3] = {T(0), T(0), T(0)};
        T nn = T(0);
        for (int a = 0; a < g.k; ++a) {
            const bool has = ((p / S[a]) % g.L[a]) + 1 < g.L[a];
            T v = ldexp_t(q[((int64_t)a * B + b) * N + p], -im.e) * (T)c.wmax;
            if (c.wh[a] == 0.0 || !has || !isfinite(v)) v = T(0);
            u[a] = v;
            nn += v * v;
        }
        if (c.huber == 2) {  // anisotropic Huber: a box per component, its edge weight's radius
            for (int a = 0; a < g.k; ++a) {
                const T ra = ALPHA ? rad * static_cast<const T *>(bf.alpha)[(int64_t)a * N + p] : rad;
                u[a] = u[a] > ra ? ra : (u[a] < -ra ? -ra : u[a]);
            }
        } else {
            const T rp = c.huber ? (ALPHA ? rad * al[p] : rad) : pixel_radius<T, ALPHA>(rad, bnd, al, p);
            const T nr = sqrt_t(nn);
            if (nr > rp) {
                const T sc = rp / nr;
                for (int a = 0; a < g.k; ++a) u[a] *= sc;
            }
        }
        for (int a = 0; a < g.k; ++a) {
            U[a * N + p] = u[a];
            V[a * N + p] = u[a];
        }
    }
}

// ---------------------------------------------------------------------------
// Per-image control: the scalar part of one fdpg iteration (tv_iso.cpp:528-537)
// ---------------------------------------------------------------------------

// Runs in thread 0 of the last block of an image after a step launch that
// started from iteration st.it. gap: the gap of that starting state, when
// do_gap; dot: the restart test's <v - u+, u+ - u>, when test.
__device__ void control(IsoState &st, const IsoImage &im, int max_iter, bool do_gap, bool test, double gap,
                        double dot, int par_in, int *live) {
    if (do_gap) {
        st.gp = gap;
        if (gap <= im.target) {  // the loop condition of tv_iso.cpp:491
            st.status = kConverged;
            st.fin_par = par_in;
            atomicSub(live, 1);
            return;
        }
        if (st.it >= max_iter) {
            st.status = kNotConv;
            st.fin_par = par_in;
            atomicSub(live, 1);
            return;
        }
    }
    // The update of this launch stands.
    st.dot = dot;
    st.since += 1;
    const bool restart = test && dot > 0.0 && st.since >= st.last;
    double t = st.tn;
    if (restart) {
        t = 1.0;
        st.last = st.since;
        st.since = 0;
    }
    st.vsel = restart ? 1 : 0;
    st.zero_in = 0;
    st.it += 1;
    const double tn = fista_t(t);
    st.beta = (t - 1.0) / tn;
    st.tn = tn;
    st.fin_par = par_in ^ 1;
}

// The image of launch slot z (-1: none, the live list is shorter).
__device__ __forceinline__ int step_image(const IsoBuffers &bf, unsigned z) {
    if (!bf.lmap) return (int)z;
    return (int)z < *bf.lcnt ? bf.lmap[z] : -1;
}

// The live images in order: one block scans the states in chunks.
__global__ void __launch_bounds__(1024) live_list_kernel(const IsoState *st, int64_t B, int *lmap, int *lcnt) {
    __shared__ int wsum[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t c0 = 0; c0 < B; c0 += blockDim.x) {
        const int64_t i = c0 + threadIdx.x;
        const int f = (i < B && st[i].status == kLive) ? 1 : 0;
        int x = f;  // inclusive scan in the warp
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
            wsum[lane] = w;  // inclusive over warps
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

struct StepArgs {
    Geometry g;
    int max_iter;
    int par;
    int rows;
    int64_t nimg;  // launch slots (host side: the grid's image extent)
    int row_part;  // lean 2D step: per-row partial sums (H x column blocks slots)
};

constexpr int kLeanRowsMax = 32;  // rows per block of the lean 2D step
// blocks a lean launch should have before its blocks grow (tuning hint
// FASTPROX_B200_TAIL_BLOCKS)
int64_t tail_blocks() {
    static const int64_t v = [] {
        const char *e = std::getenv("FASTPROX_B200_TAIL_BLOCKS");
        const long long n = e ? std::atoll(e) : 0;
        return (int64_t)(n > 0 ? n : 148 * 4);
    }();
    return v;
}

// ---------------------------------------------------------------------------
// The lean 2D step: a warp spans 32 * VEC consecutive columns, a block
// BX * VEC of them, and each thread walks down `rows` rows keeping the
// current and next rows of z, u and v in registers, so every array is read
// from HBM once per iteration (36 B per pixel in FP32: d, u, v in; u, v out).
// Horizontal neighbours come from the next lane by shuffle. The per-pixel
// work is the arithmetic of the iteration. Offsets are 32-bit within an image
// (images have fewer than 2^31 pixels), row pointers advance by W, the gap
// and the cold start are compile-time variants (one per block: every live
// image of a launch shares its branch), the projection multiplies by a
// reciprocal square root, and lane 31 carries the three scalars of the next
// warp's first column instead of re-reading them.
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T rsqrt_t(T v);
// float: the hardware reciprocal square root (rsqrtf's result on normal
// numbers) with arguments below the smallest normal float taken as that
// smallest normal (no rescaling of subnormal arguments; at a zero radius the
// projection's scale stays rp times a finite number, 0)
template <>
__device__ __forceinline__ float rsqrt_t<float>(float v) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(fmaxf(v, FLT_MIN)));
    return r;
}
template <>
__device__ __forceinline__ double rsqrt_t<double>(double v) { return rsqrt(v); }

template <class T, int VEC, bool ALPHA, bool GAP, bool ZIN>
__device__ __forceinline__ void lean_rows(const T *__restrict__ D, const T *__restrict__ U0, const T *__restrict__ U1,
                                          const T *__restrict__ V0, const T *__restrict__ V1, T *__restrict__ UO0,
                                          T *__restrict__ UO1, T *__restrict__ VO0, T *__restrict__ VO1,
                                          const T *__restrict__ AL, int H, int W, int cb, int r0, int r1, T wh0, T wh1,
                                          T tau, T beta, T rad, T bnd, bool test, bool store, double &gap_acc,
                                          double &dot_acc, double *rowp = nullptr) {
    const int lane = threadIdx.x & 31;
    const bool colok = cb < W;
    const bool ext = lane == 31 && cb + VEC < W;  // the next warp's first column
    auto ld = [&](const T *P, int off, T(&o)[VEC]) {
        if (!ZIN && colok) load_pack<T, VEC>(P + off, o);
        else
#pragma unroll
            for (int j = 0; j < VEC; ++j) o[j] = T(0);
    };
    auto ldd = [&](int off, T(&o)[VEC]) {
        if (colok) load_pack<T, VEC>(D + off, o);
        else
#pragma unroll
            for (int j = 0; j < VEC; ++j) o[j] = T(0);
    };
    auto zrow = [&](const T(&dd)[VEC], const T(&p0)[VEC], const T(&p0p)[VEC], const T(&p1)[VEC], T left, T(&z)[VEC]) {
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            z[j] = dd[j] + wh0 * (p0[j] - p0p[j]) + wh1 * (p1[j] - left);
            left = p1[j];
        }
    };
    int off = r0 * W + cb;
    // row r0 and the part of row r0 - 1 it needs
    T v0c[VEC], v1c[VEC], u0c[VEC], u1c[VEC], zc[VEC], zuc[VEC];
    T dc[VEC], v0p[VEC], u0p[VEC];
    ldd(off, dc);
    ld(V0, off, v0c);
    ld(V1, off, v1c);
    ld(U0, off, u0c);
    ld(U1, off, u1c);
    if (r0 > 0) {
        ld(V0, off - W, v0p);
        if (GAP) ld(U0, off - W, u0p);
    } else {
#pragma unroll
        for (int j = 0; j < VEC; ++j) v0p[j] = u0p[j] = T(0);
    }
    const T v1l = (!ZIN && colok && cb > 0) ? V1[off - 1] : T(0);
    zrow(dc, v0c, v0p, v1c, v1l, zc);
    if (GAP) zrow(dc, u0c, u0p, u1c, (colok && cb > 0) ? U1[off - 1] : T(0), zuc);
    // lane 31: z at (r0, cx) of v (and u)
    T x_v0 = T(0), x_u0 = T(0), x_z = T(0), x_zu = T(0);
    if (ext) {
        const T dx = D[off + VEC];
        if (!ZIN) {
            x_v0 = V0[off + VEC];
            x_u0 = U0[off + VEC];
        }
        const T pv = (!ZIN && r0 > 0) ? V0[off + VEC - W] : T(0);
        x_z = dx + wh0 * (x_v0 - pv) + wh1 * ((ZIN ? T(0) : V1[off + VEC]) - v1c[VEC - 1]);
        if (GAP) {
            const T pu = r0 > 0 ? U0[off + VEC - W] : T(0);
            x_zu = dx + wh0 * (x_u0 - pu) + wh1 * (U1[off + VEC] - u1c[VEC - 1]);
        }
    }
    for (int i = r0; i < r1; ++i) {
        const bool hasn = i + 1 < H;
        const int offn = off + W;
        T dn[VEC], v0n[VEC], v1n[VEC], u0n[VEC], u1n[VEC], zn[VEC], zun[VEC];
        T nx_v0 = T(0), nx_u0 = T(0), nx_z = T(0), nx_zu = T(0);
        if (hasn) {
            ldd(offn, dn);
            ld(V0, offn, v0n);
            ld(V1, offn, v1n);
            ld(U0, offn, u0n);
            ld(U1, offn, u1n);
            zrow(dn, v0n, v0c, v1n, (!ZIN && colok && cb > 0) ? V1[offn - 1] : T(0), zn);
            if (GAP) zrow(dn, u0n, u0c, u1n, (colok && cb > 0) ? U1[offn - 1] : T(0), zun);
            if (ext) {
                const T dx = D[offn + VEC];
                if (!ZIN) {
                    nx_v0 = V0[offn + VEC];
                    nx_u0 = U0[offn + VEC];
                }
                nx_z = dx + wh0 * (nx_v0 - x_v0) + wh1 * ((ZIN ? T(0) : V1[offn + VEC]) - v1n[VEC - 1]);
                if (GAP) nx_zu = dx + wh0 * (nx_u0 - x_u0) + wh1 * (U1[offn + VEC] - u1n[VEC - 1]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < VEC; ++j) zn[j] = zun[j] = u0n[j] = u1n[j] = v0n[j] = v1n[j] = T(0);
        }
        T al[VEC];
        if (ALPHA) {
            if (colok) load_pack<T, VEC>(AL + off, al);
            else
#pragma unroll
                for (int j = 0; j < VEC; ++j) al[j] = T(0);
        }
        T zr = __shfl_down_sync(0xffffffffu, zc[0], 1);
        if (lane == 31) zr = x_z;
        T zur = T(0);
        if (GAP) {
            zur = __shfl_down_sync(0xffffffffu, zuc[0], 1);
            if (lane == 31) zur = x_zu;
        }
        if (colok) {
            T uo0[VEC], uo1[VEC], vo0[VEC], vo1[VEC];
#pragma unroll
            for (int j = 0; j < VEC; ++j) {
                const bool hasr = cb + j + 1 < W;
                const T zright = j + 1 < VEC ? zc[j + 1] : zr;
                const T g0 = hasn ? wh0 * (zn[j] - zc[j]) : T(0);
                const T g1 = hasr ? wh1 * (zright - zc[j]) : T(0);
                const T cv0 = v0c[j] + tau * g0;  // wh = 0 gives g = 0 and v = 0 on that axis
                const T cv1 = v1c[j] + tau * g1;
                const T nn = cv0 * cv0 + cv1 * cv1;
                T rp = rad;
                if (ALPHA) {
                    const T r = rad * al[j];
                    rp = al[j] == T(0) ? T(0) : (r <= bnd ? r : bnd);
                }
                const T sc = nn > rp * rp ? rp * rsqrt_t(nn) : T(1);
                const T un0 = cv0 * sc, un1 = cv1 * sc;
                if (test) dot_acc += (double)((v0c[j] - un0) * (un0 - u0c[j]) + (v1c[j] - un1) * (un1 - u1c[j]));
                vo0[j] = un0 + beta * (un0 - u0c[j]);
                vo1[j] = un1 + beta * (un1 - u1c[j]);
                uo0[j] = un0;
                uo1[j] = un1;
                if (GAP) {
                    const T zuright = j + 1 < VEC ? zuc[j + 1] : zur;
                    const T gu0 = hasn ? wh0 * (zun[j] - zuc[j]) : T(0);
                    const T gu1 = hasr ? wh1 * (zuright - zuc[j]) : T(0);
                    gap_acc += (double)(rp * sqrt_t(gu0 * gu0 + gu1 * gu1) - (gu0 * u0c[j] + gu1 * u1c[j]));
                }
            }
            if (store) {
                store_pack<T, VEC>(UO0 + off, uo0);
                store_pack<T, VEC>(UO1 + off, uo1);
                store_pack<T, VEC>(VO0 + off, vo0);
                store_pack<T, VEC>(VO1 + off, vo1);
            }
        }
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            v0c[j] = v0n[j];
            v1c[j] = v1n[j];
            u0c[j] = u0n[j];
            u1c[j] = u1n[j];
            zc[j] = zn[j];
            if (GAP) zuc[j] = zun[j];
        }
        x_v0 = nx_v0;
        x_u0 = nx_u0;
        x_z = nx_z;
        x_zu = nx_zu;
        off = offn;
        if (rowp && (GAP || test)) {
            // this row's sums over the warp (a fixed tree), per warp in shared
            // memory: rowp[(row - r0) * 8 + 2 * warp + (0: gap, 1: dot)]
            double gv = gap_acc, dv = dot_acc;
            for (int o = 16; o > 0; o >>= 1) {
                gv += __shfl_down_sync(0xffffffffu, gv, o);
                dv += __shfl_down_sync(0xffffffffu, dv, o);
            }
            if (lane == 0) {
                rowp[(i - r0) * 8 + 2 * (threadIdx.x >> 5) + 0] = gv;
                rowp[(i - r0) * 8 + 2 * (threadIdx.x >> 5) + 1] = dv;
            }
            gap_acc = dot_acc = 0.0;
        }
    }
}

// GAP and ZIN are chosen by the host from the launch index (every live image
// of a call is at the same iteration); an image at another iteration (which
// a single call never has) is flagged as an error rather than solved wrongly.
template <class T, int VEC, bool ALPHA, bool GAP, bool ZIN>
__global__ void __launch_bounds__(128, 5) iso2d_lean_kernel(StepArgs A, IsoCall c, IsoBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    // launched as a programmatic dependent of the previous step: nothing of
    // its output (states, iterates, live list) is read before it completes
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int b = step_image(bf, blockIdx.z);
    if (b < 0) return;
    const IsoState st = bf.st[b];
    if (st.status != kLive) return;
    const int it = st.it;
    const bool do_gap = (it > 0 && ((it & 3) == 0 || it == A.max_iter)) || (it == 0 && st.warm);
    const bool zin = st.zero_in != 0;
    if (do_gap != GAP || zin != ZIN) {
        if (threadIdx.x == 0) atomicExch(bf.err, 3);
        return;
    }
    const IsoImage im = bf.img[b];
    const int H = (int)A.g.L[0], W = (int)A.g.L[1];
    const int64_t N = A.g.N;
    const bool do_upd = it < A.max_iter;
    const bool test = do_upd && (it & 3) == 0;
    const int pin = A.par, pout = A.par ^ 1;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *U0 = static_cast<const T *>(bf.U[pin]) + (int64_t)b * 2 * N;
    const T *V0 = st.vsel ? U0 : static_cast<const T *>(bf.V[pin]) + (int64_t)b * 2 * N;
    T *UO0 = static_cast<T *>(bf.U[pout]) + (int64_t)b * 2 * N;
    T *VO0 = static_cast<T *>(bf.V[pout]) + (int64_t)b * 2 * N;
    const T *AL = ALPHA ? static_cast<const T *>(bf.alpha) + (int64_t)b * c.alpha_stride : nullptr;
    const int cb = (blockIdx.x * blockDim.x + threadIdx.x) * VEC;
    const int r0 = blockIdx.y * A.rows;
    const int r1 = min(H, r0 + A.rows);
    double gap_acc = 0.0, dot_acc = 0.0;
    __shared__ double rowp[kLeanRowsMax * 8];
    lean_rows<T, VEC, ALPHA, GAP, ZIN>(D, U0, U0 + N, V0, V0 + N, UO0, UO0 + N, VO0, VO0 + N, AL, H, W, cb, r0, r1,
                                       (T)c.wh[0], (T)c.wh[1], (T)c.tau, (T)st.beta, (T)im.radius, (T)im.bound, test,
                                       do_upd, gap_acc, dot_acc, A.row_part ? rowp : nullptr);
    // the next step's blocks may be scheduled now (they wait for this one)
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const unsigned nblk = gridDim.x * gridDim.y;
    const unsigned blk = blockIdx.y * gridDim.x + blockIdx.x;
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    unsigned nslot = nblk;
    if (A.row_part) {
        // one slot per (row, column block), each the sum of its warps in
        // order: the same sums however many rows a block takes
        __syncthreads();
        const int nw = (int)(blockDim.x >> 5);
        if ((GAP || test) && (int)threadIdx.x < r1 - r0) {
            double gv = 0.0, dv = 0.0;
            for (int w = 0; w < nw; ++w) {
                gv += rowp[threadIdx.x * 8 + 2 * w];
                dv += rowp[threadIdx.x * 8 + 2 * w + 1];
            }
            const int64_t slot = (int64_t)(r0 + threadIdx.x) * gridDim.x + blockIdx.x;
            part[slot * 2 + 0] = gv;
            part[slot * 2 + 1] = dv;
        }
        nslot = (unsigned)H * gridDim.x;
    } else {
        const double gsum = GAP ? block_sum(gap_acc, sh) : 0.0;
        const double dsum = test ? block_sum(dot_acc, sh) : 0.0;
        if (threadIdx.x == 0) {
            part[blk * 2 + 0] = gsum;
            part[blk * 2 + 1] = dsum;
        }
    }
    if (!arrive_last(bf.ticket + b, nblk, &flag)) return;
    const double gap = GAP ? sum_partials(part, nslot, 2, 0, sh) : 0.0;
    const double dot = test ? sum_partials(part, nslot, 2, 1, sh) : 0.0;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2 = st;
    control(s2, im, A.max_iter, GAP, test, gap, dot, pin, bf.live);
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// Two iterations in one pass over memory (temporal blocking of the lean step).
//
// Iteration it = 1 mod 4 carries no check and no restart test, so the next
// needs nothing of it but its iterates u' = P(v + tau G z(v)), v' = u' +
// beta (u' - u); the next beta is the one the per-image control would set,
// (tn - 1) / fista_t(tn). The pair (it, it + 1) is one launch: a block covers
// whole rows and marches them like the lean step, the first iteration in
// registers as lean_rows does, on its rows and one more above and below, the
// second one row behind it, with the first's v' (and u') passing between
// threads by shuffles, and between warps through shared memory (a warp's
// first and last columns, for its neighbours' z(v'), z(u')). Only the
// second's u'', v'' are written.
// Traffic per pixel and two iterations: d, u, v (and alpha) read once over
// R + 4 rows for R output rows, u'' and v'' written once: about 50 B against
// 2 x 40 B for two lean steps.
// GAP2: it = 3 mod 4, the second iteration (0 mod 4) carrying the gap check
// at u' and the restart test, with lean_rows' per-row partial sums; u' is
// not stored: when the check passes (the final iterate is u'), the state
// keeps fin_par = the launch's input parity and redo = 1, and iso_redo forms
// u' again from those untouched buffers before the solve's outputs are read.
// Each iteration's arithmetic and every sum's order are lean_rows' (the same
// expressions), so the iterates and the checks are those of two lean steps.
// ---------------------------------------------------------------------------
constexpr int kPairCols = 512;  // columns a block covers: 128 threads x 4

// Asynchronous copies global -> shared of a thread's own data (cp.async),
// counted per thread in commit groups.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
template <int BYTES>
__device__ __forceinline__ void cp_async_small(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "n"(BYTES)
                 : "memory");
}
// One entry, or zeros when n is 0 (nothing is read then).
template <int BYTES>
__device__ __forceinline__ void cp_async_zfill(void *dst, const void *src, unsigned n) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "n"(BYTES), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// The pair kernel's row ring: three rows of each thread's inputs (d, v0, v1,
// u0, u1, alpha: VEC entries each; v1 of the column before, lane 31's d, v0,
// v1 of the column after, and the halo columns' entries of a block's edge
// threads), in flight up to three rows ahead. Ten scalars per thread with the
// halo columns, four without (a smaller ring leaves more of the SM's shared
// storage to the L1 cache: 1% on 64 x 512^2).
constexpr int kPairRing = 3;
template <bool WIDE>
constexpr int pair_scalars() {
    return WIDE ? 10 : 4;
}
template <class T, bool ALPHA, bool WIDE>
constexpr size_t pair_slot_bytes() {
    return (size_t)128 * ((ALPHA ? 6 : 5) * 4 * sizeof(T) + pair_scalars<WIDE>() * sizeof(T));
}
template <class T, bool ALPHA, bool WIDE>
constexpr size_t pair_ring_bytes() {
    return kPairRing * pair_slot_bytes<T, ALPHA, WIDE>();
}

// What one pair pass needs: an image's arrays, the block's rows [r0, r1) and
// first column c0, the step's constants and the momenta of both iterations.
template <class T>
struct PairTile {
    const T *D, *U0, *V0, *AL;
    T *UO0, *VO0;
    int64_t N;
    int H, W, r0, r1, c0;
    T wh0, wh1, tau, rad, bnd, beta1, beta2;
};

// Both iterations of a pair launch over one block's rows. ROWSUMS: the second
// iteration's gap and restart-test sums per row and warp into rowp (the
// batched launch's per-row slots); else kept per thread in gap_acc, dot_acc
// over the block's rows (the ragged step's per-tile slot).
template <class T, bool ALPHA, bool GAP2, bool WIDE, bool ROWSUMS>
__device__ __forceinline__ void pair_pass(const PairTile<T> &p, double *rowp, double &gap_acc, double &dot_acc) {
    constexpr int VEC = 4;
    // what warps pass on per row (two rows in flight): a warp's first column
    // (d, v0', v1', u0', u1') to the warp on its left, its last column's v1'
    // (u1') to the warp on its right
    __shared__ T xf[2][4][5];
    __shared__ T xl[2][4][2];
    // the edge threads' halo column (rows wider than a block): v0, v1, u0, u1,
    // alpha, z and, for the column after the block, v0 and z one further right
    __shared__ T hst[2][8];
    extern __shared__ __align__(16) unsigned char pair_ring[];
    const int H = p.H, W = p.W;
    const int64_t N = p.N;
    const T *D = p.D, *U0 = p.U0, *V0 = p.V0, *AL = p.AL;
    const T *U1 = U0 + N, *V1 = V0 + N;
    T *UO0 = p.UO0, *VO0 = p.VO0;
    T *UO1 = UO0 + N, *VO1 = VO0 + N;
    const T wh0 = p.wh0, wh1 = p.wh1, tau = p.tau, rad = p.rad, bnd = p.bnd, beta1 = p.beta1, beta2 = p.beta2;

    const int lane = threadIdx.x & 31;
    const int c0 = WIDE ? p.c0 : 0;  // the block's first column
    const int cb = c0 + (int)threadIdx.x * VEC;
    const bool colok = cb < W;
    const bool ext = lane == 31 && cb + VEC < W;  // the next warp's first column (first iteration)
    // Rows wider than a block: the first iteration also runs on the column
    // before the block (thread 0: its v1', u1' are the left neighbours of the
    // second iteration's first column) and the column after it (the last
    // thread: its v', u' give z(v'), z(u') of the second iteration's right
    // neighbour), with the arithmetic of the blocks that own those columns.
    const bool lext = WIDE && threadIdx.x == 0 && c0 > 0;
    const bool rext = WIDE && threadIdx.x == blockDim.x - 1 && cb + VEC < W;
    const int r0 = p.r0, r1 = p.r1;
    const int s0 = r0 > 0 ? r0 - 1 : 0;       // rows of the first iteration: s0 .. s1
    const int s1 = r1 < H ? r1 : H - 1;

    auto ld = [&](const T *P, int off, T(&o)[VEC]) {
        if (colok) load_pack<T, VEC>(P + off, o);
        else
#pragma unroll
            for (int j = 0; j < VEC; ++j) o[j] = T(0);
    };
    auto zrow = [&](const T(&dd)[VEC], const T(&p0)[VEC], const T(&p0p)[VEC], const T(&p1)[VEC], T left, T(&z)[VEC]) {
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            z[j] = dd[j] + wh0 * (p0[j] - p0p[j]) + wh1 * (p1[j] - left);
            left = p1[j];
        }
    };
    auto radius = [&](const T(&al)[VEC], int j) -> T {
        if (!ALPHA) return rad;
        const T r = rad * al[j];
        return al[j] == T(0) ? T(0) : (r <= bnd ? r : bnd);
    };

    // The rows after s0 come through the ring: row r is copied into slot
    // r % 3 two steps before it is read (issued at step r - 3, read at step
    // r - 1), each thread copying and reading only its own entries, so no
    // barrier guards the ring; a slot is refilled one step after it was read.
    constexpr int NARR = ALPHA ? 6 : 5;
    constexpr int AB = VEC * (int)sizeof(T);  // bytes of one array's entries per thread
    const unsigned tid = threadIdx.x;
    auto slot_arr = [&](int r, int a) -> T * {
        return reinterpret_cast<T *>(pair_ring + (size_t)(r % kPairRing) * pair_slot_bytes<T, ALPHA, WIDE>() +
                                     ((size_t)a * 128 + tid) * AB);
    };
    auto slot_sc = [&](int r, int q) -> T * {
        return reinterpret_cast<T *>(pair_ring + (size_t)(r % kPairRing) * pair_slot_bytes<T, ALPHA, WIDE>() +
                                     (size_t)NARR * 128 * AB + ((size_t)tid * pair_scalars<WIDE>() + q) * sizeof(T));
    };
    auto issue = [&](int r) {  // one commit group per row, empty past the rows this block reads
        if (r <= s1 + 1 && r < H && colok) {
            const int o = r * W + cb;
            const T *src[6] = {D + o, V0 + o, V1 + o, U0 + o, U1 + o, ALPHA ? AL + o : nullptr};
#pragma unroll
            for (int a = 0; a < NARR; ++a)
#pragma unroll
                for (int q = 0; q < AB; q += 16) cp_async16(reinterpret_cast<char *>(slot_arr(r, a)) + q,
                                                            reinterpret_cast<const char *>(src[a]) + q);
            if (cb > 0) cp_async_small<sizeof(T)>(slot_sc(r, 0), V1 + o - 1);
            if (ext) {
                cp_async_small<sizeof(T)>(slot_sc(r, 1), D + o + VEC);
                cp_async_small<sizeof(T)>(slot_sc(r, 2), V0 + o + VEC);
                cp_async_small<sizeof(T)>(slot_sc(r, 3), V1 + o + VEC);
            }
            if (lext) {  // column c0 - 1 (v1 there is entry 0), and v1 of c0 - 2
                cp_async_small<sizeof(T)>(slot_sc(r, 4), D + o - 1);
                cp_async_small<sizeof(T)>(slot_sc(r, 5), V0 + o - 1);
                cp_async_small<sizeof(T)>(slot_sc(r, 6), U0 + o - 1);
                cp_async_small<sizeof(T)>(slot_sc(r, 7), U1 + o - 1);
                if (ALPHA) cp_async_small<sizeof(T)>(slot_sc(r, 8), AL + o - 1);
                cp_async_small<sizeof(T)>(slot_sc(r, 9), V1 + o - 2);
            }
            if (rext) {  // column c0 + 512 (d, v0, v1 there are entries 1-3), and c0 + 513
                cp_async_small<sizeof(T)>(slot_sc(r, 4), U0 + o + VEC);
                cp_async_small<sizeof(T)>(slot_sc(r, 5), U1 + o + VEC);
                if (ALPHA) cp_async_small<sizeof(T)>(slot_sc(r, 6), AL + o + VEC);
                cp_async_small<sizeof(T)>(slot_sc(r, 7), D + o + VEC + 1);
                cp_async_small<sizeof(T)>(slot_sc(r, 8), V0 + o + VEC + 1);
                cp_async_small<sizeof(T)>(slot_sc(r, 9), V1 + o + VEC + 1);
            }
        }
        cp_async_commit();
    };
    auto rd = [&](int r, int a, T(&o)[VEC]) {
        if (colok) {
            const T *p = slot_arr(r, a);
#pragma unroll
            for (int j = 0; j < VEC; ++j) o[j] = p[j];
        } else {
#pragma unroll
            for (int j = 0; j < VEC; ++j) o[j] = T(0);
        }
    };
    issue(s0 + 1);
    issue(s0 + 2);

    // first iteration: row s0 and the part of row s0 - 1 it needs (lean_rows)
    int off = s0 * W + cb;
    T dc[VEC], v0c[VEC], v1c[VEC], u0c[VEC], u1c[VEC], zc[VEC], v0p[VEC], aln[VEC];
    ld(D, off, dc);
    ld(V0, off, v0c);
    ld(V1, off, v1c);
    ld(U0, off, u0c);
    ld(U1, off, u1c);
    if (s0 > 0) ld(V0, off - W, v0p);
    else
#pragma unroll
        for (int j = 0; j < VEC; ++j) v0p[j] = T(0);
    zrow(dc, v0c, v0p, v1c, (colok && cb > 0) ? V1[off - 1] : T(0), zc);
    T x_v0 = T(0), x_z = T(0), x_d = T(0), x_v1 = T(0);
    if (ext) {
        x_d = D[off + VEC];
        x_v0 = V0[off + VEC];
        x_v1 = V1[off + VEC];
        const T pv = s0 > 0 ? V0[off + VEC - W] : T(0);
        x_z = x_d + wh0 * (x_v0 - pv) + wh1 * (x_v1 - v1c[VEC - 1]);
    }
    // the halo column's row s0 (in shared memory: two threads use it)
    if (lext) {
        const int o = off - 1;
        T *hs = hst[0];
        hs[0] = V0[o];
        hs[1] = V1[o];
        hs[2] = U0[o];
        hs[3] = U1[o];
        hs[4] = ALPHA ? AL[o] : T(0);
        const T pv = s0 > 0 ? V0[o - W] : T(0);
        hs[5] = D[o] + wh0 * (hs[0] - pv) + wh1 * (hs[1] - V1[o - 1]);
        hs[6] = hs[7] = T(0);
    }
    if (rext) {
        const int o = off + VEC;
        T *hs = hst[1];
        hs[0] = x_v0;
        hs[1] = x_v1;
        hs[2] = U0[o];
        hs[3] = U1[o];
        hs[4] = ALPHA ? AL[o] : T(0);
        hs[5] = x_z;
        hs[6] = V0[o + 1];
        const T pv = s0 > 0 ? V0[o + 1 - W] : T(0);
        hs[7] = D[o + 1] + wh0 * (hs[6] - pv) + wh1 * (V1[o + 1] - x_v1);
    }
    // the second iteration's inputs on the row above: v', u', alpha, and z(v'),
    // z(u') on five columns (the last the right neighbour's first)
    T pv0[VEC], pv1[VEC], pu0[VEC], pu1[VEC], pal[VEC], zp[VEC + 1], zup[VEC + 1];
#pragma unroll
    for (int j = 0; j < VEC; ++j) pv0[j] = pv1[j] = pu0[j] = pu1[j] = pal[j] = T(0);
#pragma unroll
    for (int j = 0; j <= VEC; ++j) zp[j] = zup[j] = T(0);
    T xv0p = T(0), xu0p = T(0);  // lane 31: v0', u0' of the right neighbour's first column, row above

    // the second iteration on row j from z(v') (and z(u')) of rows j and j + 1
    auto second = [&](int j, bool hasn, const T(&zq)[VEC + 1], const T(&zuq)[VEC + 1]) {
        if (colok) {
            T uo0[VEC], uo1[VEC], vo0[VEC], vo1[VEC];
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                const bool hasr = cb + q + 1 < W;
                const T zright = q + 1 < VEC ? zp[q + 1] : zp[VEC];
                const T g0 = hasn ? wh0 * (zq[q] - zp[q]) : T(0);
                const T g1 = hasr ? wh1 * (zright - zp[q]) : T(0);
                const T cv0 = pv0[q] + tau * g0;
                const T cv1 = pv1[q] + tau * g1;
                const T nn = cv0 * cv0 + cv1 * cv1;
                const T rp = radius(pal, q);
                const T sc = nn > rp * rp ? rp * rsqrt_t(nn) : T(1);
                const T un0 = cv0 * sc, un1 = cv1 * sc;
                if (GAP2) dot_acc += (double)((pv0[q] - un0) * (un0 - pu0[q]) + (pv1[q] - un1) * (un1 - pu1[q]));
                vo0[q] = un0 + beta2 * (un0 - pu0[q]);
                vo1[q] = un1 + beta2 * (un1 - pu1[q]);
                uo0[q] = un0;
                uo1[q] = un1;
                if (GAP2) {
                    const T zuright = q + 1 < VEC ? zup[q + 1] : zup[VEC];
                    const T gu0 = hasn ? wh0 * (zuq[q] - zup[q]) : T(0);
                    const T gu1 = hasr ? wh1 * (zuright - zup[q]) : T(0);
                    gap_acc += (double)(rp * sqrt_t(gu0 * gu0 + gu1 * gu1) - (gu0 * pu0[q] + gu1 * pu1[q]));
                }
            }
            const int o = j * W + cb;
            store_pack<T, VEC>(UO0 + o, uo0);
            store_pack<T, VEC>(UO1 + o, uo1);
            store_pack<T, VEC>(VO0 + o, vo0);
            store_pack<T, VEC>(VO1 + o, vo1);
        }
        if (GAP2 && ROWSUMS) {
            // this row's sums over the warp (a fixed tree), per warp in shared
            // memory, as lean_rows: rowp[(row - r0) * 8 + 2 * warp + (0: gap, 1: dot)]
            double gv = gap_acc, dv = dot_acc;
            for (int o = 16; o > 0; o >>= 1) {
                gv += __shfl_down_sync(0xffffffffu, gv, o);
                dv += __shfl_down_sync(0xffffffffu, dv, o);
            }
            if (lane == 0) {
                rowp[(j - r0) * 8 + 2 * (threadIdx.x >> 5) + 0] = gv;
                rowp[(j - r0) * 8 + 2 * (threadIdx.x >> 5) + 1] = dv;
            }
            gap_acc = dot_acc = 0.0;
        }
    };

    if (ALPHA) ld(AL, off, aln);
    for (int i = s0; i <= s1; ++i) {
        const bool hasn = i + 1 < H;
        const int offn = off + W;
        T dn[VEC], v0n[VEC], v1n[VEC], u0n[VEC], u1n[VEC], zn[VEC], al[VEC];
        T nx_v0 = T(0), nx_z = T(0), nx_d = T(0), nx_v1 = T(0);
#pragma unroll
        for (int j = 0; j < VEC; ++j) al[j] = aln[j];
        cp_async_wait<1>();  // row i + 1 is in (row i + 2 may still be in flight)
        if (hasn) {
            rd(i + 1, 0, dn);
            rd(i + 1, 1, v0n);
            rd(i + 1, 2, v1n);
            rd(i + 1, 3, u0n);
            rd(i + 1, 4, u1n);
            if (ALPHA) rd(i + 1, 5, aln);
            zrow(dn, v0n, v0c, v1n, (colok && cb > 0) ? *slot_sc(i + 1, 0) : T(0), zn);
            if (ext) {
                nx_d = *slot_sc(i + 1, 1);
                nx_v0 = *slot_sc(i + 1, 2);
                nx_v1 = *slot_sc(i + 1, 3);
                nx_z = nx_d + wh0 * (nx_v0 - x_v0) + wh1 * (nx_v1 - v1n[VEC - 1]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < VEC; ++j) zn[j] = u0n[j] = u1n[j] = v0n[j] = v1n[j] = dn[j] = T(0);
        }
        // the first iteration on row i at the halo column, as its owner computes it
        T hun0 = T(0), hun1 = T(0), hvo0 = T(0), hvo1 = T(0);
        if (lext || rext) {
            T *hs = hst[lext ? 0 : 1];  // row i
            T n[8] = {T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0)};  // row i + 1
            if (hasn && lext) {  // column c0 - 1
                n[0] = *slot_sc(i + 1, 5);
                n[1] = *slot_sc(i + 1, 0);
                n[2] = *slot_sc(i + 1, 6);
                n[3] = *slot_sc(i + 1, 7);
                if (ALPHA) n[4] = *slot_sc(i + 1, 8);
                n[5] = *slot_sc(i + 1, 4) + wh0 * (n[0] - hs[0]) + wh1 * (n[1] - *slot_sc(i + 1, 9));
            }
            if (hasn && rext) {  // column c0 + 512, and v0, z at c0 + 513
                n[0] = nx_v0;
                n[1] = nx_v1;
                n[2] = *slot_sc(i + 1, 4);
                n[3] = *slot_sc(i + 1, 5);
                if (ALPHA) n[4] = *slot_sc(i + 1, 6);
                n[5] = nx_z;
                n[6] = *slot_sc(i + 1, 8);
                n[7] = *slot_sc(i + 1, 7) + wh0 * (n[6] - hs[6]) + wh1 * (*slot_sc(i + 1, 9) - nx_v1);
            }
            // z there, below it and to its right (this thread's first column
            // for c0 - 1, column c0 + 513 for c0 + 512)
            const T zh = hs[5], zhn = n[5], zhr = lext ? zc[0] : hs[7];
            const T g0 = hasn ? wh0 * (zhn - zh) : T(0);
            const T g1 = wh1 * (zhr - zh);
            const T cv0 = hs[0] + tau * g0;
            const T cv1 = hs[1] + tau * g1;
            const T nn = cv0 * cv0 + cv1 * cv1;
            T rp = rad;
            if (ALPHA) {
                const T r = rad * hs[4];
                rp = hs[4] == T(0) ? T(0) : (r <= bnd ? r : bnd);
            }
            const T sc = nn > rp * rp ? rp * rsqrt_t(nn) : T(1);
            hun0 = cv0 * sc;
            hun1 = cv1 * sc;
            hvo0 = hun0 + beta1 * (hun0 - hs[2]);
            hvo1 = hun1 + beta1 * (hun1 - hs[3]);
#pragma unroll
            for (int q = 0; q < 8; ++q) hs[q] = n[q];
        }
        issue(i + 3);  // into the slot of row i, read at the last step
        T zr = __shfl_down_sync(0xffffffffu, zc[0], 1);
        if (lane == 31) zr = x_z;
        // the first iteration on row i
        T un0[VEC], un1[VEC], vo0[VEC], vo1[VEC];
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            const bool hasr = cb + j + 1 < W;
            const T zright = j + 1 < VEC ? zc[j + 1] : zr;
            const T g0 = hasn ? wh0 * (zn[j] - zc[j]) : T(0);
            const T g1 = hasr ? wh1 * (zright - zc[j]) : T(0);
            const T cv0 = v0c[j] + tau * g0;
            const T cv1 = v1c[j] + tau * g1;
            const T nn = cv0 * cv0 + cv1 * cv1;
            const T rp = radius(al, j);
            const T sc = nn > rp * rp ? rp * rsqrt_t(nn) : T(1);
            un0[j] = cv0 * sc;
            un1[j] = cv1 * sc;
            vo0[j] = un0[j] + beta1 * (un0[j] - u0c[j]);
            vo1[j] = un1[j] + beta1 * (un1[j] - u1c[j]);
        }
        const int w = (int)(threadIdx.x >> 5);
        if (colok) {
            if (lane == 0) {
                xf[i & 1][w][0] = dc[0];
                xf[i & 1][w][1] = vo0[0];
                xf[i & 1][w][2] = vo1[0];
                if (GAP2) {
                    xf[i & 1][w][3] = un0[0];
                    xf[i & 1][w][4] = un1[0];
                }
            }
            if (lane == 31) {
                xl[i & 1][w][0] = vo1[VEC - 1];
                if (GAP2) xl[i & 1][w][1] = un1[VEC - 1];
            }
        }
        __syncthreads();
        // the left neighbour's last v1' (u1'), and the right neighbour's first column
        T lv1 = __shfl_up_sync(0xffffffffu, vo1[VEC - 1], 1);
        T lu1 = GAP2 ? __shfl_up_sync(0xffffffffu, un1[VEC - 1], 1) : T(0);
        if (lane == 0) {
            lv1 = w > 0 ? xl[i & 1][w - 1][0] : (lext ? hvo1 : T(0));
            if (GAP2) lu1 = w > 0 ? xl[i & 1][w - 1][1] : (lext ? hun1 : T(0));
        }
        const bool hasx = lane == 31 && colok && cb + VEC < W;
        T nd = T(0), nv0 = T(0), nv1 = T(0), nu0 = T(0), nu1 = T(0);
        if (rext) {
            nd = x_d;
            nv0 = hvo0;
            nv1 = hvo1;
            nu0 = hun0;
            nu1 = hun1;
        } else if (hasx) {
            nd = xf[i & 1][w + 1][0];
            nv0 = xf[i & 1][w + 1][1];
            nv1 = xf[i & 1][w + 1][2];
            if (GAP2) {
                nu0 = xf[i & 1][w + 1][3];
                nu1 = xf[i & 1][w + 1][4];
            }
        }
        if (i >= r0) {
            // z(v') and z(u') on row i: own columns, and the right neighbour's first
            T zq[VEC + 1], zuq[VEC + 1], pr[VEC];
#pragma unroll
            for (int j = 0; j < VEC; ++j) pr[j] = i > 0 ? pv0[j] : T(0);
            zrow(dc, vo0, pr, vo1, lv1, reinterpret_cast<T(&)[VEC]>(zq));
            zq[VEC] = __shfl_down_sync(0xffffffffu, zq[0], 1);
            if (lane == 31)
                zq[VEC] = hasx ? nd + wh0 * (nv0 - (i > 0 ? xv0p : T(0))) + wh1 * (nv1 - vo1[VEC - 1]) : T(0);
            if (GAP2) {
#pragma unroll
                for (int j = 0; j < VEC; ++j) pr[j] = i > 0 ? pu0[j] : T(0);
                zrow(dc, un0, pr, un1, lu1, reinterpret_cast<T(&)[VEC]>(zuq));
                zuq[VEC] = __shfl_down_sync(0xffffffffu, zuq[0], 1);
                if (lane == 31)
                    zuq[VEC] = hasx ? nd + wh0 * (nu0 - (i > 0 ? xu0p : T(0))) + wh1 * (nu1 - un1[VEC - 1]) : T(0);
            }
            if (i - 1 >= r0) second(i - 1, true, zq, zuq);
#pragma unroll
            for (int j = 0; j <= VEC; ++j) {
                zp[j] = zq[j];
                if (GAP2) zup[j] = zuq[j];
            }
        }
        xv0p = nv0;
        xu0p = nu0;
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            pv0[j] = vo0[j];
            pv1[j] = vo1[j];
            pu0[j] = un0[j];
            pu1[j] = un1[j];
            if (ALPHA) pal[j] = al[j];
            dc[j] = dn[j];
            v0c[j] = v0n[j];
            v1c[j] = v1n[j];
            u0c[j] = u0n[j];
            u1c[j] = u1n[j];
            zc[j] = zn[j];
        }
        x_v0 = nx_v0;
        x_z = nx_z;
        x_d = nx_d;
        x_v1 = nx_v1;
        off = offn;
    }
    cp_async_wait<0>();
    // the last row of the image has no row below
    if (r1 == H && H - 1 >= r0) {
        T zq[VEC + 1];
#pragma unroll
        for (int j = 0; j <= VEC; ++j) zq[j] = T(0);
        second(H - 1, false, zq, zq);
    }
}

template <class T, bool ALPHA, bool GAP2, bool WIDE>
__global__ void __launch_bounds__(128, GAP2 ? 3 : 4) iso2d_pair_kernel(StepArgs A, IsoCall c, IsoBuffers bf) {
    __shared__ double rowp[GAP2 ? kLeanRowsMax * 8 : 1];
    __shared__ double sh[32];
    __shared__ int flag;
    asm volatile("griddepcontrol.wait;" ::: "memory");  // a programmatic dependent of the previous step
    const int b = step_image(bf, blockIdx.z);
    if (b < 0) return;
    const IsoState st = bf.st[b];
    if (st.status != kLive) return;
    const int it = st.it;
    if (it <= 0 || (it & 3) != (GAP2 ? 3 : 1) || it + 1 >= A.max_iter || st.zero_in) {
        if (threadIdx.x == 0) atomicExch(bf.err, 3);
        return;
    }
    const IsoImage im = bf.img[b];
    const int H = (int)A.g.L[0];
    const int64_t N = A.g.N;
    const int pin = A.par, pout = A.par ^ 1;
    PairTile<T> p;
    p.D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    p.U0 = static_cast<const T *>(bf.U[pin]) + (int64_t)b * 2 * N;
    p.V0 = st.vsel ? p.U0 : static_cast<const T *>(bf.V[pin]) + (int64_t)b * 2 * N;
    p.AL = ALPHA ? static_cast<const T *>(bf.alpha) + (int64_t)b * c.alpha_stride : nullptr;
    p.UO0 = static_cast<T *>(bf.U[pout]) + (int64_t)b * 2 * N;
    p.VO0 = static_cast<T *>(bf.V[pout]) + (int64_t)b * 2 * N;
    p.N = N;
    p.H = H;
    p.W = (int)A.g.L[1];
    p.r0 = blockIdx.y * A.rows;
    p.r1 = min(H, p.r0 + A.rows);
    p.c0 = WIDE ? (int)blockIdx.x * kPairCols : 0;
    p.wh0 = (T)c.wh[0];
    p.wh1 = (T)c.wh[1];
    p.tau = (T)c.tau;
    p.rad = (T)im.radius;
    p.bnd = (T)im.bound;
    p.beta1 = (T)st.beta;
    p.beta2 = (T)((st.tn - 1.0) / fista_t(st.tn));
    double gap_acc = 0.0, dot_acc = 0.0;
    pair_pass<T, ALPHA, GAP2, WIDE, true>(p, rowp, gap_acc, dot_acc);
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int r0 = p.r0, r1 = p.r1;
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (GAP2) {
        // one slot per row, the sum of its warps in order (as lean_rows)
        __syncthreads();
        if ((int)threadIdx.x < r1 - r0) {
            double gv = 0.0, dv = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                gv += rowp[threadIdx.x * 8 + 2 * w];
                dv += rowp[threadIdx.x * 8 + 2 * w + 1];
            }
            const int64_t slot = WIDE ? (int64_t)(r0 + (int)threadIdx.x) * gridDim.x + blockIdx.x
                                      : (int64_t)(r0 + (int)threadIdx.x);
            part[slot * 2 + 0] = gv;
            part[slot * 2 + 1] = dv;
        }
    }
    if (!arrive_last(bf.ticket + b, gridDim.x * gridDim.y, &flag)) return;
    const int nslot = H * (int)gridDim.x;
    const double gap = GAP2 ? sum_partials(part, nslot, 2, 0, sh) : 0.0;
    const double dot = GAP2 ? sum_partials(part, nslot, 2, 1, sh) : 0.0;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2 = st;
    control(s2, im, A.max_iter, false, false, 0.0, 0.0, pin, bf.live);
    if (GAP2) {
        // the check is at u'; the update to u'' (in pout) stands unless it
        // passes, and then the final u is u', formed again from pin
        control(s2, im, A.max_iter, true, true, gap, dot, pin, bf.live);
        if (s2.status != kLive) {
            s2.redo = 1;
            s2.redo_vsel = st.vsel;
        }
    } else {
        control(s2, im, A.max_iter, false, false, 0.0, 0.0, pin, bf.live);
    }
    bf.st[b] = s2;
}

// The final iterate of the images whose checked pair passed at its first
// iterate u' (state redo): u' formed again from the pair's input buffers (the
// state's fin_par, reading v = u when redo_vsel) with the pair's first-
// iteration arithmetic (the same expressions, so the same bits), into the
// other parity's u; iso2d_redo_state then points fin_par there.
template <class T, bool ALPHA>
__global__ void __launch_bounds__(256) iso2d_redo_kernel(Geometry g, IsoCall c, IsoBuffers bf) {
    const int b = (int)blockIdx.y;
    const IsoState st = bf.st[b];
    if (st.redo != 1) return;
    const IsoImage im = bf.img[b];
    const int H = (int)g.L[0], W = (int)g.L[1];
    const int64_t N = g.N;
    const int pin = st.fin_par, pout = pin ^ 1;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *U0 = static_cast<const T *>(bf.U[pin]) + (int64_t)b * 2 * N;
    const T *V0 = st.redo_vsel ? U0 : static_cast<const T *>(bf.V[pin]) + (int64_t)b * 2 * N;
    const T *V1 = V0 + N;
    T *UO0 = static_cast<T *>(bf.U[pout]) + (int64_t)b * 2 * N;
    T *UO1 = UO0 + N;
    const T *AL = ALPHA ? static_cast<const T *>(bf.alpha) + (int64_t)b * c.alpha_stride : nullptr;
    const T wh0 = (T)c.wh[0], wh1 = (T)c.wh[1], tau = (T)c.tau;
    const T rad = (T)im.radius, bnd = (T)im.bound;
    auto zat = [&](int r, int q) -> T {  // z(v) at (r, q), as the pair's rows form it
        const int64_t o = (int64_t)r * W + q;
        const T up = r > 0 ? V0[o - W] : T(0);
        const T left = q > 0 ? V1[o - 1] : T(0);
        return D[o] + wh0 * (V0[o] - up) + wh1 * (V1[o] - left);
    };
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(p / W), q = (int)(p % W);
        const T z = zat(r, q);
        const T g0 = r + 1 < H ? wh0 * (zat(r + 1, q) - z) : T(0);
        const T g1 = q + 1 < W ? wh1 * (zat(r, q + 1) - z) : T(0);
        const T cv0 = V0[p] + tau * g0;
        const T cv1 = V1[p] + tau * g1;
        const T nn = cv0 * cv0 + cv1 * cv1;
        const T rp = pixel_radius<T, ALPHA>(rad, bnd, AL, p);
        const T sc = nn > rp * rp ? rp * rsqrt_t(nn) : T(1);
        UO0[p] = cv0 * sc;
        UO1[p] = cv1 * sc;
    }
}

__global__ void iso2d_redo_state(IsoState *st, int64_t B) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < B && st[i].redo) {
        st[i].fin_par ^= 1;
        st[i].redo = 0;
    }
}

// ---------------------------------------------------------------------------
// Four iterations in one pass over memory (the quad launch).
//
// Iterations it .. it + 3 with it = 1 mod 4: the first three carry no check
// and no restart test, the fourth (it + 3 = 0 mod 4) carries the gap check
// of the state it starts from (the third iterate) and the restart test, so
// nothing global is decided inside the pass, and the momenta of all four are
// the ones the per-image control would set ((tn - 1) / fista_t(tn), tn
// advanced by fista_t). Only the fourth iterate's u, v are written; when the
// check passes, the final iterate is the third's u, formed again by the redo
// variant of this kernel from the pass's untouched input buffers (state
// redo = 3).
//
// Layout: each warp owns a strip of the image: a window of 64 columns (two
// per lane) marching down the block's rows, whose middle 56 columns it writes;
// one iteration needs one column of the previous iterate on each side, so the
// four iterations need 4 columns of halo on each side, and strips overlap by
// 8 columns (rows of any width; the halo columns are recomputed, their loads
// mostly hit L2). Warps never wait on each other: the iterations pass between
// lanes by shuffles only. A warp's rows are staged in a ring of shared memory
// by cp.async (every lane copies 16-byte pieces of the window's rows, three
// rows ahead of the row being read), v and u in four slots, d and the pixel
// radii (gamma alpha_p capped at bound, formed once per row, used by all four
// iterations) in eight.
//
// At step s iteration l (1..4) updates row s - l: it forms z of its input
// (iteration l - 1's output, or the staged row for l = 1) on row s - l + 1,
// the row iteration l - 1 has just produced, and updates row s - l from z on
// that row and on its own row (kept from the last step) and its carried input
// row. Each iteration is active only on the rows the block's output rows
// depend on: r0 - (4 - l) .. r1 + (4 - l).
// The per-pixel arithmetic is the lean step's (the same expressions), so the
// iterates are those of four single steps while the restart decisions agree;
// the gap and restart-test sums are formed per row and strip (a lane's two
// columns, then the warp's tree) into H x strips slots, summed in order by the
// image's last block: a fixed order of its own (an image gives the same bits
// alone and in any batch).
// Traffic per pixel and four iterations: d, u, v, alpha read once (rows of a
// block's halo again, from L2 mostly), u, v written once: about 40 B against
// 4 x 40 B for four single steps.
// ---------------------------------------------------------------------------
constexpr int kQuadWin = 64;                        // window columns of a warp: two per lane
constexpr int kQuadHalo = 4;                        // one column per iteration on each side
constexpr int kQuadOut = kQuadWin - 2 * kQuadHalo;  // columns a warp writes
constexpr int kQuadWarps = 4;                       // strips side by side per block
constexpr int kQuadAhead = 3;                       // rows in flight beyond the row being read
constexpr int kQuadSlotsUV = 4;                     // ring rows of v0, v1, u0, u1 (read at their own step)
constexpr int kQuadSlotsD = 8;                      // ring rows of d and the radii (read by all four iterations)
constexpr int kQuadRingFloats = kQuadSlotsUV * 4 * kQuadWin + kQuadSlotsD * 2 * kQuadWin;
constexpr size_t kQuadSmem = (size_t)kQuadWarps * kQuadRingFloats * sizeof(float);

// Strips of a row of W columns: one window when W <= 64 (its edges are the
// image's, so it needs no halo); else a first window at column 0 writing
// columns 0 .. 59 (no halo on the image's edge), windows at 56 k writing
// 56 k + 4 .. 56 k + 59, and a last window ending at column W writing the rest
// (9 strips for a row of 512, against 10 with a halo on every side).
__host__ __device__ constexpr int quad_strips(int W) {
    return W <= kQuadWin ? 1
                         : 2 + ((W - 2 * (kQuadWin - kQuadHalo) > 0)
                                    ? (W - 2 * (kQuadWin - kQuadHalo) + kQuadOut - 1) / kQuadOut
                                    : 0);
}
// Strip k's window (first column, a multiple of 4) and the columns it writes.
__host__ __device__ inline void quad_strip_cols(int W, int k, int &c0, int &lo, int &hi) {
    const int n = quad_strips(W);
    if (n == 1) {
        c0 = 0, lo = 0, hi = W;
    } else if (k == 0) {
        c0 = 0, lo = 0, hi = kQuadWin - kQuadHalo;
    } else if (k < n - 1) {
        c0 = k * kQuadOut, lo = c0 + kQuadHalo, hi = c0 + kQuadWin - kQuadHalo;
    } else {
        c0 = W - kQuadWin, lo = (n - 2) * kQuadOut + kQuadWin - kQuadHalo, hi = W;
    }
}

__device__ __forceinline__ void cp_async16_zfill(void *dst, const void *src, unsigned n) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(n)
                 : "memory");
}

// What one quad pass needs: an image's arrays (v = u when vsel), its
// geometry, the step's constants, the momenta of the four iterations, and
// where the per-row sums go.
struct QuadTile {
    const float *D, *U0, *V0, *AL;
    float *UO0, *VO0;
    int64_t N;
    int H, W;
    float wh0, wh1, tau, rad, bnd;
    float beta[4];
    double *rowpart;  // ROWSUMS: the image's per-row, per-strip slots
};

// The momenta of four iterations from the state's tn and beta, as the
// control would set them.
__device__ __forceinline__ void quad_betas(double tn, double beta0, float (&beta)[4]) {
    beta[0] = (float)beta0;
#pragma unroll
    for (int l = 1; l < 4; ++l) {
        const double t2 = fista_t(tn);
        beta[l] = (float)((tn - 1.0) / t2);
        tn = t2;
    }
}

// Packed float pairs (a lane's two columns): sm_100's f32x2 arithmetic, each
// half one IEEE float32 operation rounded to nearest (the same result as the
// scalar operation; nothing is fused that the scalar steps do not fuse).
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {  // a - b
    float2 d;
    asm("{.reg .b64 a, b, d;\n\t"
        "mov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
        "sub.rn.f32x2 d, a, b;\n\tmov.b64 {%0, %1}, d;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {  // a b
    float2 d;
    asm("{.reg .b64 a, b, d;\n\t"
        "mov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
        "mul.rn.f32x2 d, a, b;\n\tmov.b64 {%0, %1}, d;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {  // a b + c, one rounding
    float2 d;
    asm("{.reg .b64 a, b, c, d;\n\t"
        "mov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\tmov.b64 c, {%6, %7};\n\t"
        "fma.rn.f32x2 d, a, b, c;\n\tmov.b64 {%0, %1}, d;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

// One warp's march over a strip, rows [r0, r1) out. The pass's state: per
// level l, the input row above the one it takes next (v, u of it and z of
// v), carried from step to step; the check's z of u on that row. Each entry
// is a lane's two columns.
template <int LV>
struct QuadCarry {
    float2 cv0[LV], cv1[LV], cu0[LV], cu1[LV], cz[LV];
    float2 czu;
};

// One step s of the march: stage row s, then iteration l + 1 (l = 0 ..
// LV - 1) updates row s - l - 1 from its input rows s - l - 1 (carried) and
// s - l (the staged row for l = 0, else iteration l's output of this step).
// OUT: the last level's row is an output row of the tile (stores, and the
// check's sums); before that (the first 2 LV steps) the levels run on the rows
// above the tile with the same arithmetic and nothing leaves the warp. Rows
// outside the image have d = v = u = 0 and radius 0, so their updates give
// u = v = 0 (the zero padding of the divergence) without a branch; a lane's
// columns outside the image likewise. The left neighbour of a lane's first
// column and the right one of its second come by shuffle; lane 0 and lane 31
// read their own values there, which is wrong for their columns but only
// moves one column inward per iteration, within the window's 4-column halo.
// The arithmetic per pixel is the single step's (iso2d_lean_kernel), operation
// for operation, with each multiply-add the single step's compiler fuses
// written as one fused operation here.
template <bool ALPHA, bool REDO, bool ROWSUMS, bool OUT, int LV>
__device__ __forceinline__ void quad_step(const QuadTile &p, QuadCarry<LV> &q, int s, int ustart, int strip,
                                          float *ruv, float *rd, int wc, bool outcol, bool ledge, float wh1r1,
                                          double &gsum, double &dsum, float *uo, float *vo) {
    const int H = p.H, W = p.W;
    const float2 W0 = make_float2(p.wh0, p.wh0), W1 = make_float2(p.wh1, p.wh1), WR = make_float2(p.wh1, wh1r1);
    const float2 TAU = make_float2(p.tau, p.tau);
    auto ld2 = [](const float *a) { return *reinterpret_cast<const float2 *>(a); };
    const float *rs = ruv + (s & (kQuadSlotsUV - 1)) * 4 * kQuadWin + wc;
    float2 nv0 = ld2(rs + 0 * kQuadWin), nv1 = ld2(rs + 1 * kQuadWin);
    float2 nu0 = ld2(rs + 2 * kQuadWin), nu1 = ld2(rs + 3 * kQuadWin);
#pragma unroll
    for (int l = 0; l < LV; ++l) {
        const int rn = s - l, r = rn - 1;  // this level's new input row; the row it updates
        const float2 dn = ld2(rd + (rn & (kQuadSlotsD - 1)) * 2 * kQuadWin + wc);
        const float sl = __shfl_up_sync(0xffffffffu, nv1.y, 1);
        const float left = ledge ? 0.f : sl;
        // z = d + wh0 (v0 - v0 above) + wh1 (v1 - v1 left)
        const float2 nz = fma2(W1, sub2(nv1, make_float2(left, nv1.x)), fma2(W0, sub2(nv0, q.cv0[l]), dn));
        const bool last = l == LV - 1;
        const bool check = !REDO && last;
        float2 nzu = make_float2(0.f, 0.f);
        if (check) {  // z of the third iterate's u on row rn
            const float slu = __shfl_up_sync(0xffffffffu, nu1.y, 1);
            const float lu = ledge ? 0.f : slu;
            nzu = fma2(W1, sub2(nu1, make_float2(lu, nu1.x)), fma2(W0, sub2(nu0, q.cu0[l]), dn));
        }
        const float wh0n = rn < H ? p.wh0 : 0.f;  // no vertical difference on the image's last row
        const float2 W0N = make_float2(wh0n, wh0n);
        const float zr = __shfl_down_sync(0xffffffffu, q.cz[l].x, 1);
        const float2 rp = ld2(rd + ((r & (kQuadSlotsD - 1)) * 2 + 1) * kQuadWin + wc);
        float2 un0, un1, ov0, ov1;
        // above the tile, level l's updates are first needed at step ustart + 2 l
        // (their rows feed the output rows' halo); before it only its z and
        // carried rows are kept, and its output is not read
        if (OUT || s >= ustart + 2 * l) {
            const float2 g0 = mul2(W0N, sub2(nz, q.cz[l]));
            const float2 g1 = mul2(WR, sub2(make_float2(q.cz[l].y, zr), q.cz[l]));
            const float2 a0 = fma2(TAU, g0, q.cv0[l]);
            const float2 a1 = fma2(TAU, g1, q.cv1[l]);
            const float2 nn = fma2(a0, a0, mul2(a1, a1));
            const float2 rr = mul2(rp, rp);
            const float2 pr = mul2(rp, make_float2(rsqrt_t(nn.x), rsqrt_t(nn.y)));
            const float2 sc = make_float2(nn.x > rr.x ? pr.x : 1.f, nn.y > rr.y ? pr.y : 1.f);
            un0 = mul2(a0, sc);
            un1 = mul2(a1, sc);
            const float2 B = make_float2(p.beta[l], p.beta[l]);
            ov0 = fma2(B, sub2(un0, q.cu0[l]), un0);
            ov1 = fma2(B, sub2(un1, q.cu1[l]), un1);
        } else {
            un0 = un1 = ov0 = ov1 = make_float2(0.f, 0.f);
        }
        if (OUT && last) {
            if (check) {
                // the restart test's dot (v - u_new)(u_new - u) and the gap at
                // the third iterate u with z of it
                const float2 dd = fma2(sub2(q.cv0[l], un0), sub2(un0, q.cu0[l]),
                                       mul2(sub2(q.cv1[l], un1), sub2(un1, q.cu1[l])));
                const float zur = __shfl_down_sync(0xffffffffu, q.czu.x, 1);
                const float2 gu0 = mul2(W0N, sub2(nzu, q.czu));
                const float2 gu1 = mul2(WR, sub2(make_float2(q.czu.y, zur), q.czu));
                const float2 gg = fma2(gu0, gu0, mul2(gu1, gu1));
                const float2 in = fma2(gu0, q.cu0[l], mul2(gu1, q.cu1[l]));
                const float t0 = fmaf(rp.x, sqrtf(gg.x), -in.x), t1 = fmaf(rp.y, sqrtf(gg.y), -in.y);
                double gacc = 0.0, dacc = 0.0;
                if (outcol) {
                    dacc = (double)dd.x;
                    gacc = (double)t0;
                    dacc += (double)dd.y;
                    gacc += (double)t1;
                }
                if (ROWSUMS) {
                    // this row's sums over the strip (a fixed tree) into its slot
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        gacc += __shfl_down_sync(0xffffffffu, gacc, o);
                        dacc += __shfl_down_sync(0xffffffffu, dacc, o);
                    }
                    if ((threadIdx.x & 31) == 0) {
                        double *part = p.rowpart + ((int64_t)r * quad_strips(W) + strip) * 2;
                        part[0] = gacc;
                        part[1] = dacc;
                    }
                } else {
                    gsum += gacc;
                    dsum += dacc;
                }
            }
            if (outcol) {  // the pass's output row
                const int64_t o = (int64_t)r * W;
                *reinterpret_cast<float2 *>(uo + o) = un0;
                *reinterpret_cast<float2 *>(uo + p.N + o) = un1;
                if (!REDO) {
                    *reinterpret_cast<float2 *>(vo + o) = ov0;
                    *reinterpret_cast<float2 *>(vo + p.N + o) = ov1;
                }
            }
        }
        // carry: this level's input row becomes the one above its next; the
        // next level's new input row is this level's output
        q.cv0[l] = nv0;
        q.cv1[l] = nv1;
        q.cu0[l] = nu0;
        q.cu1[l] = nu1;
        q.cz[l] = nz;
        if (check) q.czu = nzu;
        nv0 = ov0;
        nv1 = ov1;
        nu0 = un0;
        nu1 = un1;
    }
}

// The march of one warp over strip `strip`, output rows [r0, r1): steps
// r0 - LV .. r1 + LV - 1, a row staged per step (three ahead), the first 2 LV
// steps before any output row. REDO: three iterations, the third's u written.
// ROWSUMS: each output row's gap and restart-test sums over the strip into
// p.rowpart[row x strips + strip] (the batched launch); else they accumulate
// per lane in gsum, dsum (the ragged step's per-tile slot).
template <bool ALPHA, bool REDO, bool ROWSUMS>
__device__ __forceinline__ void quad_pass(const QuadTile &p, int strip, int r0, int r1, double &gsum,
                                          double &dsum) {
    constexpr int LV = REDO ? 3 : 4;  // iterations of the pass
    extern __shared__ __align__(16) float quad_ring[];
    const int H = p.H, W = p.W;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *ring = quad_ring + warp * kQuadRingFloats;
    float *ruv = ring;                                  // [slot][v0, v1, u0, u1][64]
    float *rd = ring + kQuadSlotsUV * 4 * kQuadWin;     // [slot][d, radius][64]
    int C0, lo, hi;  // the window's first column (a multiple of 4); the columns it writes
    quad_strip_cols(W, strip, C0, lo, hi);
    const int wc = 2 * lane;                            // this lane's first window column
    const int col = C0 + wc;
    const bool colin = col < W;                         // both columns (W and col are even)
    const bool outcol = col >= lo && col < hi;          // written columns (lo, hi multiples of 4)
    const bool ledge = C0 == 0 && lane == 0;            // column 0: its left neighbour is the zero padding
    const float wh1r1 = col + 2 < W ? p.wh1 : 0.f;      // the second column's right difference
    const float radl = colin ? p.rad : 0.f;             // the radius of this lane's columns (no pixel weights)
    // the copies: 16-byte pieces of the window's rows, a piece per lane and
    // array; pieces outside the image are zero-filled (from a valid address)
    const int ch = lane & 15, half = lane >> 4;
    const int cc = C0 + 4 * ch;
    const bool colok = cc >= 0 && cc < W;
    const int ccs = colok ? cc : 0;
    const float *src_v = (half ? p.V0 + p.N : p.V0) + ccs;
    const float *src_u = (half ? p.U0 + p.N : p.U0) + ccs;
    const float *src_d = (half ? p.AL : p.D) + ccs;
    float *dst_v = ruv + half * kQuadWin + 4 * ch;
    float *dst_u = ruv + (2 + half) * kQuadWin + 4 * ch;
    float *dst_d = rd + half * kQuadWin + 4 * ch;
    const bool copy_d = ALPHA || half == 0;
    auto issue = [&](int row, int se) {
        if (row <= se) {
            const bool rowin = (unsigned)row < (unsigned)H;
            const int64_t ro = (int64_t)(rowin ? row : 0) * W;
            const unsigned n = rowin && colok ? 16u : 0u;
            cp_async16_zfill(dst_v + (row & (kQuadSlotsUV - 1)) * 4 * kQuadWin, src_v + ro, n);
            cp_async16_zfill(dst_u + (row & (kQuadSlotsUV - 1)) * 4 * kQuadWin, src_u + ro, n);
            if (copy_d) cp_async16_zfill(dst_d + (row & (kQuadSlotsD - 1)) * 2 * kQuadWin, src_d + ro, n);
        }
        cp_async_commit();
    };
    QuadCarry<LV> q;
#pragma unroll
    for (int l = 0; l < LV; ++l) q.cv0[l] = q.cv1[l] = q.cu0[l] = q.cu1[l] = q.cz[l] = make_float2(0.f, 0.f);
    q.czu = make_float2(0.f, 0.f);
    float *uo = p.UO0 + (colin ? col : 0), *vo = p.VO0 + (colin ? col : 0);
    const int sb = r0 - LV, se = r1 + LV - 1, ustart = r0 - LV + 2;
    for (int k = 0; k < kQuadAhead; ++k) issue(sb + k, se);
    // stage row s: wait for its copies, then the radius row in place (this
    // lane's own entries): gamma alpha capped at the bound, 0 where alpha is 0
    // or outside the image
    auto stage = [&](int s) {
        __syncwarp();  // every lane is past its reads of the slots refilled now
        issue(s + kQuadAhead, se);
        cp_async_wait<kQuadAhead>();
        __syncwarp();  // row s is in, from every lane's copies
        float *ra = rd + ((s & (kQuadSlotsD - 1)) * 2 + 1) * kQuadWin + wc;
        float rp[2];
        if (ALPHA) {
            const float2 al = *reinterpret_cast<const float2 *>(ra);
            const float r0f = p.rad * al.x, r1f = p.rad * al.y;
            rp[0] = al.x == 0.f ? 0.f : (r0f <= p.bnd ? r0f : p.bnd);
            rp[1] = al.y == 0.f ? 0.f : (r1f <= p.bnd ? r1f : p.bnd);
        } else {
            rp[0] = rp[1] = (unsigned)s < (unsigned)H ? radl : 0.f;
        }
        *reinterpret_cast<float2 *>(ra) = make_float2(rp[0], rp[1]);
    };
    int s = sb;
    for (; s < r0 + LV; ++s) {  // the rows above the tile
        stage(s);
        quad_step<ALPHA, REDO, ROWSUMS, false, LV>(p, q, s, ustart, strip, ruv, rd, wc, outcol, ledge, wh1r1, gsum, dsum, uo, vo);
    }
    for (; s <= se; ++s) {  // output rows
        stage(s);
        quad_step<ALPHA, REDO, ROWSUMS, true, LV>(p, q, s, ustart, strip, ruv, rd, wc, outcol, ledge, wh1r1, gsum,
                                                  dsum, uo, vo);
    }
    cp_async_wait<0>();
}

// The per-image control after a quad pass: three plain iterations, then the
// fourth with the check at the third iterate and the restart test; the update
// to the fourth (in the other parity) stands unless the check passes, and then
// the final u is the third's, formed again from pin by the redo.
__device__ __forceinline__ void quad_control(const IsoState &st, const IsoImage &im, int max_iter, double gap,
                                             double dot, int pin, int *live, IsoState *out) {
    IsoState s2 = st;
    for (int l = 0; l < 3; ++l) control(s2, im, max_iter, false, false, 0.0, 0.0, pin, live);
    control(s2, im, max_iter, true, true, gap, dot, pin, live);
    if (s2.status != kLive) {
        s2.redo = 3;
        s2.redo_vsel = st.vsel;
        s2.redo_tn = st.tn;
        s2.redo_beta = st.beta;
    }
    *out = s2;
}

// REDO: the final iterate (the third's u) of images whose quad's check passed
// (state redo == 3), from that quad's input buffers (fin_par, v = u when
// redo_vsel) and momenta (redo_tn, redo_beta), into the other parity's u.
template <bool ALPHA, bool REDO>
__global__ void __launch_bounds__(32 * kQuadWarps, 4) iso2d_quad_kernel(StepArgs A, IsoCall c, IsoBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    if (!REDO) asm volatile("griddepcontrol.wait;" ::: "memory");  // a programmatic dependent of the previous step
    const int b = REDO ? (int)blockIdx.z : step_image(bf, blockIdx.z);
    if (b < 0) return;
    const IsoState st = bf.st[b];
    if (REDO) {
        if (st.redo != 3) return;
    } else {
        if (st.status != kLive) return;
        const int it = st.it;
        if (it <= 0 || (it & 3) != 1 || it + 3 >= A.max_iter || st.zero_in) {
            if (threadIdx.x == 0) atomicExch(bf.err, 3);
            return;
        }
    }
    const IsoImage im = bf.img[b];
    const int H = (int)A.g.L[0], W = (int)A.g.L[1];
    const int64_t N = A.g.N;
    const int pin = REDO ? st.fin_par : A.par, pout = pin ^ 1;
    const bool vsel = REDO ? st.redo_vsel != 0 : st.vsel != 0;
    QuadTile p;
    p.D = static_cast<const float *>(bf.d) + (int64_t)b * N;
    p.U0 = static_cast<const float *>(bf.U[pin]) + (int64_t)b * 2 * N;
    p.V0 = vsel ? p.U0 : static_cast<const float *>(bf.V[pin]) + (int64_t)b * 2 * N;
    p.AL = ALPHA ? static_cast<const float *>(bf.alpha) + (int64_t)b * c.alpha_stride : nullptr;
    p.UO0 = static_cast<float *>(bf.U[pout]) + (int64_t)b * 2 * N;
    p.VO0 = static_cast<float *>(bf.V[pout]) + (int64_t)b * 2 * N;
    p.N = N;
    p.H = H;
    p.W = W;
    p.wh0 = (float)c.wh[0];
    p.wh1 = (float)c.wh[1];
    p.tau = (float)c.tau;
    p.rad = (float)im.radius;
    p.bnd = (float)im.bound;
    quad_betas(REDO ? st.redo_tn : st.tn, REDO ? st.redo_beta : st.beta, p.beta);
    p.rowpart = bf.part + (int64_t)b * bf.max_part * 2;
    // the block's warps take consecutive tiles (strip, band of A.rows rows) of
    // the image, strips fastest
    const int nstrips = quad_strips(W), nbands = (H + A.rows - 1) / A.rows;
    const int t = (int)blockIdx.x * kQuadWarps + (int)(threadIdx.x >> 5);
    double gs = 0.0, ds = 0.0;
    if (t < nstrips * nbands) {
        const int band = t / nstrips, r0 = band * A.rows;
        quad_pass<ALPHA, REDO, true>(p, t - band * nstrips, r0, min(H, r0 + A.rows), gs, ds);
    }
    if (REDO) return;
    __syncthreads();
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (!arrive_last(bf.ticket + b, gridDim.x * gridDim.y, &flag)) return;
    const int nslot = H * nstrips;
    const double *part = bf.part + (int64_t)b * bf.max_part * 2;
    const double gap = sum_partials(part, nslot, 2, 0, sh);
    const double dot = sum_partials(part, nslot, 2, 1, sh);
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2;
    quad_control(st, im, A.max_iter, gap, dot, pin, bf.live, &s2);
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// The ragged step: images of any size in one arena, a device-resident work
// list of (image, tile) items, each image at its own iteration with its own
// buffer parity (its state's fin_par). One launch of single steps (each
// block in the variant its image's state asks for: cold start, gap check or
// plain) per step, and on the list of 4-wide float rows two pair variants
// after it (two iterations per launch, as the batched pair launch); an
// image's blocks run in the launch its state asks for.
// ---------------------------------------------------------------------------

// Whether the ragged step's quad launch takes an image (four iterations from
// iteration 1 mod 4, not across max_iter; slots with quad tiles only).
__device__ __forceinline__ bool ragged_quad_ok(const IsoState &st, const RagSlot &sl) {
    const int it = st.it;
    return sl.nquad > 0 && it > 0 && (it & 3) == 1 && it + 3 < sl.max_iter && !st.zero_in && sl.H >= 2;
}

// The pair variant an image's state asks for in the ragged step: 0 (iterations
// 1 and 2 mod 4), 1 (3 and 4 mod 4, with the check), -1 (a single step).
// As the batched launches: after the cold first iteration, not across
// max_iter, images of two rows or more.
__device__ __forceinline__ int ragged_pair_kind(const IsoState &st, const RagSlot &sl) {
    const int it = st.it;
    if (it <= 0 || it + 1 >= sl.max_iter || st.zero_in || (it & 1) == 0 || sl.H < 2) return -1;
    return (it & 3) == 3 ? 1 : 0;
}

// One single step of an item's tile, in the variant (GAP: gap check; ZIN:
// cold start from a zero dual) its image's state asks for.
template <class T, int VEC, bool GAP, bool ZIN>
__device__ __forceinline__ void ragged_single(const RagItem &item, const RagSlot &sl, const IsoState &st,
                                              const IsoBuffers &bf, double *sh, int *flag) {
    const int b = item.slot;
    const int it = st.it;
    const IsoImage im = bf.img[b];
    const int H = sl.H, W = sl.W;
    const int64_t N = (int64_t)H * W;
    const bool do_upd = it < sl.max_iter;
    const bool test = do_upd && (it & 3) == 0;
    const int pin = st.fin_par, pout = pin ^ 1;
    const T *D = static_cast<const T *>(bf.d) + sl.off;
    const T *U0 = static_cast<const T *>(bf.U[pin]) + 2 * sl.off;
    const T *V0 = st.vsel ? U0 : static_cast<const T *>(bf.V[pin]) + 2 * sl.off;
    T *UO0 = static_cast<T *>(bf.U[pout]) + 2 * sl.off;
    T *VO0 = static_cast<T *>(bf.V[pout]) + 2 * sl.off;
    const int cb = item.cs + (int)threadIdx.x * VEC;
    const int r0 = item.r0;
    const int r1 = min(H, r0 + sl.rows);
    double gap_acc = 0.0, dot_acc = 0.0;
    lean_rows<T, VEC, false, GAP, ZIN>(D, U0, U0 + N, V0, V0 + N, UO0, UO0 + N, VO0, VO0 + N, nullptr, H, W, cb, r0, r1,
                                       (T)sl.wh0, (T)sl.wh1, (T)sl.tau, (T)st.beta, (T)im.radius, (T)im.bound, test,
                                       do_upd, gap_acc, dot_acc);
    const double gsum = GAP ? block_sum(gap_acc, sh) : 0.0;
    const double dsum = test ? block_sum(dot_acc, sh) : 0.0;
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[item.blk * 2 + 0] = gsum;
        part[item.blk * 2 + 1] = dsum;
    }
    if (!arrive_last(bf.ticket + b, sl.nblk, flag)) return;
    const double gap = GAP ? sum_partials(part, sl.nblk, 2, 0, sh) : 0.0;
    const double dot = test ? sum_partials(part, sl.nblk, 2, 1, sh) : 0.0;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2 = st;
    control(s2, im, sl.max_iter, GAP, test, gap, dot, pin, bf.live);
    bf.st[b] = s2;
}

// The single steps of a ragged step, one launch: each item's block runs the
// variant its image's state asks for (cold start, gap check or plain), or
// exits when the pair variants take the image.
template <class T, int VEC>
__global__ void __launch_bounds__(128) iso2d_ragged_kernel(const RagItem *__restrict__ items,
                                                           const int *__restrict__ n_items,
                                                           const RagSlot *__restrict__ slots, IsoBuffers bf,
                                                           int pairs) {
    __shared__ double sh[32];
    __shared__ int flag;
    if ((int)blockIdx.x >= *n_items) return;
    const RagItem item = items[blockIdx.x];
    const RagSlot sl = slots[item.slot];
    const IsoState st = bf.st[item.slot];
    if (st.status != kLive) return;
    if (ragged_quad_ok(st, sl)) return;                  // the quad takes it
    if (pairs && ragged_pair_kind(st, sl) >= 0) return;  // the pair variants take it
    const int it = st.it;
    const bool do_gap = (it > 0 && ((it & 3) == 0 || it == sl.max_iter)) || (it == 0 && st.warm);
    const bool zin = st.zero_in != 0;
    if (zin && !do_gap) ragged_single<T, VEC, false, true>(item, sl, st, bf, sh, &flag);
    else if (!zin && do_gap) ragged_single<T, VEC, true, false>(item, sl, st, bf, sh, &flag);
    else if (!zin) ragged_single<T, VEC, false, false>(item, sl, st, bf, sh, &flag);
}

// The ragged step's pair variants: an item's tile (the slot's rows x 512
// columns) of an image whose state asks for two iterations, the batched pair
// launch's pass; the tile's gap and restart-test sums go to its partial slot.
template <class T, bool GAP2>
__global__ void __launch_bounds__(128, GAP2 ? 3 : 4) iso2d_ragged_pair_kernel(const RagItem *__restrict__ items,
                                                                              const int *__restrict__ n_items,
                                                                              const RagSlot *__restrict__ slots,
                                                                              IsoBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    if ((int)blockIdx.x >= *n_items) return;
    const RagItem item = items[blockIdx.x];
    const int b = item.slot;
    const RagSlot sl = slots[b];
    const IsoState st = bf.st[b];
    if (st.status != kLive || ragged_quad_ok(st, sl) || ragged_pair_kind(st, sl) != (GAP2 ? 1 : 0)) return;
    const IsoImage im = bf.img[b];
    const int pin = st.fin_par, pout = pin ^ 1;
    PairTile<T> p;
    p.D = static_cast<const T *>(bf.d) + sl.off;
    p.U0 = static_cast<const T *>(bf.U[pin]) + 2 * sl.off;
    p.V0 = st.vsel ? p.U0 : static_cast<const T *>(bf.V[pin]) + 2 * sl.off;
    p.AL = nullptr;
    p.UO0 = static_cast<T *>(bf.U[pout]) + 2 * sl.off;
    p.VO0 = static_cast<T *>(bf.V[pout]) + 2 * sl.off;
    p.N = (int64_t)sl.H * sl.W;
    p.H = sl.H;
    p.W = sl.W;
    p.r0 = item.r0;
    p.r1 = min(sl.H, item.r0 + sl.rows);
    p.c0 = item.cs;
    p.wh0 = (T)sl.wh0;
    p.wh1 = (T)sl.wh1;
    p.tau = (T)sl.tau;
    p.rad = (T)im.radius;
    p.bnd = (T)im.bound;
    p.beta1 = (T)st.beta;
    p.beta2 = (T)((st.tn - 1.0) / fista_t(st.tn));
    double gap_acc = 0.0, dot_acc = 0.0;
    pair_pass<T, false, GAP2, true, false>(p, nullptr, gap_acc, dot_acc);
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (GAP2) {
        const double gsum = block_sum(gap_acc, sh);
        const double dsum = block_sum(dot_acc, sh);
        if (threadIdx.x == 0) {
            part[item.blk * 2 + 0] = gsum;
            part[item.blk * 2 + 1] = dsum;
        }
    }
    if (!arrive_last(bf.ticket + b, sl.nblk, &flag)) return;
    const double gap = GAP2 ? sum_partials(part, sl.nblk, 2, 0, sh) : 0.0;
    const double dot = GAP2 ? sum_partials(part, sl.nblk, 2, 1, sh) : 0.0;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2 = st;
    control(s2, im, sl.max_iter, false, false, 0.0, 0.0, pin, bf.live);
    if (GAP2) {
        // the check is at u'; the update to u'' (in pout) stands unless it
        // passes, and then the final u is u', formed again from pin
        control(s2, im, sl.max_iter, true, true, gap, dot, pin, bf.live);
        if (s2.status != kLive) {
            s2.redo = 1;
            s2.redo_vsel = st.vsel;
        }
    } else {
        control(s2, im, sl.max_iter, false, false, 0.0, 0.0, pin, bf.live);
    }
    bf.st[b] = s2;
}

// The ragged step's quad variant: an item's block of strips (the slot's quad
// rows x kQuadWarps strips) of an image whose state asks for four iterations;
// the block's gap and restart-test sums (each lane's over the block's rows,
// then the block's tree) go to the item's partial slot, summed in order by
// the image's last block.
__global__ void __launch_bounds__(32 * kQuadWarps, 4) iso2d_ragged_quad_kernel(const RagItem *__restrict__ items,
                                                                              const int *__restrict__ n_items,
                                                                              const RagSlot *__restrict__ slots,
                                                                              IsoBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    if ((int)blockIdx.x >= *n_items) return;
    const RagItem item = items[blockIdx.x];
    const int b = item.slot;
    const RagSlot sl = slots[b];
    const IsoState st = bf.st[b];
    if (st.status != kLive || !ragged_quad_ok(st, sl)) return;
    const IsoImage im = bf.img[b];
    const int pin = st.fin_par, pout = pin ^ 1;
    QuadTile p;
    p.D = static_cast<const float *>(bf.d) + sl.off;
    p.U0 = static_cast<const float *>(bf.U[pin]) + 2 * sl.off;
    p.V0 = st.vsel ? p.U0 : static_cast<const float *>(bf.V[pin]) + 2 * sl.off;
    p.AL = nullptr;
    p.UO0 = static_cast<float *>(bf.U[pout]) + 2 * sl.off;
    p.VO0 = static_cast<float *>(bf.V[pout]) + 2 * sl.off;
    p.N = (int64_t)sl.H * sl.W;
    p.H = sl.H;
    p.W = sl.W;
    p.wh0 = (float)sl.wh0;
    p.wh1 = (float)sl.wh1;
    p.tau = (float)sl.tau;
    p.rad = (float)im.radius;
    p.bnd = (float)im.bound;
    quad_betas(st.tn, st.beta, p.beta);
    p.rowpart = nullptr;
    const int strip = item.cs + (int)(threadIdx.x >> 5);
    double gs = 0.0, ds = 0.0;
    if (strip < quad_strips(sl.W)) quad_pass<false, false, false>(p, strip, item.r0, min(sl.H, item.r0 + sl.qrows), gs, ds);
    const double gsum = block_sum(gs, sh);
    const double dsum = block_sum(ds, sh);
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[item.blk * 2 + 0] = gsum;
        part[item.blk * 2 + 1] = dsum;
    }
    if (!arrive_last(bf.ticket + b, sl.nquad, &flag)) return;
    const double gap = sum_partials(part, sl.nquad, 2, 0, sh);
    const double dot = sum_partials(part, sl.nquad, 2, 1, sh);
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2;
    quad_control(st, im, sl.max_iter, gap, dot, pin, bf.live, &s2);
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// Generic step: one thread per pixel, 2D or 3D, any extents. Neighbours are
// read through the caches.
// ---------------------------------------------------------------------------

template <class T, int K, bool ALPHA>
__global__ void __launch_bounds__(256) iso_generic_kernel(StepArgs A, IsoCall c, IsoBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = step_image(bf, blockIdx.y);
    if (b < 0) return;
    const IsoState st = bf.st[b];
    if (st.status != kLive) return;
    const IsoImage im = bf.img[b];
    const int64_t N = A.g.N;
    const int it = st.it;
    const bool do_gap = (it > 0 && ((it & 3) == 0 || it == A.max_iter)) || (it == 0 && st.warm);
    const bool do_upd = it < A.max_iter;
    const bool test = do_upd && (it & 3) == 0;
    const bool zin = st.zero_in != 0;
    const int pin = A.par, pout = A.par ^ 1;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *U = static_cast<const T *>(bf.U[pin]) + (int64_t)b * K * N;
    const T *V = st.vsel ? U : static_cast<const T *>(bf.V[pin]) + (int64_t)b * K * N;
    T *UO = static_cast<T *>(bf.U[pout]) + (int64_t)b * K * N;
    T *VO = static_cast<T *>(bf.V[pout]) + (int64_t)b * K * N;
    const T *AL = ALPHA ? static_cast<const T *>(bf.alpha) + (int64_t)b * c.alpha_stride : nullptr;
    T wh[K];
    int64_t L[K], S[K];
    for (int a = 0; a < K; ++a) {
        wh[a] = (T)c.wh[a];
        L[a] = A.g.L[a];
    }
    S[K - 1] = 1;
    for (int a = K - 2; a >= 0; --a) S[a] = S[a + 1] * L[a + 1];
    const T tau = (T)c.tau, beta = (T)st.beta, rad = (T)im.radius, bnd = (T)im.bound;

    // z(P) at q, with the coordinates of q
    auto zat = [&](const T *P, int64_t q, const int64_t *co) -> T {
        T z = D[q];
        for (int a = 0; a < K; ++a) {
            if (wh[a] == T(0)) continue;
            const T cur = zin ? T(0) : P[a * N + q];
            const T prev = (zin || co[a] == 0) ? T(0) : P[a * N + q - S[a]];
            z += wh[a] * (cur - prev);
        }
        return z;
    };
    double gap_acc = 0.0, dot_acc = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        int64_t co[K];
        for (int a = 0; a < K; ++a) co[a] = (p / S[a]) % L[a];
        const T z0 = zat(V, p, co);
        T gv[K];
        for (int a = 0; a < K; ++a) {
            gv[a] = T(0);
            if (wh[a] != T(0) && co[a] + 1 < L[a]) {
                int64_t cn[K];
                for (int e = 0; e < K; ++e) cn[e] = co[e];
                cn[a] += 1;
                gv[a] = wh[a] * (zat(V, p + S[a], cn) - z0);
            }
        }
        T cv[K], uc[K], vc[K];
        T nn = T(0);
        for (int a = 0; a < K; ++a) {
            uc[a] = zin ? T(0) : U[a * N + p];
            vc[a] = zin ? T(0) : V[a * N + p];
            cv[a] = wh[a] != T(0) ? vc[a] + tau * gv[a] : T(0);
            nn += cv[a] * cv[a];
        }
        const T nr = sqrt_t(nn);
        const T rp = pixel_radius<T, ALPHA>(rad, bnd, AL, p);
        const T sc = nr > rp ? rp / nr : T(1);
        for (int a = 0; a < K; ++a) {
            const T un = cv[a] * sc;
            if (test) dot_acc += (double)((vc[a] - un) * (un - uc[a]));
            if (do_upd) {
                VO[a * N + p] = un + beta * (un - uc[a]);
                UO[a * N + p] = un;
            }
        }
        if (do_gap) {
            const T zu0 = zat(U, p, co);
            double gg = 0.0, gu = 0.0;
            for (int a = 0; a < K; ++a) {
                if (wh[a] != T(0) && co[a] + 1 < L[a]) {
                    int64_t cn[K];
                    for (int e = 0; e < K; ++e) cn[e] = co[e];
                    cn[a] += 1;
                    const double ga = (double)(wh[a] * (zat(U, p + S[a], cn) - zu0));
                    gg += ga * ga;
                    gu += ga * (double)uc[a];
                }
            }
            gap_acc += (double)rp * sqrt(gg) - gu;
        }
    }
    const unsigned nblk = gridDim.x;
    const double gsum = do_gap ? block_sum(gap_acc, sh) : 0.0;
    const double dsum = test ? block_sum(dot_acc, sh) : 0.0;
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2 + 0] = gsum;
        part[blockIdx.x * 2 + 1] = dsum;
    }
    if (!arrive_last(bf.ticket + b, nblk, &flag)) return;
    const double gap = do_gap ? sum_partials(part, nblk, 2, 0, sh) : 0.0;
    const double dot = test ? sum_partials(part, nblk, 2, 1, sh) : 0.0;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2 = st;
    control(s2, im, A.max_iter, do_gap, test, gap, dot, pin, bf.live);
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// Huber-smoothed TV (the reference's planned analysis prior, stage 1:
// ROADMAP.md "Stage 1, Huber-smoothed TV"): isotropic
// gamma sum_p alpha_p h(|(W D z)_p|), anisotropic gamma sum_{a,p}
// beta_{a,p} h(|w_a (D_a z)_p|), h the Huber function of fp_op_huber
// (src/ops/pointwise.cpp:189-206: t^2 / (2 delta) up to delta, t - delta / 2
// beyond). Its dual adds delta |q_p|^2 / (2 gamma alpha_p) (per component for
// the anisotropic form) to the TV dual: strongly convex, so dual FISTA with a
// constant momentum (V-FISTA, kappa = 1 + gamma alpha_max L / delta) converges
// linearly, with no restarts. At the solved scale, with u = wmax q and radius
// r = gamma wmax alpha: the step is u+ = P_r((v + tau G_h z(v)) / (1 + tau
// delta / (r wmax))), the projection onto the ball (isotropic) or the box per
// component (anisotropic); the gap sums, per pixel (per component),
// (r / wmax) h(wmax |g|) - <g, u> + delta |u|^2 / (2 r wmax) with g = G_h z(u):
// each a Fenchel-Young gap, so |z - z*|^2 <= 2 gap as for TV. The arithmetic is
// the generic step's (one thread per pixel, 2D and 3D); the gap test every
// fourth iteration and at max_iter, as for TV.
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ double huber_h(double t, double dl) {
    return t <= dl ? t * t / (2.0 * dl) : t - 0.5 * dl;
}

template <class T, int K, bool SW, bool ANISO>
__global__ void __launch_bounds__(256) huber_kernel(StepArgs A, IsoCall c, IsoBuffers bf) {
    __shared__ double sh[32];
    __shared__ int flag;
    const int b = step_image(bf, blockIdx.y);
    if (b < 0) return;
    const IsoState st = bf.st[b];
    if (st.status != kLive) return;
    const IsoImage im = bf.img[b];
    const int64_t N = A.g.N;
    const int it = st.it;
    const bool do_gap = (it > 0 && ((it & 3) == 0 || it == A.max_iter)) || (it == 0 && st.warm);
    const bool do_upd = it < A.max_iter;
    const bool zin = st.zero_in != 0;
    const int pin = A.par, pout = A.par ^ 1;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *U = static_cast<const T *>(bf.U[pin]) + (int64_t)b * K * N;
    const T *V = static_cast<const T *>(bf.V[pin]) + (int64_t)b * K * N;
    T *UO = static_cast<T *>(bf.U[pout]) + (int64_t)b * K * N;
    T *VO = static_cast<T *>(bf.V[pout]) + (int64_t)b * K * N;
    const T *SWp = SW ? static_cast<const T *>(bf.alpha) : nullptr;  // pixel (N) or edge (K N) weights
    T wh[K];
    int64_t L[K], S[K];
    for (int a = 0; a < K; ++a) {
        wh[a] = (T)c.wh[a];
        L[a] = A.g.L[a];
    }
    S[K - 1] = 1;
    for (int a = K - 2; a >= 0; --a) S[a] = S[a + 1] * L[a + 1];
    const T tau = (T)c.tau, beta = (T)st.beta, rad = (T)im.radius, wm = (T)c.wmax;
    const T dl = (T)ldexp(c.delta, -im.e);
    const double dld = ldexp(c.delta, -im.e), wmd = c.wmax;
    auto zat = [&](const T *P, int64_t q, const int64_t *co) -> T {
        T z = D[q];
        for (int a = 0; a < K; ++a) {
            if (wh[a] == T(0)) continue;
            const T cur = zin ? T(0) : P[a * N + q];
            const T prev = (zin || co[a] == 0) ? T(0) : P[a * N + q - S[a]];
            z += wh[a] * (cur - prev);
        }
        return z;
    };
    double gap_acc = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        int64_t co[K];
        for (int a = 0; a < K; ++a) co[a] = (p / S[a]) % L[a];
        T r[K];  // the radius of the pixel (of each component, anisotropic)
        for (int a = 0; a < K; ++a) r[a] = SW ? rad * SWp[(ANISO ? (int64_t)a * N : 0) + p] : rad;
        const T z0 = zat(V, p, co);
        T gv[K];
        for (int a = 0; a < K; ++a) {
            gv[a] = T(0);
            if (wh[a] != T(0) && co[a] + 1 < L[a]) {
                int64_t cn[K];
                for (int e = 0; e < K; ++e) cn[e] = co[e];
                cn[a] += 1;
                gv[a] = wh[a] * (zat(V, p + S[a], cn) - z0);
            }
        }
        T cv[K], uc[K], vc[K];
        for (int a = 0; a < K; ++a) {
            uc[a] = zin ? T(0) : U[a * N + p];
            vc[a] = zin ? T(0) : V[a * N + p];
            cv[a] = wh[a] != T(0) ? vc[a] + tau * gv[a] : T(0);
        }
        if (ANISO) {
            for (int a = 0; a < K; ++a) {
                if (!(r[a] > T(0))) {
                    cv[a] = T(0);
                    continue;
                }
                cv[a] *= r[a] * wm / (r[a] * wm + tau * dl);
                cv[a] = cv[a] > r[a] ? r[a] : (cv[a] < -r[a] ? -r[a] : cv[a]);
            }
        } else if (!(r[0] > T(0))) {
            for (int a = 0; a < K; ++a) cv[a] = T(0);
        } else {
            const T sc0 = r[0] * wm / (r[0] * wm + tau * dl);
            T nn = T(0);
            for (int a = 0; a < K; ++a) {
                cv[a] *= sc0;
                nn += cv[a] * cv[a];
            }
            const T nr = sqrt_t(nn);
            if (nr > r[0]) {
                const T sc = r[0] / nr;
                for (int a = 0; a < K; ++a) cv[a] *= sc;
            }
        }
        if (do_upd)
            for (int a = 0; a < K; ++a) {
                VO[a * N + p] = cv[a] + beta * (cv[a] - uc[a]);
                UO[a * N + p] = cv[a];
            }
        if (do_gap) {
            const T zu0 = zat(U, p, co);
            double gu[K];
            for (int a = 0; a < K; ++a) {
                gu[a] = 0.0;
                if (wh[a] != T(0) && co[a] + 1 < L[a]) {
                    int64_t cn[K];
                    for (int e = 0; e < K; ++e) cn[e] = co[e];
                    cn[a] += 1;
                    gu[a] = (double)(wh[a] * (zat(U, p + S[a], cn) - zu0));
                }
            }
            if (ANISO) {
                for (int a = 0; a < K; ++a) {
                    const double ra = (double)r[a], ua = (double)uc[a];
                    if (ra > 0.0) gap_acc += ra / wmd * huber_h<T>(wmd * fabs(gu[a]), dld) - gu[a] * ua +
                                             dld * ua * ua / (2.0 * ra * wmd);
                }
            } else if ((double)r[0] > 0.0) {
                double nn = 0.0, pu = 0.0, uu = 0.0;
                for (int a = 0; a < K; ++a) {
                    nn += gu[a] * gu[a];
                    pu += gu[a] * (double)uc[a];
                    uu += (double)uc[a] * (double)uc[a];
                }
                const double r0 = (double)r[0];
                gap_acc += r0 / wmd * huber_h<T>(wmd * sqrt(nn), dld) - pu + dld * uu / (2.0 * r0 * wmd);
            }
        }
    }
    const unsigned nblk = gridDim.x;
    const double gsum = do_gap ? block_sum(gap_acc, sh) : 0.0;
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2 + 0] = gsum;
        part[blockIdx.x * 2 + 1] = 0.0;
    }
    if (!arrive_last(bf.ticket + b, nblk, &flag)) return;
    const double gap = do_gap ? sum_partials(part, nblk, 2, 0, sh) : 0.0;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2 = st;
    if (do_gap) {
        s2.gp = gap;
        if (gap <= im.target || s2.it >= A.max_iter) {
            s2.status = gap <= im.target ? kConverged : kNotConv;
            s2.fin_par = pin;
            atomicSub(bf.live, 1);
            bf.st[b] = s2;
            return;
        }
    }
    s2.since += 1;
    s2.vsel = 0;
    s2.zero_in = 0;
    s2.it += 1;  // the momentum stays the constant set at the set-up
    s2.fin_par = pin ^ 1;
    bf.st[b] = s2;
}

// The set-up's last step for Huber-smoothed TV: the constant momentum of
// V-FISTA, (sqrt(kappa) - 1) / (sqrt(kappa) + 1), kappa = 1 + r_max wmax /
// (tau delta) at the solved scale (r_max the largest radius).
__global__ void huber_momentum(IsoCall c, IsoBuffers bf, int64_t B) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const IsoImage im = bf.img[b];
    if (im.mode != kModeFdpg) return;
    const double rmax = im.radius * (c.has_alpha ? c.alpha_max : 1.0);
    const double dl = ldexp(c.delta, -im.e);
    const double kappa = 1.0 + rmax * c.wmax / (c.tau * dl);
    const double sk = sqrt(kappa);
    bf.st[b].beta = (sk - 1.0) / (sk + 1.0);
}

// ---------------------------------------------------------------------------
// The 3D step: a block owns a kTY x kTX tile of the (axis 1, axis 2) plane and
// marches along axis 0 through a chunk of A.rows slices. For each slice it
// stages d and the dual of the next slice over the tile and a one-entry halo
// in shared memory (four slices in rotation, copied by cp.async three steps
// ahead), forms z of the next slice over
// the tile and its forward halo (two slices of z in rotation), and updates the
// tile at the current slice from z of this slice and of the next. Every array
// is read from HBM once per iteration; the halo entries are neighbouring
// tiles' and come from the caches. The per-pixel arithmetic is the generic
// step's (tv_iso.cpp:251-288, 499-524), the projection by rsqrt as in 2D.
// ---------------------------------------------------------------------------

constexpr int k3TX = 32, k3TY = 8;
constexpr int k3RX = k3TX + 2, k3RY = k3TY + 2, k3R = k3RX * k3RY;  // staged region: tile plus halo
constexpr int k3ZX = k3TX + 1, k3Z = (k3TY + 1) * k3ZX;              // z: tile plus forward halo
constexpr int k3Ring = 4;  // staged slices in rotation (two in use, two in flight; five ran 10% slower)

template <class T, bool ALPHA, bool GAP, bool ZIN>
__global__ void __launch_bounds__(k3TX * k3TY) iso3d_kernel(StepArgs A, IsoCall c, IsoBuffers bf) {
    constexpr int NA = GAP ? 7 : 4;  // staged arrays: d, v0..v2 (and u0..u2 for the gap)
    extern __shared__ __align__(16) unsigned char i3_smem[];
    T(*reg)[NA][k3R] = reinterpret_cast<T(*)[NA][k3R]>(i3_smem);
    T(*zs)[GAP ? 2 : 1][k3Z] = reinterpret_cast<T(*)[GAP ? 2 : 1][k3Z]>(i3_smem + k3Ring * NA * k3R * sizeof(T));
    __shared__ double sh[32];
    __shared__ int flag;
    asm volatile("griddepcontrol.wait;" ::: "memory");  // a programmatic dependent of the previous step
    const int b = step_image(bf, blockIdx.z);
    if (b < 0) return;
    const IsoState st = bf.st[b];
    if (st.status != kLive) return;
    const int it = st.it;
    const bool do_gap = (it > 0 && ((it & 3) == 0 || it == A.max_iter)) || (it == 0 && st.warm);
    const bool zin = st.zero_in != 0;
    if (do_gap != GAP || zin != ZIN) {
        if (threadIdx.x == 0) atomicExch(bf.err, 3);
        return;
    }
    const IsoImage im = bf.img[b];
    const int D0 = (int)A.g.L[0], D1 = (int)A.g.L[1], D2 = (int)A.g.L[2];
    const int64_t N = A.g.N;
    const int64_t S0 = (int64_t)D1 * D2;
    const bool do_upd = it < A.max_iter;
    const bool test = do_upd && (it & 3) == 0;
    const int pin = A.par, pout = A.par ^ 1;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *U = static_cast<const T *>(bf.U[pin]) + (int64_t)b * 3 * N;
    const T *V = st.vsel ? U : static_cast<const T *>(bf.V[pin]) + (int64_t)b * 3 * N;
    T *UO = static_cast<T *>(bf.U[pout]) + (int64_t)b * 3 * N;
    T *VO = static_cast<T *>(bf.V[pout]) + (int64_t)b * 3 * N;
    const T *AL = ALPHA ? static_cast<const T *>(bf.alpha) + (int64_t)b * c.alpha_stride : nullptr;
    const T wh0 = (T)c.wh[0], wh1 = (T)c.wh[1], wh2 = (T)c.wh[2];
    const T tau = (T)c.tau, beta = (T)st.beta, rad = (T)im.radius, bnd = (T)im.bound;
    const int tid = threadIdx.x, ty = tid / k3TX, tx = tid % k3TX;
    const int x0 = blockIdx.x * k3TX;
    const int nyt = (D1 + k3TY - 1) / k3TY;
    const int y0 = (blockIdx.y % nyt) * k3TY;
    const int s0 = (blockIdx.y / nyt) * A.rows;
    const int s1 = min(D0, s0 + A.rows);
    auto q3 = [](int sl) { return (sl + k3Ring) % k3Ring; };
    // The region entries this thread stages (tid and tid + 256): their
    // offsets in a slice and whether they lie in the image.
    constexpr int kE = (k3R + k3TX * k3TY - 1) / (k3TX * k3TY);
    int64_t poff[kE];
    bool inimg[kE];
#pragma unroll
    for (int e = 0; e < kE; ++e) {
        const int i = tid + e * k3TX * k3TY;
        const int gy = y0 - 1 + i / k3RX, gx = x0 - 1 + i % k3RX;
        inimg[e] = i < k3R && gy >= 0 && gy < D1 && gx >= 0 && gx < D2;
        poff[e] = inimg[e] ? (int64_t)gy * D2 + gx : 0;
    }
    // Slices come into the ring by cp.async (zeros outside the image), issued
    // three steps before the work on them: slice sl + 3 goes into the slot of
    // slice sl - 1 once every thread is past the last step's reads of it.
    auto issue = [&](int sl) {
        if (sl <= s1) {
            T(*r)[k3R] = reg[q3(sl)];
#pragma unroll
            for (int e = 0; e < kE; ++e) {
                const int i = tid + e * k3TX * k3TY;
                if (i < k3R) {
                    const bool in = inimg[e] && sl >= 0 && sl < D0;
                    const int64_t o = in ? (int64_t)sl * S0 + poff[e] : 0;
                    cp_async_zfill<sizeof(T)>(&r[0][i], D + o, in ? sizeof(T) : 0);
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        cp_async_zfill<sizeof(T)>(&r[1 + a][i], V + a * N + o, (in && !ZIN) ? sizeof(T) : 0);
                    if (GAP)
#pragma unroll
                        for (int a = 0; a < 3; ++a)
                            cp_async_zfill<sizeof(T)>(&r[(GAP ? 4 : 1) + a][i], U + a * N + o,
                                                      (in && !ZIN) ? sizeof(T) : 0);
                }
            }
        }
        cp_async_commit();
    };
    // z of slice sl (of v, and of u for the gap) over the tile and its forward halo
    auto zslice = [&](int sl) {
        const T(*r)[k3R] = reg[q3(sl)];
        const T(*rp)[k3R] = reg[q3(sl - 1)];
        T(*z)[k3Z] = zs[sl & 1];
        for (int i = tid; i < k3Z; i += k3TX * k3TY) {
            const int zy = i / k3ZX, zx = i % k3ZX;
            const int j = (zy + 1) * k3RX + zx + 1;
            z[0][i] = r[0][j] + wh0 * (r[1][j] - rp[1][j]) + wh1 * (r[2][j] - r[2][j - k3RX]) +
                      wh2 * (r[3][j] - r[3][j - 1]);
            if (GAP)
                z[GAP ? 1 : 0][i] = r[0][j] + wh0 * (r[4][j] - rp[4][j]) + wh1 * (r[5][j] - r[5][j - k3RX]) +
                                    wh2 * (r[6][j] - r[6][j - 1]);
        }
    };
    const int gy = y0 + ty, gx = x0 + tx;
    const bool own = gy < D1 && gx < D2;
    const int64_t ooff = own ? (int64_t)gy * D2 + gx : 0;
    // u at this thread's entry of a slice (the gap variant stages it)
    T pu[3] = {T(0), T(0), T(0)};
    auto fetch_u = [&](int sl) {
        if (GAP || ZIN || !own || sl >= s1) return;
        const int64_t o = (int64_t)sl * S0 + ooff;
#pragma unroll
        for (int a = 0; a < 3; ++a) pu[a] = U[a * N + o];
    };
    double gap_acc = 0.0, dot_acc = 0.0;
#pragma unroll
    for (int q = -1; q <= k3Ring - 2; ++q) issue(s0 + q);
    fetch_u(s0);
    cp_async_wait<k3Ring - 2>();  // slices s0 - 1 and s0 are in
    __syncthreads();
    zslice(s0);
    for (int sl = s0; sl < s1; ++sl) {
        T uc[3] = {pu[0], pu[1], pu[2]};
        if (sl + 1 < s1) fetch_u(sl + 1);
        cp_async_wait<k3Ring - 3>();  // slice sl + 1 is in (the later ones may still be in flight)
        __syncthreads();
        issue(sl + k3Ring - 1);
        zslice(sl + 1);
        __syncthreads();
        if (own) {
            const T(*r)[k3R] = reg[q3(sl)];
            const T(*zc)[k3Z] = zs[sl & 1];
            const T(*zn)[k3Z] = zs[(sl + 1) & 1];
            const int i = ty * k3ZX + tx, j = (ty + 1) * k3RX + tx + 1;
            const int64_t o = (int64_t)sl * S0 + ooff;
            const bool h0 = sl + 1 < D0, h1 = gy + 1 < D1, h2 = gx + 1 < D2;
            const T z0 = zc[0][i];
            const T g0 = h0 ? wh0 * (zn[0][i] - z0) : T(0);
            const T g1 = h1 ? wh1 * (zc[0][i + k3ZX] - z0) : T(0);
            const T g2 = h2 ? wh2 * (zc[0][i + 1] - z0) : T(0);
            T vc[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                vc[a] = r[1 + a][j];
                if (GAP) uc[a] = r[(GAP ? 4 : 1) + a][j];
            }
            const T cv0 = wh0 != T(0) ? vc[0] + tau * g0 : T(0);
            const T cv1 = wh1 != T(0) ? vc[1] + tau * g1 : T(0);
            const T cv2 = wh2 != T(0) ? vc[2] + tau * g2 : T(0);
            const T nn = cv0 * cv0 + cv1 * cv1 + cv2 * cv2;
            const T rp = pixel_radius<T, ALPHA>(rad, bnd, AL, (int64_t)o);
            const T sc = nn > rp * rp ? rp * rsqrt_t(nn) : T(1);
            const T un[3] = {cv0 * sc, cv1 * sc, cv2 * sc};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (test) dot_acc += (double)((vc[a] - un[a]) * (un[a] - uc[a]));
                if (do_upd) {
                    VO[a * N + o] = un[a] + beta * (un[a] - uc[a]);
                    UO[a * N + o] = un[a];
                }
            }
            if (GAP) {
                const T zu = zc[GAP ? 1 : 0][i];
                const T gu0 = h0 ? wh0 * (zn[GAP ? 1 : 0][i] - zu) : T(0);
                const T gu1 = h1 ? wh1 * (zc[GAP ? 1 : 0][i + k3ZX] - zu) : T(0);
                const T gu2 = h2 ? wh2 * (zc[GAP ? 1 : 0][i + 1] - zu) : T(0);
                gap_acc += (double)(rp * sqrt_t(gu0 * gu0 + gu1 * gu1 + gu2 * gu2) -
                                    (gu0 * uc[0] + gu1 * uc[1] + gu2 * uc[2]));
            }
        }
    }
    cp_async_wait<0>();
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const unsigned nblk = gridDim.x * gridDim.y;
    const unsigned blk = blockIdx.y * gridDim.x + blockIdx.x;
    const double gsum = GAP ? block_sum(gap_acc, sh) : 0.0;
    const double dsum = test ? block_sum(dot_acc, sh) : 0.0;
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[blk * 2 + 0] = gsum;
        part[blk * 2 + 1] = dsum;
    }
    if (!arrive_last(bf.ticket + b, nblk, &flag)) return;
    const double gap = GAP ? sum_partials(part, nblk, 2, 0, sh) : 0.0;
    const double dot = test ? sum_partials(part, nblk, 2, 1, sh) : 0.0;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2 = st;
    control(s2, im, A.max_iter, GAP, test, gap, dot, pin, bf.live);
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// The 3D step with two voxels per thread (float32, rows of an even number of
// voxels): a block owns a k3VY x k3VX tile of the (axis 1, axis 2) plane, a
// warp a row of it, a lane two adjacent voxels, and marches along axis 0
// like iso3d_kernel. The staged region (the tile and a one-entry halo) comes
// in by 8-byte cp.async pieces (the halo columns by 4-byte ones), z of the
// next slice is formed by each thread at its own two voxels (the forward halo
// row and column by the first 41 threads), so no index is divided and each
// copy and each piece of arithmetic serves two voxels. The per-voxel
// arithmetic is iso3d_kernel's, expression for expression; its sums run in an
// order of their own (per thread over its voxels and slices, then the block),
// fixed by the volume's shape.
// ---------------------------------------------------------------------------
constexpr int k3VX = 64, k3VY = 8;        // tile: 64 voxels of axis 2 (two per lane) by 8 of axis 1 (a warp each)
constexpr int k3VRS = k3VX + 4;           // staged row stride: column c (-1 .. 64) at c + 2, interior 8-byte aligned
constexpr int k3VRows = k3VY + 2;         // staged rows -1 .. 8
constexpr int k3VR = k3VRows * k3VRS;     // staged entries per array and slice
constexpr int k3VZS = k3VX + 2;           // z row stride (columns 0 .. 64)
constexpr int k3VZ = (k3VY + 1) * k3VZS;  // z of a slice: rows 0 .. 8
constexpr int k3VPairs = k3VRows * (k3VX / 2);  // 8-byte staging pieces per array and slice (320)
constexpr int k3VHalo = k3VRows * 2;            // 4-byte halo-column pieces (20)

template <bool GAP>
constexpr size_t iso3d_v2_smem() {
    return (size_t)k3Ring * (GAP ? 7 : 4) * k3VR * sizeof(float) + (size_t)2 * (GAP ? 2 : 1) * k3VZ * sizeof(float);
}

template <bool ALPHA, bool GAP, bool ZIN>
__global__ void __launch_bounds__(k3VX / 2 * k3VY, 4) iso3d_v2_kernel(StepArgs A, IsoCall c, IsoBuffers bf) {
    using T = float;
    constexpr int NA = GAP ? 7 : 4;  // staged arrays: d, v0..v2 (and u0..u2 for the gap)
    constexpr int NT = k3VX / 2 * k3VY;
    extern __shared__ __align__(16) unsigned char i3v_smem[];
    T(*reg)[NA][k3VR] = reinterpret_cast<T(*)[NA][k3VR]>(i3v_smem);
    T(*zs)[GAP ? 2 : 1][k3VZ] = reinterpret_cast<T(*)[GAP ? 2 : 1][k3VZ]>(i3v_smem + k3Ring * NA * k3VR * sizeof(T));
    __shared__ double sh[32];
    __shared__ int flag;
    asm volatile("griddepcontrol.wait;" ::: "memory");  // a programmatic dependent of the previous step
    const int b = step_image(bf, blockIdx.z);
    if (b < 0) return;
    const IsoState st = bf.st[b];
    if (st.status != kLive) return;
    const int it = st.it;
    const bool do_gap = (it > 0 && ((it & 3) == 0 || it == A.max_iter)) || (it == 0 && st.warm);
    const bool zin = st.zero_in != 0;
    if (do_gap != GAP || zin != ZIN) {
        if (threadIdx.x == 0) atomicExch(bf.err, 3);
        return;
    }
    const IsoImage im = bf.img[b];
    const int D0 = (int)A.g.L[0], D1 = (int)A.g.L[1], D2 = (int)A.g.L[2];
    const int64_t N = A.g.N;
    const int64_t S0 = (int64_t)D1 * D2;
    const bool do_upd = it < A.max_iter;
    const bool test = do_upd && (it & 3) == 0;
    const int pin = A.par, pout = A.par ^ 1;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *U = static_cast<const T *>(bf.U[pin]) + (int64_t)b * 3 * N;
    const T *V = st.vsel ? U : static_cast<const T *>(bf.V[pin]) + (int64_t)b * 3 * N;
    T *UO = static_cast<T *>(bf.U[pout]) + (int64_t)b * 3 * N;
    T *VO = static_cast<T *>(bf.V[pout]) + (int64_t)b * 3 * N;
    const T *AL = ALPHA ? static_cast<const T *>(bf.alpha) + (int64_t)b * c.alpha_stride : nullptr;
    const T wh0 = (T)c.wh[0], wh1 = (T)c.wh[1], wh2 = (T)c.wh[2];
    const T tau = (T)c.tau, beta = (T)st.beta, rad = (T)im.radius, bnd = (T)im.bound;
    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int x0 = blockIdx.x * k3VX;
    const int nyt = (D1 + k3VY - 1) / k3VY;
    const int y0 = (blockIdx.y % nyt) * k3VY;
    const int s0 = (blockIdx.y / nyt) * A.rows;
    const int s1 = min(D0, s0 + A.rows);
    auto q3 = [](int sl) { return (sl + k3Ring) % k3Ring; };
    // This thread's staging pieces: 8-byte pieces tid and tid + NT (of 320),
    // a 4-byte halo piece tid (of 20); offsets in a slice, whether in the
    // image, and where they go in a staged array.
    int64_t po[3];
    bool pok[3];
    int pj[3];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int q = tid + e * NT;
        const int r = q / (k3VX / 2), cp = q % (k3VX / 2);  // constant divisors (powers of two)
        const int gy = y0 - 1 + r, gx = x0 + 2 * cp;
        pok[e] = q < k3VPairs && gy >= 0 && gy < D1 && gx < D2;
        po[e] = pok[e] ? (int64_t)gy * D2 + gx : 0;
        pj[e] = r * k3VRS + 2 + 2 * cp;
    }
    {
        const int r = tid >> 1, side = tid & 1;
        const int gy = y0 - 1 + r, gx = side ? x0 + k3VX : x0 - 1;
        pok[2] = tid < k3VHalo && gy >= 0 && gy < D1 && gx >= 0 && gx < D2;
        po[2] = pok[2] ? (int64_t)gy * D2 + gx : 0;
        pj[2] = r * k3VRS + (side ? k3VX + 2 : 1);
    }
    // Slices come into the ring by cp.async (zeros outside the image), issued
    // three steps before the work on them: slice sl + 3 goes into the slot of
    // slice sl - 1 once every thread is past the last step's reads of it.
    auto issue = [&](int sl) {
        if (sl <= s1) {
            T(*r)[k3VR] = reg[q3(sl)];
            const bool sin = sl >= 0 && sl < D0;
            const int64_t so = sin ? (int64_t)sl * S0 : 0;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (tid + e * NT < k3VPairs) {
                    const bool in = pok[e] && sin;
                    const int64_t o = in ? so + po[e] : 0;
                    cp_async_zfill<8>(&r[0][pj[e]], D + o, in ? 8u : 0u);
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        cp_async_zfill<8>(&r[1 + a][pj[e]], V + a * N + o, (in && !ZIN) ? 8u : 0u);
                    if (GAP)
#pragma unroll
                        for (int a = 0; a < 3; ++a)
                            cp_async_zfill<8>(&r[(GAP ? 4 : 1) + a][pj[e]], U + a * N + o, (in && !ZIN) ? 8u : 0u);
                }
            }
            if (tid < k3VHalo) {
                const bool in = pok[2] && sin;
                const int64_t o = in ? so + po[2] : 0;
                cp_async_zfill<4>(&r[0][pj[2]], D + o, in ? 4u : 0u);
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    cp_async_zfill<4>(&r[1 + a][pj[2]], V + a * N + o, (in && !ZIN) ? 4u : 0u);
                if (GAP)
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        cp_async_zfill<4>(&r[(GAP ? 4 : 1) + a][pj[2]], U + a * N + o, (in && !ZIN) ? 4u : 0u);
            }
        }
        cp_async_commit();
    };
    // z of slice sl (of v, and of u for the gap) at entry (row zy, column zx)
    // of the tile and its forward halo: iso3d_kernel's expression
    auto zat = [&](int sl, int zy, int zx) {
        const T(*r)[k3VR] = reg[q3(sl)];
        const T(*rp)[k3VR] = reg[q3(sl - 1)];
        T(*z)[k3VZ] = zs[sl & 1];
        const int i = zy * k3VZS + zx;
        const int j = (zy + 1) * k3VRS + zx + 2;
        z[0][i] = r[0][j] + wh0 * (r[1][j] - rp[1][j]) + wh1 * (r[2][j] - r[2][j - k3VRS]) +
                  wh2 * (r[3][j] - r[3][j - 1]);
        if (GAP)
            z[GAP ? 1 : 0][i] = r[0][j] + wh0 * (r[4][j] - rp[4][j]) + wh1 * (r[5][j] - r[5][j - k3VRS]) +
                                wh2 * (r[6][j] - r[6][j - 1]);
    };
    auto zslice = [&](int sl) {
        zat(sl, w, 2 * l);
        zat(sl, w, 2 * l + 1);
        if (tid < 32) {  // the forward halo row
            zat(sl, k3VY, 2 * tid);
            zat(sl, k3VY, 2 * tid + 1);
        } else if (tid < 32 + k3VY + 1) {  // the forward halo column, rows 0 .. 8
            zat(sl, tid - 32, k3VX);
        }
    };
    const int gy = y0 + w, gx = x0 + 2 * l;
    const bool own = gy < D1 && gx < D2;  // both voxels (D2 even)
    const int64_t ooff = own ? (int64_t)gy * D2 + gx : 0;
    // u at this thread's voxels of a slice (the gap variant stages it)
    float2 pu[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    auto fetch_u = [&](int sl) {
        if (GAP || ZIN || !own || sl >= s1) return;
        const int64_t o = (int64_t)sl * S0 + ooff;
#pragma unroll
        for (int a = 0; a < 3; ++a) pu[a] = *reinterpret_cast<const float2 *>(U + a * N + o);
    };
    double gap_acc = 0.0, dot_acc = 0.0;
#pragma unroll
    for (int q = -1; q <= k3Ring - 2; ++q) issue(s0 + q);
    fetch_u(s0);
    cp_async_wait<k3Ring - 2>();  // slices s0 - 1 and s0 are in
    __syncthreads();
    zslice(s0);
    for (int sl = s0; sl < s1; ++sl) {
        const float2 uc2[3] = {pu[0], pu[1], pu[2]};
        if (sl + 1 < s1) fetch_u(sl + 1);
        cp_async_wait<k3Ring - 3>();  // slice sl + 1 is in (the later ones may still be in flight)
        __syncthreads();
        issue(sl + k3Ring - 1);
        zslice(sl + 1);
        __syncthreads();
        if (own) {
            const T(*r)[k3VR] = reg[q3(sl)];
            const T(*zc)[k3VZ] = zs[sl & 1];
            const T(*zn)[k3VZ] = zs[(sl + 1) & 1];
            const int64_t o = (int64_t)sl * S0 + ooff;
            const bool h0 = sl + 1 < D0, h1 = gy + 1 < D1;
            T vo[2][3], uo[2][3];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int i = w * k3VZS + 2 * l + e, j = (w + 1) * k3VRS + 2 * l + e + 2;
                const bool h2 = gx + e + 1 < D2;
                T uc[3] = {e ? uc2[0].y : uc2[0].x, e ? uc2[1].y : uc2[1].x, e ? uc2[2].y : uc2[2].x};
                const T z0 = zc[0][i];
                const T g0 = h0 ? wh0 * (zn[0][i] - z0) : T(0);
                const T g1 = h1 ? wh1 * (zc[0][i + k3VZS] - z0) : T(0);
                const T g2 = h2 ? wh2 * (zc[0][i + 1] - z0) : T(0);
                T vc[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    vc[a] = r[1 + a][j];
                    if (GAP) uc[a] = r[(GAP ? 4 : 1) + a][j];
                }
                const T cv0 = wh0 != T(0) ? vc[0] + tau * g0 : T(0);
                const T cv1 = wh1 != T(0) ? vc[1] + tau * g1 : T(0);
                const T cv2 = wh2 != T(0) ? vc[2] + tau * g2 : T(0);
                const T nn = cv0 * cv0 + cv1 * cv1 + cv2 * cv2;
                const T rp = pixel_radius<T, ALPHA>(rad, bnd, AL, o + e);
                const T sc = nn > rp * rp ? rp * rsqrt_t(nn) : T(1);
                const T un[3] = {cv0 * sc, cv1 * sc, cv2 * sc};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    if (test) dot_acc += (double)((vc[a] - un[a]) * (un[a] - uc[a]));
                    vo[e][a] = un[a] + beta * (un[a] - uc[a]);
                    uo[e][a] = un[a];
                }
                if (GAP) {
                    const T zu = zc[GAP ? 1 : 0][i];
                    const T gu0 = h0 ? wh0 * (zn[GAP ? 1 : 0][i] - zu) : T(0);
                    const T gu1 = h1 ? wh1 * (zc[GAP ? 1 : 0][i + k3VZS] - zu) : T(0);
                    const T gu2 = h2 ? wh2 * (zc[GAP ? 1 : 0][i + 1] - zu) : T(0);
                    gap_acc += (double)(rp * sqrt_t(gu0 * gu0 + gu1 * gu1 + gu2 * gu2) -
                                        (gu0 * uc[0] + gu1 * uc[1] + gu2 * uc[2]));
                }
            }
            if (do_upd)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    *reinterpret_cast<float2 *>(VO + a * N + o) = make_float2(vo[0][a], vo[1][a]);
                    *reinterpret_cast<float2 *>(UO + a * N + o) = make_float2(uo[0][a], uo[1][a]);
                }
        }
    }
    cp_async_wait<0>();
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const unsigned nblk = gridDim.x * gridDim.y;
    const unsigned blk = blockIdx.y * gridDim.x + blockIdx.x;
    const double gsum = GAP ? block_sum(gap_acc, sh) : 0.0;
    const double dsum = test ? block_sum(dot_acc, sh) : 0.0;
    double *part = bf.part + (int64_t)b * bf.max_part * 2;
    if (threadIdx.x == 0) {
        part[blk * 2 + 0] = gsum;
        part[blk * 2 + 1] = dsum;
    }
    if (!arrive_last(bf.ticket + b, nblk, &flag)) return;
    const double gap = GAP ? sum_partials(part, nblk, 2, 0, sh) : 0.0;
    const double dot = test ? sum_partials(part, nblk, 2, 1, sh) : 0.0;
    if (threadIdx.x != 0) return;
    bf.ticket[b] = 0;
    IsoState s2 = st;
    control(s2, im, A.max_iter, GAP, test, gap, dot, pin, bf.live);
    bf.st[b] = s2;
}

// ---------------------------------------------------------------------------
// Finalisation: z = d - G^T u (tv_iso.cpp:484-487, 539) back at the input's
// scale (tv_iso.cpp:403-413), the dual q = u / wmax 2^e into bf.dual.
// ---------------------------------------------------------------------------

template <class T>
__global__ void finalize_kernel(Geometry g, IsoCall c, IsoBuffers bf, T *__restrict__ out) {
    const int b = blockIdx.y;
    const IsoImage im = bf.img[b];
    if (im.mode == kModeTv1d || im.mode == kModeInf) return;
    const IsoState st = bf.st[b];
    const int64_t N = g.N, B = g.B;
    const int K = g.k;
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    const T *U = static_cast<const T *>(bf.U[st.fin_par]) + (int64_t)b * K * N;
    T *Q = static_cast<T *>(bf.dual);
    T *O = out + (int64_t)b * N;
    int64_t S[3], L[3];
    for (int a = 0; a < K; ++a) L[a] = g.L[a];
    S[K - 1] = 1;
    for (int a = K - 2; a >= 0; --a) S[a] = S[a + 1] * L[a + 1];
    const T inv = (T)(1.0 / c.wmax);
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
        if (im.mode == kModeNan) {
            O[p] = (T)CUDART_NAN;
            for (int a = 0; a < K; ++a) Q[((int64_t)a * B + b) * N + p] = (T)CUDART_NAN;
            continue;
        }
        if (im.mode == kModeIdentity) {
            O[p] = D[p];
            for (int a = 0; a < K; ++a) Q[((int64_t)a * B + b) * N + p] = T(0);
            continue;
        }
        T z = D[p];
        for (int a = 0; a < K; ++a) {
            const T wa = (T)c.wh[a];
            if (wa == T(0)) continue;
            const bool first = ((p / S[a]) % L[a]) == 0;
            z += wa * (U[a * N + p] - (first ? T(0) : U[a * N + p - S[a]]));
        }
        O[p] = im.e ? ldexp_t(z, im.e) : z;
        for (int a = 0; a < K; ++a) {
            T q = U[a * N + p] * inv;
            if (im.e) q = ldexp_t(q, im.e);
            Q[((int64_t)a * B + b) * N + p] = q;
        }
    }
}

// ---------------------------------------------------------------------------
// One active axis without pixel weights: exact 1D TV along it (tv_iso.cpp:381-398)
// ---------------------------------------------------------------------------
}  // namespace

}  // namespace fpb

#include "tv1d.cuh"

namespace fpb {
namespace {

template <class T>
__global__ void iso_tv1d_kernel(Geometry g, IsoCall c, IsoBuffers bf, T *__restrict__ out) {
    const int b = blockIdx.y;
    const IsoImage im = bf.img[b];
    if (im.mode != kModeTv1d) return;
    const int a = c.act_axis;
    const int64_t N = g.N, B = g.B;
    const int K = g.k;
    int64_t S[3];
    S[K - 1] = 1;
    for (int x = K - 2; x >= 0; --x) S[x] = S[x + 1] * g.L[x + 1];
    const int64_t L = g.L[a], s = S[a];
    const int64_t nfib = N / L;
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfib) return;
    const int64_t base = (f / s) * L * s + (f % s);
    const T *D = static_cast<const T *>(bf.d) + (int64_t)b * N;
    T *Z = static_cast<T *>(bf.U[0]) + (int64_t)b * K * N;  // solved-scale z, scratch
    T *O = out + (int64_t)b * N;
    T *Q = static_cast<T *>(bf.dual);
    const double lam = ldexp(im.gamma_in, -im.e) * c.w_act;
    const T *Db = D + base;
    T *Zb = Z + base;
    auto fin = [Db, s](int64_t i) -> double { return (double)Db[i * s]; };
    auto fout = [Zb, s](int64_t i, double v) { Zb[i * s] = (T)v; };
    tv1d_fiber<double>(fin, fout, L, lam, false, NoWeight{}, DivRecip<double>{});
    double cs = 0.0;
    for (int64_t i = 0; i < L; ++i) {
        const int64_t o = base + i * s;
        const T z = Z[o];
        cs += (double)D[o] - (double)z;
        O[o] = im.e ? ldexp_t(z, im.e) : z;
        for (int x = 0; x < K; ++x) {
            double q = 0.0;
            if (x == a && i + 1 < L) q = -cs / c.w_act;
            if (im.e) q = ldexp(q, im.e);
            Q[((int64_t)x * B + b) * N + o] = (T)q;
        }
    }
}

template <class T>
__global__ void conj_kernel(const T *__restrict__ y, T *__restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = y[i] - out[i];
}

// x = d 2^e per image (the staged input back at its own scale)
template <class T>
__global__ void unscale_kernel(const T *__restrict__ d, const int *__restrict__ e, int64_t N, int64_t B,
                               T *__restrict__ x) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B * N; i += (int64_t)gridDim.x * blockDim.x) {
        const int ex = e[i / N];
        x[i] = ex ? ldexp_t(d[i], ex) : d[i];
    }
}

__global__ void fill_double_kernel(double *dst, double v, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = v;
}

struct StridedDesc {
    int ndim;
    int64_t shape[FP_MAX_NDIM_DEV];
    int64_t ss[FP_MAX_NDIM_DEV];
    int64_t ds[FP_MAX_NDIM_DEV];
};

template <class S, class D>
__global__ void strided_kernel(const S *__restrict__ src, D *__restrict__ dst, StridedDesc sd, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = i, so = 0, doff = 0;
        for (int d = sd.ndim - 1; d >= 0; --d) {
            const int64_t ext = sd.shape[d];
            const int64_t c = r % ext;
            r /= ext;
            so += c * sd.ss[d];
            doff += c * sd.ds[d];
        }
        dst[doff] = (D)src[so];
    }
}

int grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    return (int)g;
}

template <class T>
cudaError_t setup_t(const Geometry &g, const IsoCall &c, const IsoBuffers &bf, const void *x, int warm, int par,
                    cudaStream_t s) {
    const int nb = iso_setup_blocks(g);
    const dim3 grid(nb, (unsigned)g.B);
    scan1_kernel<T><<<grid, kScanThreads, 0, s>>>(static_cast<const T *>(x), static_cast<T *>(bf.d), g, c, bf);
    scan2_kernel<T><<<grid, kScanThreads, 0, s>>>(static_cast<T *>(bf.d), g, c, bf);
    scan3_kernel<T><<<grid, kScanThreads, 0, s>>>(static_cast<const T *>(bf.d), g, c, bf, warm);
    if (warm) {
        const dim3 wg((unsigned)std::min<int64_t>((g.N + 255) / 256, 4096), (unsigned)g.B);
        if (c.has_alpha) warm_kernel<T, true><<<wg, 256, 0, s>>>(g, c, bf, par);
        else warm_kernel<T, false><<<wg, 256, 0, s>>>(g, c, bf, par);
    }
    if (c.huber) huber_momentum<<<(unsigned)((g.B + 127) / 128), 128, 0, s>>>(c, bf, g.B);
    return cudaGetLastError();
}

// Launches a step so that it may start while the previous kernel on the
// stream finishes (programmatic dependent launch): its blocks are scheduled
// once every block of the previous step has finished its pass over the
// iterates (griddepcontrol.launch_dependents), and wait
// (griddepcontrol.wait) for that step to complete before reading anything.
// FASTPROX_B200_PDL=0 launches plainly (for comparison).
template <class K>
void launch_step(K kernel, dim3 grid, unsigned bx, size_t smem, cudaStream_t s, const StepArgs &A, const IsoCall &c,
                 const IsoBuffers &bf) {
    static const bool pdl = [] {
        const char *v = std::getenv("FASTPROX_B200_PDL");
        return !(v && v[0] == '0' && v[1] == 0);
    }();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(bx);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, A, c, bf);
}

template <class T, int VEC, bool ALPHA>
void launch_lean_a(const StepShape &sh, StepArgs A, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s,
                   int variant) {
    const dim3 grid(sh.gx, sh.gy, (unsigned)A.nimg);
    if (variant == 1) launch_step(iso2d_lean_kernel<T, VEC, ALPHA, false, true>, grid, sh.bx, 0, s, A, c, bf);
    else if (variant == 2) launch_step(iso2d_lean_kernel<T, VEC, ALPHA, true, false>, grid, sh.bx, 0, s, A, c, bf);
    else launch_step(iso2d_lean_kernel<T, VEC, ALPHA, false, false>, grid, sh.bx, 0, s, A, c, bf);
}

// Two iterations per launch: blocks of whole rows (the first iteration's
// halo is 4 rows) with the lean step's threads per block (the same warps, so
// the same per-row sums).
// The pair kernels' ring passes 48 KB in float64: their attribute, once per device.
template <class T, bool ALPHA, bool GAP2, bool WIDE>
void launch_pair_k(dim3 grid, unsigned bx, cudaStream_t s, const StepArgs &A, const IsoCall &c,
                   const IsoBuffers &bf) {
    static std::atomic<unsigned long long> done{0};  // the attribute is per function and device
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64 && !(done.load() & (1ull << dev))) {
        cudaFuncSetAttribute(iso2d_pair_kernel<T, ALPHA, GAP2, WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)pair_ring_bytes<T, ALPHA, WIDE>());
        done.fetch_or(1ull << dev);
    }
    launch_step(iso2d_pair_kernel<T, ALPHA, GAP2, WIDE>, grid, bx, pair_ring_bytes<T, ALPHA, WIDE>(), s, A, c, bf);
}

template <class T, bool WIDE>
void launch_pair_w(dim3 grid, unsigned bx, cudaStream_t s, const StepArgs &A, const IsoCall &c, const IsoBuffers &bf,
                   bool gap) {
    if (gap) {
        if (c.has_alpha) launch_pair_k<T, true, true, WIDE>(grid, bx, s, A, c, bf);
        else launch_pair_k<T, false, true, WIDE>(grid, bx, s, A, c, bf);
    } else {
        if (c.has_alpha) launch_pair_k<T, true, false, WIDE>(grid, bx, s, A, c, bf);
        else launch_pair_k<T, false, false, WIDE>(grid, bx, s, A, c, bf);
    }
}

template <class T>
void launch_pair(const StepShape &sh, StepArgs A, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s, bool gap) {
    static const int rows_hint = [] {  // tuning hint FASTPROX_B200_PAIR_ROWS
        const char *v = std::getenv("FASTPROX_B200_PAIR_ROWS");
        const int r = v ? std::atoi(v) : 0;
        return (r >= 8 && r <= kLeanRowsMax) ? r : 0;
    }();
    const int64_t H = A.g.L[0];
    // 12 rows per block: on 64 x 512^2 836 images/s, against 815 at 8 and 822 at 16
    // (shorter blocks spread better, longer ones recompute less of the halo);
    // fewer, down to 4, while the launch has too few blocks to spread (the
    // tail of a batch, a few images live)
    int rows = rows_hint ? rows_hint : 12;
    while (!rows_hint && rows > 4 && A.nimg * sh.gx * ((H + rows - 1) / rows) < tail_blocks())
        rows = rows / 2 > 4 ? rows / 2 : 4;
    A.rows = rows;
    const dim3 grid((unsigned)sh.gx, (unsigned)((H + rows - 1) / rows), (unsigned)A.nimg);
    // rows wider than a block: the kernel with the halo columns of the first iteration
    if (sh.gx > 1) launch_pair_w<T, true>(grid, (unsigned)sh.bx, s, A, c, bf, gap);
    else launch_pair_w<T, false>(grid, (unsigned)sh.bx, s, A, c, bf, gap);
}

template <class T, int VEC>
void launch_lean(const StepShape &sh, StepArgs A, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s,
                 int variant) {
    if (c.has_alpha) launch_lean_a<T, VEC, true>(sh, A, c, bf, s, variant);
    else launch_lean_a<T, VEC, false>(sh, A, c, bf, s, variant);
}

// Dynamic shared memory of the 3D step: k3Ring staged slices and two of z.
template <class T, bool GAP>
constexpr size_t iso3d_smem() {
    return (size_t)k3Ring * (GAP ? 7 : 4) * k3R * sizeof(T) + (size_t)2 * (GAP ? 2 : 1) * k3Z * sizeof(T);
}

// The attribute is per function and device: set once, to the kernel's size.
template <class T, bool ALPHA, bool GAP, bool ZIN>
void iso3d_attr() {
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    const unsigned long long bit = 1ull << dev;
    if (done.load() & bit) return;
    cudaFuncSetAttribute(iso3d_kernel<T, ALPHA, GAP, ZIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)iso3d_smem<T, GAP>());
    done.fetch_or(bit);
}

template <class T, bool ALPHA, bool GAP, bool ZIN>
void launch_3d_v(const dim3 &grid, StepArgs A, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s) {
    iso3d_attr<T, ALPHA, GAP, ZIN>();
    launch_step(iso3d_kernel<T, ALPHA, GAP, ZIN>, grid, k3TX * k3TY, iso3d_smem<T, GAP>(), s, A, c, bf);
}

template <bool ALPHA, bool GAP, bool ZIN>
void launch_3d_v2(const dim3 &grid, StepArgs A, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s) {
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64 && !(done.load() & (1ull << dev))) {
        cudaFuncSetAttribute(iso3d_v2_kernel<ALPHA, GAP, ZIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)iso3d_v2_smem<GAP>());
        done.fetch_or(1ull << dev);
    }
    launch_step(iso3d_v2_kernel<ALPHA, GAP, ZIN>, grid, k3VX / 2 * k3VY, iso3d_v2_smem<GAP>(), s, A, c, bf);
}

template <class T, bool ALPHA>
void launch_3d_a(const StepShape &sh, StepArgs A, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s, int variant) {
    const dim3 grid(sh.gx, sh.gy, (unsigned)A.nimg);
    if constexpr (std::is_same<T, float>::value) {
        if (sh.vec == 2) {  // two voxels per thread (iso_pick_shape)
            if (variant == 1) launch_3d_v2<ALPHA, false, true>(grid, A, c, bf, s);
            else if (variant == 2) launch_3d_v2<ALPHA, true, false>(grid, A, c, bf, s);
            else launch_3d_v2<ALPHA, false, false>(grid, A, c, bf, s);
            return;
        }
    }
    if (variant == 1) launch_3d_v<T, ALPHA, false, true>(grid, A, c, bf, s);
    else if (variant == 2) launch_3d_v<T, ALPHA, true, false>(grid, A, c, bf, s);
    else launch_3d_v<T, ALPHA, false, false>(grid, A, c, bf, s);
}

// The quad launch: blocks of kQuadWarps tiles (a strip by `rows` rows). A
// tile's march takes rows + 8 steps and the SMs hold a fixed number of
// blocks at once, so the rows are chosen (8 to 64, in steps of 4) for the
// fewest waves of resident blocks times steps per tile: 48 on 64 images of
// 512^2 (three waves of 56 steps, against five of 40 at 32 rows), 8 for one
// image (a single wave of short tiles).
void launch_quad(StepArgs A, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s) {
    static const int rows_hint = [] {  // tuning hint FASTPROX_B200_QUAD_ROWS
        const char *v = std::getenv("FASTPROX_B200_QUAD_ROWS");
        const int r = v ? std::atoi(v) : 0;
        return (r >= 4 && r <= 256) ? r : 0;
    }();
    static const int64_t slots = [] {  // resident quad blocks on the device
        int dev = 0, sms = 148, per = 4;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, iso2d_quad_kernel<true, false>, 32 * kQuadWarps,
                                                          kQuadSmem) != cudaSuccess || per < 1)
            per = 4;
        cudaGetLastError();
        return (int64_t)sms * per;
    }();
    const int64_t H = A.g.L[0], ns = quad_strips((int)A.g.L[1]);
    auto blocks = [&](int rows) { return (ns * ((H + rows - 1) / rows) + kQuadWarps - 1) / kQuadWarps; };
    int rows = rows_hint;
    if (!rows) {
        double best = 0.0;
        for (int r = 8; r <= 64; r += 4) {
            const int64_t waves = (A.nimg * blocks(r) + slots - 1) / slots;
            const double cost = (double)waves * (double)(std::min<int64_t>(r, H) + 8);
            if (!rows || cost < best) {
                rows = r;
                best = cost;
            }
        }
    }
    A.rows = rows;
    const dim3 grid((unsigned)blocks(rows), 1, (unsigned)A.nimg);
    if (c.has_alpha) launch_step(iso2d_quad_kernel<true, false>, grid, 32 * kQuadWarps, kQuadSmem, s, A, c, bf);
    else launch_step(iso2d_quad_kernel<false, false>, grid, 32 * kQuadWarps, kQuadSmem, s, A, c, bf);
}

template <class T>
cudaError_t step_t(const Geometry &g, const IsoCall &c, const IsoBuffers &bf, const StepShape &sh, int par,
                   int variant, int64_t nimg, cudaStream_t s) {
    StepArgs A;
    A.g = g;
    A.max_iter = c.max_iter;
    A.par = par;
    A.rows = sh.rows;
    A.nimg = nimg;
    A.row_part = 0;
    if (nimg <= 0) return cudaSuccess;
    if (c.huber) {  // Huber-smoothed TV: its own step, one thread per pixel
        const dim3 grid(sh.gx, (unsigned)nimg);
        const bool sw = c.has_alpha != 0;
        if (g.k == 2) {
            if (c.huber == 2) {
                if (sw) huber_kernel<T, 2, true, true><<<grid, sh.bx, 0, s>>>(A, c, bf);
                else huber_kernel<T, 2, false, true><<<grid, sh.bx, 0, s>>>(A, c, bf);
            } else {
                if (sw) huber_kernel<T, 2, true, false><<<grid, sh.bx, 0, s>>>(A, c, bf);
                else huber_kernel<T, 2, false, false><<<grid, sh.bx, 0, s>>>(A, c, bf);
            }
        } else {
            if (c.huber == 2) {
                if (sw) huber_kernel<T, 3, true, true><<<grid, sh.bx, 0, s>>>(A, c, bf);
                else huber_kernel<T, 3, false, true><<<grid, sh.bx, 0, s>>>(A, c, bf);
            } else {
                if (sw) huber_kernel<T, 3, true, false><<<grid, sh.bx, 0, s>>>(A, c, bf);
                else huber_kernel<T, 3, false, false><<<grid, sh.bx, 0, s>>>(A, c, bf);
            }
        }
        return cudaGetLastError();
    }
    if (variant == kVariantQuad) {
        if constexpr (std::is_same<T, float>::value) {
            launch_quad(A, c, bf, s);
            return cudaGetLastError();
        }
        return cudaErrorInvalidValue;
    }
    if (variant == kVariantPair || variant == kVariantPairGap) {
        launch_pair<T>(sh, A, c, bf, s, variant == kVariantPairGap);
        return cudaGetLastError();
    }
    StepShape sh2 = sh;
    if (sh.kind == 4 && (int64_t)sh.gx * g.L[0] <= bf.max_part && sh.rows <= kLeanRowsMax) {
        // per-row partial sums make the sums independent of the rows per
        // block, so a launch over few live images (the tail of a batch) takes
        // shorter blocks, more of them, to spread over the SMs
        A.row_part = 1;
        const int64_t H = g.L[0];
        int rows = sh.rows;
        while (rows > 2 && nimg * sh.gx * ((H + rows - 1) / rows) < tail_blocks()) rows /= 2;
        sh2.rows = rows;
        sh2.gy = (int)((H + rows - 1) / rows);
        A.rows = rows;
    }
    if (sh.kind == 5) {
        if (c.has_alpha) launch_3d_a<T, true>(sh, A, c, bf, s, variant);
        else launch_3d_a<T, false>(sh, A, c, bf, s, variant);
    } else if (sh.kind == 4) {
        if (sh.vec == 4) launch_lean<T, 4>(sh2, A, c, bf, s, variant);
        else if (sh.vec == 2) launch_lean<T, 2>(sh2, A, c, bf, s, variant);
        else launch_lean<T, 1>(sh2, A, c, bf, s, variant);
    } else {
        const dim3 grid(sh.gx, (unsigned)nimg);
        if (g.k == 2) {
            if (c.has_alpha) iso_generic_kernel<T, 2, true><<<grid, sh.bx, 0, s>>>(A, c, bf);
            else iso_generic_kernel<T, 2, false><<<grid, sh.bx, 0, s>>>(A, c, bf);
        } else {
            if (c.has_alpha) iso_generic_kernel<T, 3, true><<<grid, sh.bx, 0, s>>>(A, c, bf);
            else iso_generic_kernel<T, 3, false><<<grid, sh.bx, 0, s>>>(A, c, bf);
        }
    }
    return cudaGetLastError();
}

template <class T>
cudaError_t finalize_t(const Geometry &g, const IsoCall &c, const IsoBuffers &bf, void *out, cudaStream_t s) {
    const dim3 grid((unsigned)std::min<int64_t>((g.N + 255) / 256, 2048), (unsigned)g.B);
    finalize_kernel<T><<<grid, 256, 0, s>>>(g, c, bf, static_cast<T *>(out));
    if (c.na == 1 && !c.has_alpha) {
        const int64_t nfib = g.N / g.L[c.act_axis];
        const dim3 g1((unsigned)((nfib + 127) / 128), (unsigned)g.B);
        iso_tv1d_kernel<T><<<g1, 128, 0, s>>>(g, c, bf, static_cast<T *>(out));
    }
    return cudaGetLastError();
}

template <bool GAP2>
void launch_ragged_pair(const RagItem *items, const int *n_items, int grid, const RagSlot *slots,
                        const IsoBuffers &bf, cudaStream_t s) {
    constexpr size_t smem = pair_ring_bytes<float, false, true>();
    static std::atomic<unsigned long long> done{0};  // the attribute is per function and device
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64 && !(done.load() & (1ull << dev))) {
        cudaFuncSetAttribute(iso2d_ragged_pair_kernel<float, GAP2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        done.fetch_or(1ull << dev);
    }
    iso2d_ragged_pair_kernel<float, GAP2><<<grid, 128, smem, s>>>(items, n_items, slots, bf);
}

template <class T, int VEC>
void launch_ragged_t(const RagItem *items, const int *n_items, int grid, const RagSlot *slots, const IsoCall &c,
                     const IsoBuffers &bf, cudaStream_t s, bool pairs) {
    iso2d_ragged_kernel<T, VEC><<<grid, 128, 0, s>>>(items, n_items, slots, bf, pairs);
    if constexpr (std::is_same<T, float>::value && VEC == 4) {
        if (pairs) {
            launch_ragged_pair<false>(items, n_items, grid, slots, bf, s);
            launch_ragged_pair<true>(items, n_items, grid, slots, bf, s);
        }
    }
}

}  // namespace

cudaError_t iso_ragged_step(int dtype, int vec, const RagItem *items, const int *n_items, int grid,
                            const RagSlot *slots, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s) {
    if (grid <= 0) return cudaSuccess;
    if (dtype == 1) {
        const bool pairs = iso_ragged_pairs(dtype, vec);
        if (vec == 4) launch_ragged_t<float, 4>(items, n_items, grid, slots, c, bf, s, pairs);
        else launch_ragged_t<float, 1>(items, n_items, grid, slots, c, bf, s, false);
    } else {
        if (vec == 2) launch_ragged_t<double, 2>(items, n_items, grid, slots, c, bf, s, false);
        else launch_ragged_t<double, 1>(items, n_items, grid, slots, c, bf, s, false);
    }
    return cudaGetLastError();
}

bool iso_ragged_pairs(int dtype, int vec) {
    return pairs_enabled() && dtype == 1 && vec == 4;
}

cudaError_t iso_ragged_quad_step(const RagItem *items, const int *n_items, int grid, const RagSlot *slots,
                                 const IsoBuffers &bf, cudaStream_t s) {
    if (grid <= 0) return cudaSuccess;
    iso2d_ragged_quad_kernel<<<grid, 32 * kQuadWarps, kQuadSmem, s>>>(items, n_items, slots, bf);
    return cudaGetLastError();
}

int iso_quad_strips(int W) { return quad_strips(W); }
int iso_quad_warps() { return kQuadWarps; }

int iso_setup_blocks(const Geometry &g) {
    int64_t nb = (g.N + kScanThreads * 8 - 1) / (kScanThreads * 8);
    if (nb > 128) nb = 128;
    if (nb < 1) nb = 1;
    return (int)nb;
}

bool iso3d_v2_enabled() {
    static const bool on = [] {
        const char *v = std::getenv("FASTPROX_B200_3D_V2");
        return !(v && v[0] == '0' && v[1] == 0);
    }();
    return on;
}

StepShape iso_pick_shape(int dtype, const Geometry &g, int rows_hint, int bx_hint, int kind_hint) {
    StepShape sh;
    const int64_t W = g.k == 2 ? g.L[1] : 0;
    const int vmax = dtype == 1 ? 4 : 2;
    if (g.k == 2 && W >= 32 && kind_hint != 1) {
        sh.kind = 4;
        sh.vec = (W % vmax == 0) ? vmax : ((W % 2 == 0) ? 2 : 1);
        const int64_t cols = (W + sh.vec - 1) / sh.vec;
        int bx = bx_hint > 0 ? bx_hint : (int)std::min<int64_t>(128, ((cols + 31) / 32) * 32);
        sh.bx = bx;
        sh.gx = (int)((cols + bx - 1) / bx);
        const int64_t H = g.L[0];
        // The block partition of an image depends on its shape only, so an
        // image gives the same bits alone and in any batch.
        int rows = rows_hint;
        if (rows <= 0) rows = (int)std::max<int64_t>(4, std::min<int64_t>(16, H / 32));
        sh.rows = rows;
        sh.gy = (int)((H + rows - 1) / rows);
    } else if (g.k == 3 && kind_hint != 1 && g.L[0] * g.L[1] * g.L[2] < 2147483647LL) {
        // 3D: tiles of the (axis 1, axis 2) plane marching through chunks of
        // slices; chunks short enough for a few blocks per SM, at most 4096
        // blocks per image (the partial sums)
        sh.kind = 5;
        // float32 volumes with rows of an even number of voxels: two voxels per
        // thread (iso3d_v2_kernel; tuning hint FASTPROX_B200_3D_V2=0: one)
        sh.vec = (dtype == 1 && g.L[2] % 2 == 0 && iso3d_v2_enabled()) ? 2 : 1;
        const int tx = sh.vec == 2 ? k3VX : k3TX, ty = sh.vec == 2 ? k3VY : k3TY;
        sh.bx = sh.vec == 2 ? k3VX / 2 * k3VY : k3TX * k3TY;
        const int64_t xt = (g.L[2] + tx - 1) / tx, yt = (g.L[1] + ty - 1) / ty;
        // 16 slices per block (62.4 volumes/s on 8 x 128^3 against 59.8 at 8,
        // 62.0 at 32), fewer while a launch would have too few blocks to
        // spread over the SMs (small volumes)
        int64_t rows = rows_hint > 0 ? rows_hint : 16;
        while (rows_hint <= 0 && rows > 4 && xt * yt * ((g.L[0] + rows - 1) / rows) * g.B < tail_blocks()) rows /= 2;
        while (xt * yt * ((g.L[0] + rows - 1) / rows) > 4096) rows *= 2;
        sh.rows = (int)rows;
        sh.gx = (int)xt;
        sh.gy = (int)(yt * ((g.L[0] + rows - 1) / rows));
    } else {
        sh.kind = 1;
        sh.vec = 1;
        sh.bx = bx_hint > 0 ? bx_hint : 256;
        int64_t gx = (g.N + sh.bx - 1) / sh.bx;
        if (gx > 1024) gx = 1024;  // shape-only, as above
        sh.gx = (int)std::max<int64_t>(1, gx);
        sh.gy = 1;
    }
    return sh;
}

cudaError_t iso_setup(int dtype, const Geometry &g, const IsoCall &c, const IsoBuffers &bf, const void *x, int warm,
                      int par, cudaStream_t s) {
    return dtype == 1 ? setup_t<float>(g, c, bf, x, warm, par, s) : setup_t<double>(g, c, bf, x, warm, par, s);
}

cudaError_t iso_step(int dtype, const Geometry &g, const IsoCall &c, const IsoBuffers &bf, const StepShape &sh,
                     int par, int variant, int64_t nimg, cudaStream_t s) {
    return dtype == 1 ? step_t<float>(g, c, bf, sh, par, variant, nimg, s)
                      : step_t<double>(g, c, bf, sh, par, variant, nimg, s);
}

bool pairs_enabled() {
    static const bool on = [] {  // tuning hint FASTPROX_B200_PAIRS=0: single steps only
        const char *v = std::getenv("FASTPROX_B200_PAIRS");
        return !(v && v[0] == '0' && v[1] == 0);
    }();
    return on;
}

bool iso_pair_ok(const Geometry &g, const StepShape &sh, int max_part) {
    // one block per row up to 512 columns (the lean step's threads), else blocks of 512 columns
    return pairs_enabled() && g.k == 2 && sh.kind == 4 && sh.vec == 4 && (sh.gx == 1 ? g.L[1] <= kPairCols : sh.bx == 128) &&
           g.L[0] >= 2 && g.L[0] * sh.gx <= max_part;
}

cudaError_t iso_live_list(const IsoState *st, int64_t B, int *lmap, int *lcnt, cudaStream_t s) {
    live_list_kernel<<<1, 1024, 0, s>>>(st, B, lmap, lcnt);
    return cudaGetLastError();
}

bool iso_quad_ok(int dtype, const Geometry &g, int max_part) {
    static const bool on = [] {  // tuning hint FASTPROX_B200_QUADS=0: no quad launches
        const char *v = std::getenv("FASTPROX_B200_QUADS");
        return !(v && v[0] == '0' && v[1] == 0);
    }();
    // rows narrower than 32 pixels keep the generic step (its gap terms in FP64)
    return on && pairs_enabled() && dtype == 1 && g.k == 2 && g.L[1] >= 32 && g.L[1] % 4 == 0 && g.L[0] >= 2 &&
           g.L[0] * g.L[1] < (int64_t(1) << 31) && iso_quad_parts(g) <= max_part;
}

int64_t iso_quad_parts(const Geometry &g) {
    return g.k == 2 ? g.L[0] * (int64_t)quad_strips((int)std::min<int64_t>(g.L[1], 1 << 30)) : 0;
}

cudaError_t iso_redo(int dtype, const Geometry &g, const IsoCall &c, const IsoBuffers &bf, cudaStream_t s,
                     bool quads) {
    if (g.k != 2 || g.B <= 0 || g.N <= 0) return cudaSuccess;
    if (quads && dtype == 1) {
        // the quad's redo: three iterations over whole images, blocks of 32 rows
        StepArgs A;
        A.g = g;
        A.max_iter = c.max_iter;
        A.par = 0;
        A.rows = 32;
        A.nimg = g.B;
        A.row_part = 0;
        const int64_t tiles = quad_strips((int)g.L[1]) * ((g.L[0] + A.rows - 1) / A.rows);
        const dim3 grid((unsigned)((tiles + kQuadWarps - 1) / kQuadWarps), 1, (unsigned)g.B);
        if (c.has_alpha) iso2d_quad_kernel<true, true><<<grid, 32 * kQuadWarps, kQuadSmem, s>>>(A, c, bf);
        else iso2d_quad_kernel<false, true><<<grid, 32 * kQuadWarps, kQuadSmem, s>>>(A, c, bf);
    }
    const dim3 grid((unsigned)std::min<int64_t>((g.N + 255) / 256, 1024), (unsigned)g.B);
    if (dtype == 1) {
        if (c.has_alpha) iso2d_redo_kernel<float, true><<<grid, 256, 0, s>>>(g, c, bf);
        else iso2d_redo_kernel<float, false><<<grid, 256, 0, s>>>(g, c, bf);
    } else {
        if (c.has_alpha) iso2d_redo_kernel<double, true><<<grid, 256, 0, s>>>(g, c, bf);
        else iso2d_redo_kernel<double, false><<<grid, 256, 0, s>>>(g, c, bf);
    }
    iso2d_redo_state<<<(unsigned)((g.B + 127) / 128), 128, 0, s>>>(bf.st, g.B);
    return cudaGetLastError();
}

cudaError_t iso_finalize(int dtype, const Geometry &g, const IsoCall &c, const IsoBuffers &bf, void *out,
                         cudaStream_t s) {
    return dtype == 1 ? finalize_t<float>(g, c, bf, out, s) : finalize_t<double>(g, c, bf, out, s);
}

cudaError_t fill_double(double *dst, double v, int64_t n, cudaStream_t s) {
    fill_double_kernel<<<grid_for(n, 256), 256, 0, s>>>(dst, v, n);
    return cudaGetLastError();
}

cudaError_t unscale_images(int dtype, const void *d, const int *e, int64_t N, int64_t B, void *x, cudaStream_t s) {
    if (N * B == 0) return cudaSuccess;
    if (dtype == 1)
        unscale_kernel<float><<<grid_for(N * B, 256), 256, 0, s>>>(static_cast<const float *>(d), e, N, B,
                                                                   static_cast<float *>(x));
    else
        unscale_kernel<double><<<grid_for(N * B, 256), 256, 0, s>>>(static_cast<const double *>(d), e, N, B,
                                                                    static_cast<double *>(x));
    return cudaGetLastError();
}

cudaError_t conj_finish(int dtype, const void *y, void *out, int64_t n, cudaStream_t s) {
    if (dtype == 1)
        conj_kernel<float><<<grid_for(n, 256), 256, 0, s>>>(static_cast<const float *>(y), static_cast<float *>(out), n);
    else
        conj_kernel<double>
            <<<grid_for(n, 256), 256, 0, s>>>(static_cast<const double *>(y), static_cast<double *>(out), n);
    return cudaGetLastError();
}

cudaError_t strided_copy(const void *src, int src_dtype, const int64_t *shape, const int64_t *src_strides, int ndim,
                         void *dst, int dst_dtype, const int64_t *dst_strides, cudaStream_t s) {
    if (ndim > FP_MAX_NDIM_DEV) return cudaErrorInvalidValue;
    StridedDesc sd;
    sd.ndim = ndim;
    int64_t n = 1;
    for (int d = 0; d < ndim; ++d) {
        sd.shape[d] = shape[d];
        sd.ss[d] = src_strides[d];
        sd.ds[d] = dst_strides[d];
        n *= shape[d];
    }
    if (n == 0) return cudaSuccess;
    const int grid = grid_for(n, 256);
    if (src_dtype == 1 && dst_dtype == 1)
        strided_kernel<float, float><<<grid, 256, 0, s>>>(static_cast<const float *>(src), static_cast<float *>(dst), sd, n);
    else if (src_dtype == 1)
        strided_kernel<float, double><<<grid, 256, 0, s>>>(static_cast<const float *>(src), static_cast<double *>(dst), sd, n);
    else if (dst_dtype == 1)
        strided_kernel<double, float><<<grid, 256, 0, s>>>(static_cast<const double *>(src), static_cast<float *>(dst), sd, n);
    else
        strided_kernel<double, double>
            <<<grid, 256, 0, s>>>(static_cast<const double *>(src), static_cast<double *>(dst), sd, n);
    return cudaGetLastError();
}

}  // namespace fpb

// ---------------------------------------------------------------------------
// fp_b200_tv_iso_noalloc: the isotropic solve for callers that cannot
// allocate device memory (see include/fastprox_b200.h). Its scratch is the
// file-scope array below, whose device address is looked up on every call.
// ---------------------------------------------------------------------------

#include "../../include/fastprox_b200.h"

namespace fpb {
namespace {

constexpr int64_t kNoAllocPixels = int64_t(1) << 20;  // batch x height x width at most
constexpr int64_t kNoAllocImages = 64;                // batch at most
// Partial-sum slots over all images of a call: enough for one slot per row
// and column block of every image (the lean step's per-row sums, as fp_prox
// uses them, so that the sums and the iterates are the same bits), and for
// the set-up scans and the generic step's blocks: with batch x height x width
// <= 2^20, batch x height x ceil(width / 128) <= 2^13 + 2^15 for rows of 32
// or more, 64 x 1024 for narrower ones.
constexpr int64_t kNoAllocPartSlots = int64_t(1) << 16;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Byte offsets of the scratch regions.
constexpr size_t kOffD = 0;
constexpr size_t kOffU0 = kOffD + align256(kNoAllocPixels * 4);
constexpr size_t kOffU1 = kOffU0 + align256(2 * kNoAllocPixels * 4);
constexpr size_t kOffV0 = kOffU1 + align256(2 * kNoAllocPixels * 4);
constexpr size_t kOffV1 = kOffV0 + align256(2 * kNoAllocPixels * 4);
constexpr size_t kOffDual = kOffV1 + align256(2 * kNoAllocPixels * 4);
constexpr size_t kOffImg = kOffDual + align256(2 * kNoAllocPixels * 4);
constexpr size_t kOffSt = kOffImg + align256(kNoAllocImages * sizeof(IsoImage));
constexpr size_t kOffGam = kOffSt + align256(kNoAllocImages * sizeof(IsoState));
constexpr size_t kOffPart = kOffGam + align256(kNoAllocImages * sizeof(double));
constexpr size_t kOffTicket = kOffPart + align256(kNoAllocPartSlots * 2 * sizeof(double));
constexpr size_t kOffLive = kOffTicket + align256(kNoAllocImages * sizeof(unsigned));
constexpr size_t kOffErr = kOffLive + 256;
constexpr size_t kOffRes = kOffErr + 256;  // per image: gap (double), iters (int); then a flag word
constexpr size_t kNoAllocBytes = kOffRes + align256(kNoAllocImages * (sizeof(double) + sizeof(int)) + 16);

// About 48 MB. The CUDA runtime loads this file's kernels, and reserves this
// array with them, on a device the first time anything of the file runs
// there (lazy module loading): the first isotropic solve or call of the
// entry point on that device. From then on the array stays reserved there
// until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Per-image results into the scratch: gap at the input's scale, iterations,
// and flag bits (1: an image did not converge, 2: an image held an Inf).
__global__ void noalloc_results(const IsoImage *img, const IsoState *st, int64_t B, double *gaps, int *iters,
                                int *flags) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const IsoImage im = img[b];
    const IsoState s = st[b];
    double gap = 0.0;
    int it = 0;
    if (im.mode == kModeInf) {
        atomicOr(flags, 2);
    } else if (im.mode == kModeNan) {
        gap = CUDART_NAN;
    } else if (im.mode == kModeFdpg) {
        gap = isnan(s.gp) ? s.gp : fmax(s.gp, 0.0);
        if (im.e) gap = ldexp(gap, 2 * im.e);
        it = s.it;
        if (s.status != kConverged) atomicOr(flags, 1);
    }
    gaps[b] = gap;
    iters[b] = it;
}

}  // namespace
}  // namespace fpb

extern "C" FP_API fp_status fp_b200_tv_iso_noalloc(const float *x, float *z, int64_t batch, int64_t height,
                                                    int64_t width, double gamma, double tol, int max_iter,
                                                    void *stream, double *gaps, int *iters) {
    using namespace fpb;
    if (batch < 0 || height < 0 || width < 0) return FP_ESHAPE;
    if (batch == 0 || height == 0 || width == 0) return FP_OK;
    if (!x || !z) return FP_EINVAL;
    if (batch > kNoAllocImages || height > kNoAllocPixels || width > kNoAllocPixels ||
        batch * height * width > kNoAllocPixels)
        return FP_ESHAPE;
    if (!std::isfinite(gamma) || gamma < 0.0 || !(gamma <= 0x1p960)) return FP_EPARAM;
    if (!(tol >= 0.0) || !std::isfinite(tol) || max_iter < 1) return FP_EPARAM;
    // The array's address on the current device, looked up on every call (no
    // cached pointer can outlive a device reset); in host code the array's
    // name is only a stand-in for it.
    void *sym = nullptr;
    if (cudaGetSymbolAddress(&sym, g_noalloc_scratch) != cudaSuccess || !sym) {
        cudaGetLastError();
        return FP_EDEVICE;
    }
    unsigned char *base = static_cast<unsigned char *>(sym);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Geometry g{};
    g.k = 2;
    g.L[0] = height;
    g.L[1] = width;
    g.L[2] = 1;
    g.N = height * width;
    g.B = batch;
    // unit axis weights: the active axes are those of extent > 1 (tv_iso.cpp:350-358)
    IsoCall c{};
    int na = 0, act = 0;
    for (int a = 0; a < 2; ++a)
        if (g.L[a] > 1) {
            ++na;
            act = a;
        }
    c.na = na;
    c.act_axis = act;
    c.w_act = 1.0;
    c.wmax = 1.0;
    c.whmin = 1.0;
    double L2 = 0.0;
    for (int a = 0; a < 3; ++a) {
        c.wh[a] = (a < 2 && g.L[a] > 1) ? 1.0 : 0.0;
        L2 += 4.0 * c.wh[a] * c.wh[a];
    }
    c.tau = L2 > 0.0 ? 1.0 / L2 : 0.0;
    c.tol = tol;
    c.max_iter = max_iter;
    c.has_alpha = 0;
    c.alpha_stride = 0;
    c.alpha_max = 0.0;
    c.step_scale = 1.0;
    // The step's shape and partial-sum slots as a workspace of this geometry
    // has them (per-row sums of the lean 2D step), so the sums, the stopping
    // decisions and the iterates are fp_prox's.
    const StepShape sh = iso_pick_shape(FP_F32, g, 0, 0, 0);
    int64_t max_part = std::max<int64_t>(iso_setup_blocks(g), (int64_t)sh.gx * sh.gy);
    if (sh.kind == 4) max_part = std::max<int64_t>(max_part, (int64_t)sh.gx * height);
    if (batch * max_part > kNoAllocPartSlots) return FP_ESHAPE;
    IsoBuffers bf;
    bf.d = base + kOffD;
    bf.U[0] = base + kOffU0;
    bf.U[1] = base + kOffU1;
    bf.V[0] = base + kOffV0;
    bf.V[1] = base + kOffV1;
    bf.dual = base + kOffDual;
    bf.alpha = nullptr;
    bf.img = reinterpret_cast<IsoImage *>(base + kOffImg);
    bf.st = reinterpret_cast<IsoState *>(base + kOffSt);
    bf.gammas = reinterpret_cast<double *>(base + kOffGam);
    bf.part = reinterpret_cast<double *>(base + kOffPart);
    bf.ticket = reinterpret_cast<unsigned *>(base + kOffTicket);
    bf.live = reinterpret_cast<int *>(base + kOffLive);
    bf.err = reinterpret_cast<int *>(base + kOffErr);
    bf.max_part = (int)max_part;
    double *rg = reinterpret_cast<double *>(base + kOffRes);
    int *ri = reinterpret_cast<int *>(base + kOffRes + kNoAllocImages * sizeof(double));
    int *rflags = ri + kNoAllocImages;
    // the scratch keeps the last call's contents: clear what must start at zero
    cudaError_t e = cudaMemsetAsync(bf.ticket, 0, (size_t)batch * sizeof(unsigned), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bf.live, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bf.err, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(rflags, 0, sizeof(int), s);
    if (e == cudaSuccess) e = fill_double(bf.gammas, gamma, batch, s);
    if (e == cudaSuccess) e = iso_setup(FP_F32, g, c, bf, x, 0, 0, s);
    if (e != cudaSuccess) return FP_EDEVICE;
    int par = 0;
    int64_t launched = 0;
    const int chunk = 8;
    for (;;) {
        for (int j = 0; j < chunk; ++j) {
            e = iso_step(FP_F32, g, c, bf, sh, par, iso_variant(launched, max_iter, false), g.B, s);
            if (e != cudaSuccess) return FP_EDEVICE;
            par ^= 1;
            ++launched;
        }
        int live = 0;  // a pageable copy: this entry point holds no pinned memory either
        if (cudaMemcpyAsync(&live, bf.live, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return FP_EDEVICE;
        if (live == 0 || launched > (int64_t)max_iter + chunk) break;
    }
    e = iso_finalize(FP_F32, g, c, bf, z, s);
    if (e == cudaSuccess) {
        noalloc_results<<<(unsigned)((batch + 127) / 128), 128, 0, s>>>(bf.img, bf.st, batch, rg, ri, rflags);
        e = cudaGetLastError();
    }
    int flags = 0, err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flags, rflags, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, bf.err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && gaps) e = cudaMemcpyAsync(gaps, rg, (size_t)batch * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && iters) e = cudaMemcpyAsync(iters, ri, (size_t)batch * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess || err) return FP_EDEVICE;
    if (flags & 2) return FP_EINVAL;
    return (flags & 1) ? FP_ENOTCONV : FP_OK;
}
