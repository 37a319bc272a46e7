// Device helpers shared by the image-TV kernels: vector loads, fixed-tree
// block reductions in FP64, and the last-block-done epilogue that turns
// per-block partial sums into per-image decisions without a host round trip.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdint>

#include "engine.h"

namespace fpb {

constexpr int kMaxThreads = 256;

// A vector of VEC consecutive T, loaded and stored in one instruction
// (16-byte aligned when VEC * sizeof(T) == 16).
template <class T, int VEC>
struct alignas(sizeof(T) * VEC) Pack {
    T v[VEC];
};

template <class T, int VEC>
__device__ __forceinline__ void load_pack(const T *p, T (&o)[VEC]) {
    const Pack<T, VEC> q = *reinterpret_cast<const Pack<T, VEC> *>(p);
#pragma unroll
    for (int j = 0; j < VEC; ++j) o[j] = q.v[j];
}

template <class T, int VEC>
__device__ __forceinline__ void store_pack(T *p, const T (&o)[VEC]) {
    Pack<T, VEC> q;
#pragma unroll
    for (int j = 0; j < VEC; ++j) q.v[j] = o[j];
    *reinterpret_cast<Pack<T, VEC> *>(p) = q;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Sum of v over the block in a fixed tree (warp shuffles, then warp 0):
// the same bits for the same inputs on every run. Valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < nw ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

__device__ __forceinline__ double block_max(double v, double *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = -CUDART_INF;
    if (wid == 0) {
        r = lane < nw ? sh[lane] : -CUDART_INF;
        r = warp_max(r);
    }
    return r;
}

// After thread 0 has written this block's partials: true in every thread of
// the one block that arrives last among the nblk blocks of an image (the
// classic threadfence reduction). That block then reads all partials.
__device__ __forceinline__ bool arrive_last(unsigned *ticket, unsigned nblk, int *sh_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        *sh_flag = (t == nblk - 1) ? 1 : 0;
    }
    __syncthreads();
    const bool last = *sh_flag != 0;
    if (last) __threadfence();
    return last;
}

// Sum of part[i * stride + off] for i < n in a fixed order (a strided pass
// per thread, then the block tree), read past L1. Valid in thread 0.
__device__ __forceinline__ double sum_partials(const double *part, int n, int stride, int off, double *sh) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += __ldcg(part + (int64_t)i * stride + off);
    return block_sum(s, sh);
}

__device__ __forceinline__ double max_partials(const double *part, int n, int stride, int off, double *sh) {
    double s = -CUDART_INF;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s = fmax(s, __ldcg(part + (int64_t)i * stride + off));
    return block_max(s, sh);
}

// t' = (1 + sqrt(1 + 4 t^2)) / 2 (the reference's fista_t, src/ops/image_util.hpp:72).
__device__ __forceinline__ double fista_t(double t) { return 0.5 * (1.0 + sqrt(1.0 + 4.0 * t * t)); }

}  // namespace fpb
