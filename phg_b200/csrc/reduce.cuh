// Device helpers shared by the iterative solvers: barrier-free grid-wide
// sums with a deterministic combination order, and 16-byte vector loads.
#pragma once
#include "common.cuh"

namespace phgb {

// Grid-wide sum of two values without block barriers: each warp reduces its
// values (fixed butterfly), the last warp of a block to arrive adds the
// block's warp sums in warp order and publishes them, and the last block to
// arrive adds the block sums in block order.  Nobody waits: a warp that is
// not last simply leaves.  Returns true in exactly one thread (lane 0 of the
// final warp), which then holds the totals.  Kernels call grid_sum_init()
// once, before any early exit that is not uniform across the block.
struct RedShared {
    double a[32], b[32];
    unsigned cnt;
};

__device__ __forceinline__ RedShared &red_smem() {
    __shared__ RedShared r;
    return r;
}

__device__ __forceinline__ void grid_sum_init() {
    if (threadIdx.x == 0) red_smem().cnt = 0u;
    __syncthreads();
}

__device__ __forceinline__ bool grid_sum2(double &a, double &b, double *partials, unsigned *ticket) {
    RedShared &R = red_smem();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    unsigned arrived = 0;
    if (lane == 0) {
        R.a[w] = a;
        R.b[w] = b;
        __threadfence_block();
        arrived = atomicAdd(&R.cnt, 1u);
    }
    arrived = __shfl_sync(0xffffffffu, arrived, 0);
    if (arrived != (unsigned)nw - 1) return false;
    __threadfence_block();
    double ta = lane < nw ? ((volatile double *)R.a)[lane] : 0.0;
    double tb = lane < nw ? ((volatile double *)R.b)[lane] : 0.0;
    ta = warp_sum(ta);
    tb = warp_sum(tb);
    if (lane == 0) {
        partials[2 * blockIdx.x] = ta;
        partials[2 * blockIdx.x + 1] = tb;
        __threadfence();
        arrived = atomicAdd(ticket, 1u);
    }
    arrived = __shfl_sync(0xffffffffu, arrived, 0);
    if (arrived != gridDim.x - 1) return false;
    __threadfence();
    // four independent accumulators per lane keep several loads in flight;
    // they are combined in a fixed order
    double sa[4] = {0.0, 0.0, 0.0, 0.0}, sb[4] = {0.0, 0.0, 0.0, 0.0};
    for (unsigned i0 = 0; i0 < gridDim.x; i0 += 128) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const unsigned i = i0 + q * 32 + lane;
            if (i < gridDim.x) {
                sa[q] += __ldcg(&partials[2 * i]);
                sb[q] += __ldcg(&partials[2 * i + 1]);
            }
        }
    }
    double ta2 = warp_sum((sa[0] + sa[1]) + (sa[2] + sa[3]));
    double tb2 = warp_sum((sb[0] + sb[1]) + (sb[2] + sb[3]));
    if (lane == 0) {
        a = ta2;
        b = tb2;
        *ticket = 0u;
    }
    return lane == 0;
}

// Loads/stores of V consecutive elements (16 bytes) at an index that is a
// multiple of V.
template <typename T> struct Vec16;
template <> struct Vec16<double> { using type = double2; static constexpr int V = 2; };
template <> struct Vec16<float> { using type = float4; static constexpr int V = 4; };

template <typename T> struct VArr { T v[Vec16<T>::V]; };

// True when every pointer is 16-byte aligned, so the vector path may be used
// (callers may pass vectors at any 8-byte offset; the scalar loop covers them).
template <typename... Ps> __device__ __forceinline__ bool aligned16(const Ps *...ps) {
    return ((reinterpret_cast<uintptr_t>(ps) | ...) & 15u) == 0;
}

template <typename T> __device__ __forceinline__ VArr<T> vload(const T *p) {
    VArr<T> a;
    *reinterpret_cast<typename Vec16<T>::type *>(a.v) = *reinterpret_cast<const typename Vec16<T>::type *>(p);
    return a;
}
template <typename T> __device__ __forceinline__ VArr<T> vload_ro(const T *p) {
    VArr<T> a;
    *reinterpret_cast<typename Vec16<T>::type *>(a.v) = __ldg(reinterpret_cast<const typename Vec16<T>::type *>(p));
    return a;
}
template <typename T> __device__ __forceinline__ void vstore(T *p, const VArr<T> &a) {
    *reinterpret_cast<typename Vec16<T>::type *>(p) = *reinterpret_cast<const typename Vec16<T>::type *>(a.v);
}

}  // namespace phgb
