// Device helpers shared by the iterative solvers: barrier-free grid-wide
// sums with a deterministic combination order, and 16-byte vector loads.
#pragma once
#include "common.cuh"
#include "solve.h"

#include <cuda/atomic>

namespace phgb {

// Grid-wide sum of two values without block barriers: each warp reduces its
// values (fixed butterfly), the last warp of a block to arrive adds the
// block's warp sums in warp order and publishes them; the last block of each
// group of kRedGroup consecutive blocks adds the group's block sums, and the
// last group adds the group sums.  Each stage is one round of loads issued
// together, so the finishing block waits for two L2 round trips however large
// the grid is (one warp summing 1184 block sums one after another took ~14 us
// per launch; the two-stage tree ~5 us).  The combination order is fixed for
// a given grid, so results are reproducible.  Nobody waits: a warp that is not
// last simply leaves.  Returns true in exactly one thread (lane 0 of the final
// warp), which then holds the totals.  Kernels call grid_sum_init() once,
// before any early exit that is not uniform across the block.
//
// Workspace: partials holds 2 * (gridDim.x + ceil(gridDim.x / kRedGroup))
// doubles at a 16-byte aligned address; tickets holds kRedTickets counters,
// zero before the first launch (every stage resets its own counter).
struct RedShared {
    double a[32], b[32];
    unsigned cnt;
};

__device__ __forceinline__ RedShared &red_smem() {
    __shared__ RedShared r;
    return r;
}

// Arrival at a ticket: a device-scope fetch-add with acquire-release order.
// The release publishes the caller's partial sum written before it; the
// last arrival's acquire makes every earlier arrival's partial visible.
// (A __threadfence before and after a relaxed atomicAdd does the same at a
// higher cost: 5.8 against 4.9 us for a 1184-block sum.)
__device__ __forceinline__ unsigned ticket_add_acq_rel(unsigned *t) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> r(*t);
    return r.fetch_add(1u, cuda::memory_order_acq_rel);
}

__device__ __forceinline__ void grid_sum_init() {
    if (threadIdx.x == 0) red_smem().cnt = 0u;
    __syncthreads();
}

__device__ __forceinline__ bool grid_sum2(double &a, double &b, double *partials, unsigned *tickets) {
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
    // stage 1: block sums -> group sums
    double2 *P = reinterpret_cast<double2 *>(partials);
    const unsigned nb = gridDim.x, g = blockIdx.x / kRedGroup, g0 = g * kRedGroup;
    const unsigned gs = min((unsigned)kRedGroup, nb - g0), ng = (nb + kRedGroup - 1) / kRedGroup;
    if (lane == 0) {
        P[blockIdx.x] = make_double2(ta, tb);
        arrived = ticket_add_acq_rel(&tickets[1 + g]);
    }
    arrived = __shfl_sync(0xffffffffu, arrived, 0);
    if (arrived != gs - 1) return false;
    __syncwarp();   // the lanes' loads below come after lane 0's acquire
    double2 p0 = lane < gs ? __ldcg(&P[g0 + lane]) : make_double2(0.0, 0.0);
    double2 p1 = lane + 32 < gs ? __ldcg(&P[g0 + lane + 32]) : make_double2(0.0, 0.0);
    ta = warp_sum(p0.x + p1.x);
    tb = warp_sum(p0.y + p1.y);
    if (lane == 0) {
        tickets[1 + g] = 0u;
        P[nb + g] = make_double2(ta, tb);
        arrived = ticket_add_acq_rel(&tickets[0]);
    }
    arrived = __shfl_sync(0xffffffffu, arrived, 0);
    if (arrived != ng - 1) return false;
    // stage 2: group sums -> total
    __syncwarp();
    p0 = lane < ng ? __ldcg(&P[nb + lane]) : make_double2(0.0, 0.0);
    ta = warp_sum(p0.x);
    tb = warp_sum(p0.y);
    if (lane == 0) {
        a = ta;
        b = tb;
        tickets[0] = 0u;
    }
    return lane == 0;
}

// The same for three sums, with the same stages and ordering.  Workspace:
// 3 * (gridDim.x + ceil(gridDim.x / kRedGroup)) doubles in `partials`.
struct RedShared3 {
    double v[3][32];
    unsigned cnt;
};

__device__ __forceinline__ RedShared3 &red_smem3() {
    __shared__ RedShared3 r;
    return r;
}

__device__ __forceinline__ void grid_sum3_init() {
    if (threadIdx.x == 0) red_smem3().cnt = 0u;
    __syncthreads();
}

__device__ __forceinline__ bool grid_sum3(double (&v)[3], double *partials, unsigned *tickets) {
    RedShared3 &R = red_smem3();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] = warp_sum(v[k]);
    unsigned arrived = 0;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 3; k++) R.v[k][w] = v[k];
        __threadfence_block();
        arrived = atomicAdd(&R.cnt, 1u);
    }
    arrived = __shfl_sync(0xffffffffu, arrived, 0);
    if (arrived != (unsigned)nw - 1) return false;
    __threadfence_block();
    double t[3];
#pragma unroll
    for (int k = 0; k < 3; k++) t[k] = warp_sum(lane < nw ? ((volatile double *)R.v[k])[lane] : 0.0);
    // stage 1: block sums -> group sums
    const unsigned nb = gridDim.x, g = blockIdx.x / kRedGroup, g0 = g * kRedGroup;
    const unsigned gs = min((unsigned)kRedGroup, nb - g0), ng = (nb + kRedGroup - 1) / kRedGroup;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 3; k++) partials[3 * (size_t)blockIdx.x + k] = t[k];
        arrived = ticket_add_acq_rel(&tickets[1 + g]);
    }
    arrived = __shfl_sync(0xffffffffu, arrived, 0);
    if (arrived != gs - 1) return false;
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double a = lane < gs ? __ldcg(&partials[3 * (size_t)(g0 + lane) + k]) : 0.0;
        const double b = lane + 32 < gs ? __ldcg(&partials[3 * (size_t)(g0 + lane + 32) + k]) : 0.0;
        t[k] = warp_sum(a + b);
    }
    if (lane == 0) {
        tickets[1 + g] = 0u;
#pragma unroll
        for (int k = 0; k < 3; k++) partials[3 * (size_t)(nb + g) + k] = t[k];
        arrived = ticket_add_acq_rel(&tickets[0]);
    }
    arrived = __shfl_sync(0xffffffffu, arrived, 0);
    if (arrived != ng - 1) return false;
    // stage 2: group sums -> totals
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 3; k++)
        t[k] = warp_sum(lane < ng ? __ldcg(&partials[3 * (size_t)(nb + lane) + k]) : 0.0);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = t[k];
        tickets[0] = 0u;
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
