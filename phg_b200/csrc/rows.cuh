// Row sums of the sliced SpMV layouts (SELL-C-sigma, pair SELL, q16), as
// device functors that the fused solver kernels share.  A layout functor L
// provides
//   int64_t nslices() const
//   int32_t row(int64_t pos) const     matrix row at stored position pos, -1 = padding
//   acc sum(int64_t s, int lane, int64_t pos, const X *x) const
//                                      (A x) of the row at position pos = 32 s + lane
// The warp of a slice calls sum() with all 32 lanes (shuffles inside).
#pragma once
#include "q16.cuh"
#include "solve.h"

namespace phgb {

// The FP32 products of the mixed solver round each product a_ij x_j and each
// partial sum to FP32 on its own (__fmul_rn, __fadd_rn): contracted into
// fused multiply-adds, the sums perturb the single-reduction recurrence
// enough to cost it a fifth more iterations at 2 million rows (264 against
// 219 on P2 64^3; 216 with exact products summed in FP64, whose conversions
// cost more time than the three iterations they save).
// FP32 values of the q16 layout, four entries per lane per step, U steps in flight.
template <int U>
struct Q16Rows32 {
    Q16View Q;
    __device__ __forceinline__ int64_t nslices() const { return Q.nslices; }
    __device__ __forceinline__ int32_t row(int64_t pos) const { return Q.perm[pos]; }
    __device__ __forceinline__ float sum(int64_t s, int lane, int64_t pos, const float *__restrict__ x) const {
        const int l = Q.len[pos];
        const int sp = Q.split[pos];
        const int32_t b0 = Q.base0[pos], b1 = Q.base1[pos];
        const int wq = (__shfl_sync(0xffffffffu, l, 0) + 3) >> 2;
        const uint2 *cp = reinterpret_cast<const uint2 *>(Q.cols + Q.sptr[s]) + lane;
        const float4 *vp = reinterpret_cast<const float4 *>(Q.vals32 + Q.sptr[s]) + lane;
        float acc = 0.0f;
        for (int jq = 0; jq < wq; jq += U) {
            uint2 c[U];
            float4 v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool ok = 4 * (jq + u) < l;
                c[u] = ok ? __ldcs(cp + 32 * (jq + u)) : make_uint2(0u, 0u);
                v[u] = ok ? __ldcs(vp + 32 * (jq + u)) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = 4 * (jq + u);
                if (j < l) acc = fma_free(acc, v[u].x, __ldg(&x[q16_col(j, sp, b0, b1, c[u].x & 0xffffu)]));
                if (j + 1 < l) acc = fma_free(acc, v[u].y, __ldg(&x[q16_col(j + 1, sp, b0, b1, c[u].x >> 16)]));
                if (j + 2 < l) acc = fma_free(acc, v[u].z, __ldg(&x[q16_col(j + 2, sp, b0, b1, c[u].y & 0xffffu)]));
                if (j + 3 < l) acc = fma_free(acc, v[u].w, __ldg(&x[q16_col(j + 3, sp, b0, b1, c[u].y >> 16)]));
            }
        }
        return acc;
    }
};

// FP64 values of the q16 layout against an FP64 vector.
struct Q16Rows64 {
    Q16View Q;
    __device__ __forceinline__ int64_t nslices() const { return Q.nslices; }
    __device__ __forceinline__ int32_t row(int64_t pos) const { return Q.perm[pos]; }
    __device__ __forceinline__ double sum_x(int64_t s, int lane, int64_t pos, const double *__restrict__ x) const {
        return q16_row64(Q, s, lane, Q.len[pos], Q.split[pos], Q.base0[pos], Q.base1[pos], x);
    }
};

// SELL-C-sigma, one entry per lane per step; VT = value type, ACC = sum type
// (FP32 sums as the other FP32 rows; FP64 values are summed in FP64).
template <typename VT, typename ACC, int U>
struct SellRows {
    int64_t nsl;
    const int32_t *perm;
    const uint16_t *len;
    const int32_t *sptr;
    const int32_t *cols;
    const VT *vals;
    __device__ __forceinline__ int64_t nslices() const { return nsl; }
    __device__ __forceinline__ int32_t row(int64_t pos) const { return perm[pos]; }
    __device__ __forceinline__ ACC sum(int64_t s, int lane, int64_t pos, const float *__restrict__ x) const {
        const int l = len[pos];
        const int w = __shfl_sync(0xffffffffu, l, 0);
        const int64_t b = (int64_t)sptr[s] + lane;
        ACC acc = (ACC)0;
        for (int j = 0; j < w; j += U) {
            int32_t c[U];
            VT v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool ok = j + u < l;
                c[u] = ok ? __ldcs(&cols[b + 32 * (j + u)]) : 0;
                v[u] = ok ? __ldcs(&vals[b + 32 * (j + u)]) : (VT)0;
            }
#pragma unroll
            for (int u = 0; u < U; u++)
                if (j + u < l) {
                    if constexpr (sizeof(ACC) == 4) acc = fma_free(acc, v[u], __ldg(&x[c[u]]));
                    else acc += (ACC)v[u] * (ACC)__ldg(&x[c[u]]);
                }
        }
        return acc;
    }
    // against an FP64 vector
    __device__ __forceinline__ double sum_x(int64_t s, int lane, int64_t pos, const double *__restrict__ x) const {
        const int l = len[pos];
        const int w = __shfl_sync(0xffffffffu, l, 0);
        const int64_t b = (int64_t)sptr[s] + lane;
        double acc = 0.0;
        for (int j = 0; j < w; j += U) {
            int32_t c[U];
            VT v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool ok = j + u < l;
                c[u] = ok ? __ldcs(&cols[b + 32 * (j + u)]) : 0;
                v[u] = ok ? __ldcs(&vals[b + 32 * (j + u)]) : (VT)0;
            }
#pragma unroll
            for (int u = 0; u < U; u++)
                if (j + u < l) acc += (double)v[u] * __ldg(&x[c[u]]);
        }
        return acc;
    }
};

// Pair SELL (two consecutive entries of a row per lane), FP32.
template <int U>
struct PairRows32 {
    int64_t nsl;
    Sell2View S2;
    __device__ __forceinline__ int64_t nslices() const { return nsl; }
    __device__ __forceinline__ int32_t row(int64_t pos) const { return S2.perm2[pos]; }
    __device__ __forceinline__ float sum(int64_t s, int lane, int64_t pos, const float *__restrict__ x) const {
        const int l = S2.len2[pos];
        const int wp = (__shfl_sync(0xffffffffu, l, 0) + 1) >> 1;
        const int2 *cp = reinterpret_cast<const int2 *>(S2.cols2 + S2.sptr2[s]) + lane;
        const float2 *vp = reinterpret_cast<const float2 *>(S2.vals2 + S2.sptr2[s]) + lane;
        float acc = 0.0f;
        for (int jp = 0; jp < wp; jp += U) {
            int2 c[U];
            float2 v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool ok = 2 * (jp + u) < l;
                c[u] = ok ? __ldcs(cp + 32 * (jp + u)) : make_int2(0, 0);
                v[u] = ok ? __ldcs(vp + 32 * (jp + u)) : make_float2(0.0f, 0.0f);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int j = 2 * (jp + u);
                if (j < l) acc = fma_free(acc, v[u].x, __ldg(&x[c[u].x]));
                if (j + 1 < l) acc = fma_free(acc, v[u].y, __ldg(&x[c[u].y]));
            }
        }
        return acc;
    }
};

}  // namespace phgb
