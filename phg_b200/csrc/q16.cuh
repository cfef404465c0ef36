// Device helpers of the 16-bit-column layout, shared by its kernels
// (q16.cu) and the epilogue products (spmv_epi.cuh).
#pragma once
#include "solve.h"

namespace phgb {

// Column of entry j of a lane's row.
__device__ __forceinline__ int32_t q16_col(int j, int sp, int32_t b0, int32_t b1, unsigned off) {
    return (j < sp ? b0 : b1) + (int32_t)off;
}

// FP64 row sum of the layout's FP64 values against a vector read through
// xv(col) -> double: acc = sum_j a_ij xv(j) for the lane's row (slice s,
// lane `lane`).
template <typename XV>
__device__ __forceinline__ double q16_row64_with(const Q16View &Q, int64_t s, int lane, int l, int sp, int32_t b0,
                                                 int32_t b1, XV xv) {
    const int wq = (__shfl_sync(0xffffffffu, l, 0) + 3) >> 2;
    const uint2 *cp = reinterpret_cast<const uint2 *>(Q.cols + Q.sptr[s]) + lane;
    const double2 *vp = reinterpret_cast<const double2 *>(Q.vals64 + Q.sptr[s]) + 2 * lane;
    double acc = 0.0;
    for (int jq = 0; jq < wq; jq++) {
        const bool ok = 4 * jq < l;
        const uint2 c = ok ? __ldcs(cp + 32 * jq) : make_uint2(0u, 0u);
        const double2 v0 = ok ? __ldcs(vp + 64 * jq) : make_double2(0.0, 0.0);
        const double2 v1 = ok ? __ldcs(vp + 64 * jq + 1) : make_double2(0.0, 0.0);
        const int j = 4 * jq;
        if (j < l) acc += v0.x * xv(q16_col(j, sp, b0, b1, c.x & 0xffffu));
        if (j + 1 < l) acc += v0.y * xv(q16_col(j + 1, sp, b0, b1, c.x >> 16));
        if (j + 2 < l) acc += v1.x * xv(q16_col(j + 2, sp, b0, b1, c.y & 0xffffu));
        if (j + 3 < l) acc += v1.y * xv(q16_col(j + 3, sp, b0, b1, c.y >> 16));
    }
    return acc;
}

// The same against an FP32 or FP64 vector x.
template <typename XT>
__device__ __forceinline__ double q16_row64(const Q16View &Q, int64_t s, int lane, int l, int sp, int32_t b0,
                                            int32_t b1, const XT *__restrict__ x) {
    return q16_row64_with(Q, s, lane, l, sp, b0, b1, [x](int32_t c) { return (double)__ldg(&x[c]); });
}

}  // namespace phgb
