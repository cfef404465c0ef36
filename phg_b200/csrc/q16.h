// The 16-bit-column SELL layout ("q16") of the matrix (q16.cu).
#pragma once
#include "solve.h"

namespace phgb {

// Writable pointers of the layout, for its construction.
struct Q16Out {
    const int32_t *sptr;
    int32_t *perm;
    uint16_t *len, *split;
    int32_t *base0, *base1;
    uint16_t *cols;
    float *vals32;
    double *vals64;
    int32_t *src;      // CSR index of each stored entry, -1 for padding (for value refills)
};

// Slice sizes (entries) of the stored slices; then the fill from CSR.
// `order[k]` is the SELL slice stored k-th (widest first), `sell_perm` /
// `sell_len` the SELL sort.  `nofit` is set to 1 when a row spans more than
// two windows (its offsets are then written as 0, so no product can read
// outside x, but the layout must not be used).
cudaError_t launch_q16_sizes(int64_t nslices, const uint16_t *sell_len, const int32_t *order, int32_t *size,
                             cudaStream_t s);
cudaError_t launch_q16_fill(int64_t nslices, const int32_t *rp, const int32_t *ci, const double *va,
                            const int32_t *sell_perm, const uint16_t *sell_len, const int32_t *order,
                            const Q16Out &O, int *nofit, cudaStream_t s);

// FP32 product y = A x (unroll 1 or 2 steps), FP64 product y = A x.
// New values for the same pattern: vals64[i] = va[src[i]], vals32[i] its
// rounding (0 for padding), over the `total` stored entries.
cudaError_t launch_q16_refill(int64_t total, const int32_t *src, const double *va, float *vals32, double *vals64,
                              cudaStream_t s);
cudaError_t launch_q16_spmv32(const Q16View &Q, int unroll, const float *x, float *y, cudaStream_t s);
cudaError_t launch_q16_spmv64(const Q16View &Q, const double *x, double *y, cudaStream_t s);

// The FP64 product computing p.Ap and alpha (x = p), for the FP64 PCG.
cudaError_t launch_q16_spmv64_dot(const Q16View &Q, const double *x, double *y, double *partials, PcgState *st,
                                  cudaStream_t s);

}  // namespace phgb
