// Shared helpers for the phg_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define PHGB_WARP 32

// Status words written by kernels into the system's device status block; the
// host reads them after the stream is synchronised.
enum {
    PHGB_DEV_OK = 0,
    PHGB_DEV_ROW_OVERFLOW = 1,   // a matrix row exceeded the row-walk capacity
    PHGB_DEV_BAD_INDEX = 2,      // a DOF / vertex index out of range
    PHGB_DEV_COUNT_MISMATCH = 3, // two passes of the row walk disagreed
    PHGB_DEV_NONFINITE = 4,      // a coordinate, kappa, f or g value is NaN or infinite
    PHGB_DEV_PATTERN_CHANGED = 5,// a rebuild found an exact zero where the pattern had none, or the reverse
    PHGB_DEV_DUPLICATE = 6       // a row's first segment names a column twice
};

// IEEE round-to-nearest double arithmetic with no contraction into fused
// multiply-adds: the assembly kernels reproduce the reference's operation
// order exactly, so each product and sum is rounded on its own.
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }

// acc + a x in FP32 with the product and the sum rounded on their own (no
// fused multiply-add): the row sums of the mixed solver's FP32 products.
__device__ __forceinline__ float fma_free(float acc, float a, float x) { return __fadd_rn(acc, __fmul_rn(a, x)); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ int warp_sumi(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

static inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Asynchronous global -> shared copies (cp.async; both addresses aligned to
// the size) and the wait for all of the calling thread's copies.
__device__ __forceinline__ void copy_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy_async8(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy_async4(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
