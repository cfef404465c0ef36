// The 16-bit-column SELL layout (q16.h): construction from CSR and the
// products of the mixed-precision solver on it.
//
// Bytes per entry of the FP32 product: 4 (value) + 2 (column offset), against
// 4 + 4 for 32-bit columns; per stored row position 16 bytes of metadata
// (row, length, split, two bases).  One warp per slice, a lane per row, four
// entries of the row per load: a warp moves 512 bytes of values and 256
// bytes of offsets per step.
#include "common.cuh"
#include "pcg_final.cuh"
#include "q16.cuh"
#include "q16.h"
#include "reduce.cuh"

#include <limits.h>

#include <algorithm>

namespace phgb {

__global__ void q16_sizes_kernel(int64_t nslices, const uint16_t *__restrict__ len, const int32_t *__restrict__ order,
                                 int32_t *__restrict__ size) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nslices; k += (int64_t)gridDim.x * blockDim.x)
        size[k] = 128 * ((len[(int64_t)order[k] * 32] + 3) / 4);
}

// One thread per stored position (the 32 positions of a slice are a warp's
// lanes).  Three passes over the row's CSR entries: the smallest column
// (base0); the size of the first window and the smallest and largest column
// outside it; the entries, first-window entries first, each window in CSR
// order.  Positions past the row's length up to the slice's width (rounded
// up to 4) are zero.
__global__ void __launch_bounds__(kVecThreads, kResidentBlocks)
q16_fill_kernel(int64_t npos, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                const double *__restrict__ va, const int32_t *__restrict__ sell_perm,
                const uint16_t *__restrict__ sell_len, const int32_t *__restrict__ order,
                const int32_t *__restrict__ sptr, int32_t *__restrict__ perm, uint16_t *__restrict__ len,
                uint16_t *__restrict__ split, int32_t *__restrict__ base0, int32_t *__restrict__ base1,
                uint16_t *__restrict__ cols, float *__restrict__ vals32, double *__restrict__ vals64,
                int32_t *__restrict__ src, int *nofit) {
    for (int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < npos;
         pos += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = pos >> 5;
        const int lane = (int)(pos & 31);
        const int64_t src0 = (int64_t)order[k] * 32;
        const int32_t row = sell_perm[src0 + lane];
        const int l = sell_len[src0 + lane];
        const int wq = (sell_len[src0] + 3) & ~3;   // SELL slices are sorted: position 0 is the widest
        const int64_t b = (int64_t)sptr[k] + 4 * lane;
        int32_t b0 = 0, b1 = 0;
        int sp = 0, j = 0;
        if (row >= 0 && l > 0) {
            const int64_t r0 = rp[row];
            b0 = INT_MAX;
            for (int t = 0; t < l; t++) b0 = min(b0, ci[r0 + t]);
            b1 = INT_MAX;
            int32_t hi = -1;
            for (int t = 0; t < l; t++) {
                const int32_t c = ci[r0 + t];
                if (c - b0 < 65536) {
                    sp++;
                } else {
                    b1 = min(b1, c);
                    hi = max(hi, c);
                }
            }
            if (hi < 0) b1 = b0;
            const bool fits = hi < 0 || hi - b1 < 65536;
            if (!fits) atomicExch(nofit, 1);
            int j0 = 0, j1 = sp;
            for (int t = 0; t < l; t++) {
                const int32_t c = ci[r0 + t];
                const bool w0 = c - b0 < 65536;
                const int jj = w0 ? j0++ : j1++;
                const int64_t idx = b + (int64_t)(jj >> 2) * 128 + (jj & 3);
                cols[idx] = fits ? (uint16_t)(c - (w0 ? b0 : b1)) : (uint16_t)0;
                const double v = va[r0 + t];
                vals64[idx] = v;
                vals32[idx] = (float)v;
                src[idx] = (int32_t)(r0 + t);
            }
            j = l;
        }
        for (; j < wq; j++) {
            const int64_t idx = b + (int64_t)(j >> 2) * 128 + (j & 3);
            cols[idx] = 0;
            vals64[idx] = 0.0;
            vals32[idx] = 0.0f;
            src[idx] = -1;
        }
        perm[pos] = row;
        len[pos] = (uint16_t)l;
        split[pos] = (uint16_t)sp;
        base0[pos] = b0;
        base1[pos] = b1;
    }
}

// FP32 product; with DOT also p.Ap (x = p) and alpha (pcg_pap_final).
template <bool DOT, int U>
__global__ void __launch_bounds__(kVecThreads, kResidentBlocks)
q16_spmv32_kernel(const Q16View Q, const float *__restrict__ x, float *__restrict__ y, double *partials,
                  PcgState *st) {
    if (DOT && st->done) return;
    if (DOT) grid_sum_init();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kVecThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kVecThreads) >> 5;
    double dot = 0.0, dummy = 0.0;
    for (int64_t s = warp; s < Q.nslices; s += nwarps) {
        const int64_t pos = s * 32 + lane;
        const int32_t row = Q.perm[pos];
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
                if (j < l) acc += v[u].x * __ldg(&x[q16_col(j, sp, b0, b1, c[u].x & 0xffffu)]);
                if (j + 1 < l) acc += v[u].y * __ldg(&x[q16_col(j + 1, sp, b0, b1, c[u].x >> 16)]);
                if (j + 2 < l) acc += v[u].z * __ldg(&x[q16_col(j + 2, sp, b0, b1, c[u].y & 0xffffu)]);
                if (j + 3 < l) acc += v[u].w * __ldg(&x[q16_col(j + 3, sp, b0, b1, c[u].y >> 16)]);
            }
        }
        if (row >= 0) {
            y[row] = acc;
            if (DOT) dot += (double)x[row] * (double)acc;
        }
    }
    if (!DOT) return;
    if (grid_sum2(dot, dummy, partials, st->ticket)) pcg_pap_final(dot, st);
}

// FP64 product; with DOT also p.Ap (x = p) and alpha, for the FP64 PCG.
template <bool DOT>
__global__ void __launch_bounds__(kVecThreads, kResidentBlocks)
q16_spmv64_kernel(const Q16View Q, const double *__restrict__ x, double *__restrict__ y, double *partials,
                  PcgState *st) {
    if (DOT && st->done) return;
    if (DOT) grid_sum_init();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kVecThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kVecThreads) >> 5;
    double dot = 0.0, dummy = 0.0;
    for (int64_t s = warp; s < Q.nslices; s += nwarps) {
        const int64_t pos = s * 32 + lane;
        const int32_t row = Q.perm[pos];
        const double acc = q16_row64(Q, s, lane, Q.len[pos], Q.split[pos], Q.base0[pos], Q.base1[pos], x);
        if (row >= 0) {
            y[row] = acc;
            if (DOT) dot += x[row] * acc;
        }
    }
    if (!DOT) return;
    if (grid_sum2(dot, dummy, partials, st->ticket)) pcg_pap_final(dot, st);
}

cudaError_t launch_q16_sizes(int64_t nslices, const uint16_t *sell_len, const int32_t *order, int32_t *size,
                             cudaStream_t s) {
    q16_sizes_kernel<<<vec_blocks(nslices), kVecThreads, 0, s>>>(nslices, sell_len, order, size);
    return cudaGetLastError();
}

cudaError_t launch_q16_fill(int64_t nslices, const int32_t *rp, const int32_t *ci, const double *va,
                            const int32_t *sell_perm, const uint16_t *sell_len, const int32_t *order,
                            const Q16Out &O, int *nofit, cudaStream_t s) {
    const int64_t npos = nslices * 32;
    q16_fill_kernel<<<vec_blocks(npos), kVecThreads, 0, s>>>(npos, rp, ci, va, sell_perm, sell_len, order, O.sptr,
                                                             O.perm, O.len, O.split, O.base0, O.base1, O.cols,
                                                             O.vals32, O.vals64, O.src, nofit);
    return cudaGetLastError();
}

__global__ void q16_refill_kernel(int64_t total, const int32_t *__restrict__ src, const double *__restrict__ va,
                                  float *__restrict__ vals32, double *__restrict__ vals64) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = src[i];
        const double v = k >= 0 ? va[k] : 0.0;
        vals64[i] = v;
        vals32[i] = (float)v;
    }
}

cudaError_t launch_q16_refill(int64_t total, const int32_t *src, const double *va, float *vals32, double *vals64,
                              cudaStream_t s) {
    q16_refill_kernel<<<vec_blocks(total), kVecThreads, 0, s>>>(total, src, va, vals32, vals64);
    return cudaGetLastError();
}

cudaError_t launch_q16_spmv32(const Q16View &Q, int unroll, const float *x, float *y, cudaStream_t s) {
    const int sb = vec_blocks(Q.nslices * 32);
    if (unroll == 2)
        q16_spmv32_kernel<false, 2><<<sb, kVecThreads, 0, s>>>(Q, x, y, nullptr, nullptr);
    else
        q16_spmv32_kernel<false, 1><<<sb, kVecThreads, 0, s>>>(Q, x, y, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_q16_spmv64(const Q16View &Q, const double *x, double *y, cudaStream_t s) {
    q16_spmv64_kernel<false><<<vec_blocks(Q.nslices * 32), kVecThreads, 0, s>>>(Q, x, y, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_q16_spmv64_dot(const Q16View &Q, const double *x, double *y, double *partials, PcgState *st,
                                  cudaStream_t s) {
    q16_spmv64_kernel<true><<<vec_blocks(Q.nslices * 32), kVecThreads, 0, s>>>(Q, x, y, partials, st);
    return cudaGetLastError();
}

}  // namespace phgb
