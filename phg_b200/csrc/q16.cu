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

// The layout of a slice: position (lane) p holds a row; the row's entries
// are stored first-window entries first (columns below base0 + 65536, base0
// the row's smallest column), then the rest (offsets from base1, the
// smallest column at or above base0 + 65536), each window in CSR order; entry
// j of lane p sits at sptr + 4 p + 128 (j / 4) + j % 4, so a lane reads four
// consecutive entries with one load.  Positions past the row's length up to
// the slice's width (rounded up to 4) are zero.

// Staged construction, one warp per slice: the warp copies the slice's 32
// CSR rows into shared memory with coalesced loads (all rows' loads issued
// before any is used), then each lane lays out its own row from there and
// writes it four entries at a time with 16-byte stores.  Slices wider than
// the staging area (kQ16StageW entries) take the lane-per-row path that
// reads the CSR directly.
constexpr int kQ16StageW = 72;     // entries of a row the staging area holds
constexpr int kQ16FillWarps = 1;   // warps per block (32 x 73 x 12 bytes of staging)

__device__ __forceinline__ void q16_row_direct(const int32_t *__restrict__ ci, const double *__restrict__ va,
                                               int64_t r0, int l, int wq, int64_t b, int32_t &b0, int32_t &b1,
                                               int &sp, uint16_t *__restrict__ cols, float *__restrict__ vals32,
                                               double *__restrict__ vals64, int32_t *__restrict__ src, int *nofit) {
    b0 = INT_MAX;
    for (int t = 0; t < l; t++) b0 = min(b0, ci[r0 + t]);
    b1 = INT_MAX;
    int32_t hi = -1;
    sp = 0;
    for (int t = 0; t < l; t++) {
        const int32_t c = ci[r0 + t];
        if (c - b0 < 65536) sp++;
        else {
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
    for (int j = l; j < wq; j++) {
        const int64_t idx = b + (int64_t)(j >> 2) * 128 + (j & 3);
        cols[idx] = 0;
        vals64[idx] = 0.0;
        vals32[idx] = 0.0f;
        src[idx] = -1;
    }
}

__global__ void __launch_bounds__(kQ16FillWarps * 32)
q16_fill_staged_kernel(int64_t nslices, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                       const double *__restrict__ va, const int32_t *__restrict__ sell_perm,
                       const uint16_t *__restrict__ sell_len, const int32_t *__restrict__ order,
                       const int32_t *__restrict__ sptr, int32_t *__restrict__ perm, uint16_t *__restrict__ len,
                       uint16_t *__restrict__ split, int32_t *__restrict__ base0, int32_t *__restrict__ base1,
                       uint16_t *__restrict__ cols, float *__restrict__ vals32, double *__restrict__ vals64,
                       int32_t *__restrict__ src, int *nofit) {
    __shared__ int32_t s_c[kQ16FillWarps][32][kQ16StageW + 1];   // +1: a lane's walk down its row spreads over banks
    __shared__ double s_v[kQ16FillWarps][32][kQ16StageW + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t nwarps = (int64_t)gridDim.x * kQ16FillWarps;
    int32_t(*C)[kQ16StageW + 1] = s_c[w];
    double(*V)[kQ16StageW + 1] = s_v[w];
    for (int64_t k = (int64_t)blockIdx.x * kQ16FillWarps + w; k < nslices; k += nwarps) {
        const int64_t src0 = (int64_t)order[k] * 32;
        const int32_t row = sell_perm[src0 + lane];
        const int lraw = sell_len[src0 + lane];
        const int l = row >= 0 ? lraw : 0;
        const int wq = (__shfl_sync(0xffffffffu, l, 0) + 3) & ~3;   // SELL slices are sorted: lane 0 is the widest
        const int64_t r0 = row >= 0 ? (int64_t)rp[row] : 0;
        const int64_t b = (int64_t)sptr[k] + 4 * lane;
        int32_t b0 = 0, b1 = 0;
        int sp = 0;
        if (wq > kQ16StageW) {   // warp-uniform
            q16_row_direct(ci, va, r0, l, wq, b, b0, b1, sp, cols, vals32, vals64, src, nofit);
            if (l == 0) b0 = b1 = 0;
        } else {
            // stage: row t's entries, lanes along the row, as asynchronous
            // copies (every row's copies are in flight before any is waited for)
            for (int t = 0; t < 32; t++) {
                const int lt = __shfl_sync(0xffffffffu, l, t);
                const int64_t rt = __shfl_sync(0xffffffffu, r0, t);
#pragma unroll
                for (int m0 = 0; m0 < kQ16StageW; m0 += 32) {
                    const int m = m0 + lane;
                    if (m < lt) {
                        copy_async4(&C[t][m], &ci[rt + m]);
                        copy_async8(&V[t][m], &va[rt + m]);
                    }
                }
            }
            copy_async_wait_all();
            __syncwarp();
            const int32_t *c = C[lane];
            const double *v = V[lane];
            b0 = INT_MAX;
            for (int t = 0; t < l; t++) b0 = min(b0, c[t]);
            b1 = INT_MAX;
            int32_t hi = -1;
            for (int t = 0; t < l; t++) {
                const int32_t ct = c[t];
                if (ct - b0 < 65536) sp++;
                else {
                    b1 = min(b1, ct);
                    hi = max(hi, ct);
                }
            }
            if (hi < 0) b1 = b0;
            const bool fits = hi < 0 || hi - b1 < 65536;
            if (l > 0 && !fits) atomicExch(nofit, 1);
            if (l == 0) b0 = b1 = 0;
            // the row in layout order (first window, then the second, each in
            // CSR order), four entries per store, zeros past the row's end
            int t0 = 0, t1 = 0;   // cursors of the two windows' scans
            for (int jq = 0; jq < wq; jq += 4) {
                uint16_t cq[4];
                float fq[4];
                double dq[4];
                int32_t sq[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int jj = jq + u;
                    int t = -1;
                    bool w0 = true;
                    if (jj < sp) {
                        while (c[t0] - b0 >= 65536) t0++;
                        t = t0++;
                    } else if (jj < l) {
                        while (c[t1] - b0 < 65536) t1++;
                        t = t1++;
                        w0 = false;
                    }
                    if (t >= 0) {
                        cq[u] = fits ? (uint16_t)(c[t] - (w0 ? b0 : b1)) : (uint16_t)0;
                        dq[u] = v[t];
                        fq[u] = (float)v[t];
                        sq[u] = (int32_t)(r0 + t);
                    } else {
                        cq[u] = 0;
                        dq[u] = 0.0;
                        fq[u] = 0.0f;
                        sq[u] = -1;
                    }
                }
                const int64_t idx = b + (int64_t)(jq >> 2) * 128;
                *reinterpret_cast<uint2 *>(cols + idx) =
                    make_uint2((uint32_t)cq[0] | ((uint32_t)cq[1] << 16), (uint32_t)cq[2] | ((uint32_t)cq[3] << 16));
                *reinterpret_cast<float4 *>(vals32 + idx) = make_float4(fq[0], fq[1], fq[2], fq[3]);
                *reinterpret_cast<double2 *>(vals64 + idx) = make_double2(dq[0], dq[1]);
                *reinterpret_cast<double2 *>(vals64 + idx + 2) = make_double2(dq[2], dq[3]);
                *reinterpret_cast<int4 *>(src + idx) = make_int4(sq[0], sq[1], sq[2], sq[3]);
            }
            __syncwarp();   // the staging area is reused by the next slice
        }
        const int64_t pos = k * 32 + lane;
        perm[pos] = row;
        len[pos] = (uint16_t)lraw;
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
        float acc = 0.0f;   // products and sums rounded on their own, as the mixed solver's
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
        if (row >= 0) {
            const float yr = acc;
            y[row] = yr;
            if (DOT) dot += (double)x[row] * (double)yr;
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
    (void)npos;
    int64_t blocks = (nslices + kQ16FillWarps - 1) / kQ16FillWarps;
    if (blocks > 148 * 8) blocks = 148 * 8;
    q16_fill_staged_kernel<<<(unsigned)(blocks < 1 ? 1 : blocks), kQ16FillWarps * 32, 0, s>>>(
        nslices, rp, ci, va, sell_perm, sell_len, order, O.sptr, O.perm, O.len, O.split, O.base0, O.base1, O.cols,
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
