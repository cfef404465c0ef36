// Block Jacobi-PCG: many right-hand sides solved together.
//
// Every column runs the reference's PCG recurrence (solver-phg.c:485-604)
// with its own scalars and stopping rule; the columns share one sparse
// matrix-matrix product per iteration, so the matrix is read once per tile
// of columns instead of once per right-hand side.  Vectors are stored row
// major, X[i * K + k] (K = padded number of columns), so the lanes of a row
// group read consecutive columns of a gathered row of P.  SpMM mapping: a
// tile of T columns, L = min(T, 32) lanes per matrix row, T / L columns per
// lane, 32 / L rows per warp (T and the tile count are autotuned).
//
// Precision: FP64 throughout, or FP32 matrix values / Krylov vectors / SpMM
// with FP64-accumulated dot products and FP64 reliable updates of the
// solution and residual (as in the single right-hand-side mixed solver),
// applied to all columns at once when any column asks for one.
#include "common.cuh"
#include "block.h"

namespace phgb {

constexpr int kBT = 256;          // threads per block
constexpr int kBMaxBlocks = 148 * 4;

// ---------------------------------------------------------------------------
template <typename VT>
__global__ void __launch_bounds__(kBT)
bdir_kernel(BlockPtrs B, const VT *__restrict__ R, const VT *__restrict__ D, VT *__restrict__ P) {
    if (B.flags[0]) return;
    const int64_t total = B.n * B.K;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % B.K);
        if (B.done[k]) continue;
        const int64_t i = t / B.K;
        const VT z = R[t] / D[i];
        if (B.nits[k] == 0) {
            P[t] = z;
        } else {
            const double rp = B.rz_prev[k];
            const VT beta = (VT)(rp == 0.0 ? 0.0 : B.rz_cur[k] / rp);
            P[t] = beta * P[t] + z;
        }
    }
}

// AP = A P for one tile of T columns; per-column partial sums of p . Ap.
template <typename VT, int T>
__global__ void __launch_bounds__(kBT)
bspmm_kernel(BlockPtrs B, const VT *__restrict__ va, const VT *__restrict__ P, VT *__restrict__ AP) {
    if (B.flags[0]) return;
    constexpr int L = T < 32 ? T : 32;          // lanes per row
    constexpr int CPL = T / L;                  // columns per lane
    constexpr int RPW = 32 / L;                 // rows per warp
    __shared__ double s_dot[kBT / 32][T];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, sub = lane / L, gl = lane % L;
    const int tile = blockIdx.y;
    const int colbase = tile * T;
    const int K = B.K;
    const int64_t warp = (int64_t)blockIdx.x * (kBT / 32) + w;
    const int64_t nwarps = (int64_t)gridDim.x * (kBT / 32);
    double dot[CPL];
#pragma unroll
    for (int c = 0; c < CPL; c++) dot[c] = 0.0;
    for (int64_t base = warp * RPW; base < B.n; base += nwarps * RPW) {
        const int64_t row = base + sub;
        VT acc[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) acc[c] = (VT)0;
        int32_t b = 0, e = 0;
        if (row < B.n) { b = B.rp[row]; e = B.rp[row + 1]; }
        int maxlen = e - b;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
        for (int j0 = 0; j0 < maxlen; j0 += L) {
            int32_t cj = 0;
            VT vj = (VT)0;
            if (j0 + gl < e - b) { cj = __ldcs(&B.ci[b + j0 + gl]); vj = __ldcs(&va[b + j0 + gl]); }
            const int cnt = min(L, maxlen - j0);
            for (int t = 0; t < cnt; t++) {
                const int32_t c = __shfl_sync(0xffffffffu, cj, sub * L + t);
                const VT v = __shfl_sync(0xffffffffu, vj, sub * L + t);
                if (j0 + t < e - b) {
                    const VT *prow = P + (int64_t)c * K + colbase + gl;
#pragma unroll
                    for (int q = 0; q < CPL; q++) acc[q] += v * __ldg(&prow[q * L]);
                }
            }
        }
        if (row < B.n) {
#pragma unroll
            for (int q = 0; q < CPL; q++) {
                const int64_t idx = row * K + colbase + gl + q * L;
                AP[idx] = acc[q];
                dot[q] += (double)P[idx] * (double)acc[q];
            }
        }
    }
    // per-column block sums: lanes with the same gl (same columns) across
    // the rows of the warp, then across warps, in a fixed order
#pragma unroll
    for (int q = 0; q < CPL; q++) {
        double v = dot[q];
        for (int o = L; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (sub == 0) s_dot[w][gl + q * L] = v;
    }
    __syncthreads();
    double *part = B.partials + (size_t)tile * kBMaxBlocks * T;
    for (int c = threadIdx.x; c < T; c += blockDim.x) {
        double s = 0.0;
        for (int ww = 0; ww < kBT / 32; ww++) s += s_dot[ww][c];
        part[(size_t)blockIdx.x * T + c] = s;
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&B.tickets[tile], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int c = threadIdx.x; c < T; c += blockDim.x) {
        double s = 0.0;
        for (unsigned bb = 0; bb < gridDim.x; bb++) s += __ldcg(&part[(size_t)bb * T + c]);
        const int k = colbase + c;
        if (!B.done[k]) {
            B.pAp[k] = s;
            if (s == 0.0) {
                B.alpha[k] = 0.0;
                B.done[k] = 1;
                B.status[k] = 1;   // breakdown
                B.nits[k] += 1;
            } else {
                B.alpha[k] = B.rz_cur[k] / s;
            }
        }
    }
    if (threadIdx.x == 0) B.tickets[tile] = 0u;
}

// X += alpha P (or Y = [reset ? 0 : Y] + alpha P), R -= alpha AP; per-column
// ||r||^2 and r.(r/D); the last block closes the iteration of every column.
template <typename VT, typename XT, bool MIXED>
__global__ void __launch_bounds__(kBT)
bupdate_kernel(BlockPtrs B, XT *__restrict__ X, VT *__restrict__ R, const VT *__restrict__ P,
               const VT *__restrict__ AP, const VT *__restrict__ D) {
    if (B.flags[0]) return;
    const int K = B.K;
    const bool reset = MIXED && B.flags[3];
    // thread t handles column (t % K) for rows t / K, t / K + stride/K, ...
    // with blockDim a multiple of K every thread keeps one column
    double rr = 0.0, rz = 0.0;
    const int k = threadIdx.x % K;
    const bool active = !B.done[k];
    const double a = B.alpha[k];
    const int64_t rows_per_step = ((int64_t)gridDim.x * blockDim.x) / K;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / K; i < B.n; i += rows_per_step) {
        if (!active) break;
        const int64_t t = i * K + k;
        if (MIXED) X[t] = (reset ? (XT)0 : X[t]) + (XT)a * (XT)P[t];
        else X[t] += (XT)(a * (double)P[t]);
        const VT ri = R[t] - (VT)a * AP[t];
        R[t] = ri;
        rr += (double)ri * (double)ri;
        rz += (double)ri * (double)(ri / D[i]);
    }
    __shared__ double s_rr[kBT], s_rz[kBT];
    s_rr[threadIdx.x] = rr;
    s_rz[threadIdx.x] = rz;
    __syncthreads();
    double *part = B.partials + (size_t)kBMaxBlocks * 64 * 2;   // after the SpMM tiles
    for (int c = threadIdx.x; c < K; c += blockDim.x) {
        double a1 = 0.0, a2 = 0.0;
        for (int t = c; t < (int)blockDim.x; t += K) { a1 += s_rr[t]; a2 += s_rz[t]; }
        part[((size_t)blockIdx.x * K + c) * 2] = a1;
        part[((size_t)blockIdx.x * K + c) * 2 + 1] = a2;
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&B.tickets[64], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ int s_open, s_ru, s_final;
    if (threadIdx.x == 0) { s_open = 0; s_ru = 0; s_final = 0; }
    __syncthreads();
    for (int c = threadIdx.x; c < K; c += blockDim.x) {
        if (B.done[c]) continue;
        double a1 = 0.0, a2 = 0.0;
        for (unsigned bb = 0; bb < gridDim.x; bb++) {
            a1 += __ldcg(&part[((size_t)bb * K + c) * 2]);
            a2 += __ldcg(&part[((size_t)bb * K + c) * 2 + 1]);
        }
        const double res = sqrt(a1);
        const int it = B.nits[c] + 1;
        B.nits[c] = it;
        B.res[c] = res;
        B.rz_prev[c] = B.rz_cur[c];
        B.rz_cur[c] = a2;
        if (!isfinite(res)) {
            B.done[c] = 1;
            B.status[c] = 2;
        } else if (MIXED) {
            if (!(res > B.tol[c]) || it >= B.flags[4]) { atomicOr(&s_ru, 1); atomicOr(&s_final, 1); }
            else if (res < B.delta * B.maxr[c]) atomicOr(&s_ru, 1);
            atomicOr(&s_open, 1);
        } else {
            if (!(res > B.tol[c]) || it >= B.flags[4]) B.done[c] = 1;
            else atomicOr(&s_open, 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        B.tickets[64] = 0u;
        if (MIXED) {
            B.flags[3] = 0;
            if (s_ru) { B.flags[1] = 1; B.flags[2] = s_final; }
        }
        if (!s_open) B.flags[0] = 1;
    }
}

// Reliable update for all open columns: X += Y, Rt -= A Y (FP64 matrix),
// R32 = (float) Rt, per-column ||Rt||^2 and r32.(r32/D).
template <int T>
__global__ void __launch_bounds__(kBT)
breliable_kernel(BlockPtrs B, const double *__restrict__ va, double *__restrict__ X, const float *__restrict__ Y,
                 double *__restrict__ Rt, float *__restrict__ R32, const float *__restrict__ D) {
    if (B.flags[0] || !B.flags[1]) return;
    constexpr int L = T < 32 ? T : 32, CPL = T / L, RPW = 32 / L;
    __shared__ double s_a[kBT / 32][T], s_b[kBT / 32][T];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, sub = lane / L, gl = lane % L;
    const int tile = blockIdx.y, colbase = tile * T, K = B.K;
    const int64_t warp = (int64_t)blockIdx.x * (kBT / 32) + w;
    const int64_t nwarps = (int64_t)gridDim.x * (kBT / 32);
    double s1[CPL], s2[CPL];
#pragma unroll
    for (int q = 0; q < CPL; q++) s1[q] = s2[q] = 0.0;
    for (int64_t base = warp * RPW; base < B.n; base += nwarps * RPW) {
        const int64_t row = base + sub;
        double acc[CPL];
#pragma unroll
        for (int q = 0; q < CPL; q++) acc[q] = 0.0;
        int32_t b = 0, e = 0;
        if (row < B.n) { b = B.rp[row]; e = B.rp[row + 1]; }
        int maxlen = e - b;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
        for (int j0 = 0; j0 < maxlen; j0 += L) {
            int32_t cj = 0;
            double vj = 0.0;
            if (j0 + gl < e - b) { cj = B.ci[b + j0 + gl]; vj = va[b + j0 + gl]; }
            const int cnt = min(L, maxlen - j0);
            for (int t = 0; t < cnt; t++) {
                const int32_t c = __shfl_sync(0xffffffffu, cj, sub * L + t);
                const double v = __shfl_sync(0xffffffffu, vj, sub * L + t);
                if (j0 + t < e - b) {
                    const float *yrow = Y + (int64_t)c * K + colbase + gl;
#pragma unroll
                    for (int q = 0; q < CPL; q++) acc[q] += v * (double)__ldg(&yrow[q * L]);
                }
            }
        }
        if (row < B.n) {
#pragma unroll
            for (int q = 0; q < CPL; q++) {
                const int k = colbase + gl + q * L;
                if (B.done[k]) continue;
                const int64_t idx = row * K + k;
                X[idx] += (double)Y[idx];
                const double rt = Rt[idx] - acc[q];
                Rt[idx] = rt;
                const float rf = (float)rt;
                R32[idx] = rf;
                s1[q] += rt * rt;
                s2[q] += (double)rf * (double)(rf / D[row]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < CPL; q++) {
        double a = s1[q], c2 = s2[q];
        for (int o = L; o < 32; o <<= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            c2 += __shfl_xor_sync(0xffffffffu, c2, o);
        }
        if (sub == 0) { s_a[w][gl + q * L] = a; s_b[w][gl + q * L] = c2; }
    }
    __syncthreads();
    double *part = B.partials + (size_t)tile * kBMaxBlocks * T * 2;
    for (int c = threadIdx.x; c < T; c += blockDim.x) {
        double a = 0.0, c2 = 0.0;
        for (int ww = 0; ww < kBT / 32; ww++) { a += s_a[ww][c]; c2 += s_b[ww][c]; }
        part[((size_t)blockIdx.x * T + c) * 2] = a;
        part[((size_t)blockIdx.x * T + c) * 2 + 1] = c2;
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&B.tickets[65 + tile], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int c = threadIdx.x; c < T; c += blockDim.x) {
        const int k = colbase + c;
        if (B.done[k]) continue;
        double a = 0.0, c2 = 0.0;
        for (unsigned bb = 0; bb < gridDim.x; bb++) {
            a += __ldcg(&part[((size_t)bb * T + c) * 2]);
            c2 += __ldcg(&part[((size_t)bb * T + c) * 2 + 1]);
        }
        const double res = sqrt(a);
        B.res[k] = res;
        B.rz_cur[k] = c2;
        B.maxr[k] = res;
        if (B.flags[2] && (!(res > B.tol[k]) || B.nits[k] >= B.flags[4])) B.done[k] = 1;
    }
    if (threadIdx.x == 0) B.tickets[65 + tile] = 0u;
    // the tiles finish independently; the last tile to finish closes the update
    __shared__ bool lastTile;
    if (threadIdx.x == 0) {
        __threadfence();
        lastTile = atomicAdd(&B.tickets[130], 1u) == gridDim.y - 1;
    }
    __syncthreads();
    if (lastTile && threadIdx.x == 0) {
        B.tickets[130] = 0u;
        int open = 0;
        for (int k = 0; k < K; k++) open |= !B.done[k];
        B.flags[1] = 0;
        B.flags[2] = 0;
        B.flags[3] = 1;
        if (!open) B.flags[0] = 1;
    }
}

// ---------------------------------------------------------------------------
static int blocks_for(int64_t work) {
    int64_t b = (work + kBT - 1) / kBT;
    if (b > kBMaxBlocks) b = kBMaxBlocks;
    return (int)(b < 1 ? 1 : b);
}

template <typename VT>
static void spmm_launch(int T, const BlockPtrs &B, const VT *va, const VT *P, VT *AP, cudaStream_t s) {
    const int L = T < 32 ? T : 32;
    const dim3 grid(blocks_for(B.n * L), B.K / T);
    switch (T) {
    case 8: bspmm_kernel<VT, 8><<<grid, kBT, 0, s>>>(B, va, P, AP); break;
    case 16: bspmm_kernel<VT, 16><<<grid, kBT, 0, s>>>(B, va, P, AP); break;
    case 32: bspmm_kernel<VT, 32><<<grid, kBT, 0, s>>>(B, va, P, AP); break;
    default: bspmm_kernel<VT, 64><<<grid, kBT, 0, s>>>(B, va, P, AP); break;
    }
}

cudaError_t launch_block_iteration(const BlockPtrs &B, int T, bool mixed, const BlockVecs &V, cudaStream_t s) {
    const int vb = blocks_for(B.n * B.K);
    // update kernel: blockDim must be a multiple of K
    const int ub = blocks_for(B.n * B.K);
    if (!mixed) {
        bdir_kernel<double><<<vb, kBT, 0, s>>>(B, V.R, V.D, V.P);
        spmm_launch<double>(T, B, V.va, V.P, V.AP, s);
        bupdate_kernel<double, double, false><<<ub, kBT, 0, s>>>(B, V.X, V.R, V.P, V.AP, V.D);
    } else {
        bdir_kernel<float><<<vb, kBT, 0, s>>>(B, V.R32, V.D32, V.P32);
        spmm_launch<float>(T, B, V.va32, V.P32, V.AP32, s);
        bupdate_kernel<float, float, true><<<ub, kBT, 0, s>>>(B, V.Y32, V.R32, V.P32, V.AP32, V.D32);
        const int L = T < 32 ? T : 32;
        const dim3 grid(blocks_for(B.n * L), B.K / T);
        switch (T) {
        case 8: breliable_kernel<8><<<grid, kBT, 0, s>>>(B, V.va, V.X, V.Y32, V.R, V.R32, V.D32); break;
        case 16: breliable_kernel<16><<<grid, kBT, 0, s>>>(B, V.va, V.X, V.Y32, V.R, V.R32, V.D32); break;
        case 32: breliable_kernel<32><<<grid, kBT, 0, s>>>(B, V.va, V.X, V.Y32, V.R, V.R32, V.D32); break;
        default: breliable_kernel<64><<<grid, kBT, 0, s>>>(B, V.va, V.X, V.Y32, V.R, V.R32, V.D32); break;
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_block_spmm64(const BlockPtrs &B, int T, const double *va, const double *P, double *AP,
                                cudaStream_t s) {
    spmm_launch<double>(T, B, va, P, AP, s);
    return cudaGetLastError();
}

cudaError_t launch_block_spmm32(const BlockPtrs &B, int T, const float *va, const float *P, float *AP,
                                cudaStream_t s) {
    spmm_launch<float>(T, B, va, P, AP, s);
    return cudaGetLastError();
}

size_t block_partials_doubles() { return (size_t)kBMaxBlocks * 64 * 2 * 2 + 64; }
size_t block_ticket_count() { return 131; }

// Initial state of every column from R (= B - A X0, FP64): tolerance
// rtol * ||r0||, r.(r/D), and for the mixed solver the FP32 copies.
template <bool MIXED>
__global__ void __launch_bounds__(kBT)
binit_kernel(BlockPtrs B, const double *__restrict__ R, const double *__restrict__ D, float *__restrict__ R32,
             float *__restrict__ D32, float *__restrict__ Y32, double rtol) {
    const int K = B.K;
    const int k = threadIdx.x % K;
    const int64_t rows_per_step = ((int64_t)gridDim.x * blockDim.x) / K;
    double rr = 0.0, rz = 0.0;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / K; i < B.n; i += rows_per_step) {
        const int64_t t = i * K + k;
        const double r = R[t];
        if (MIXED) {
            const float rf = (float)r, df = (float)D[i];
            R32[t] = rf;
            Y32[t] = 0.0f;
            if (k == 0) D32[i] = df;
            rr += r * r;
            rz += (double)rf * (double)(rf / df);
        } else {
            rr += r * r;
            rz += r * (r / D[i]);
        }
    }
    __shared__ double s_rr[kBT], s_rz[kBT];
    s_rr[threadIdx.x] = rr;
    s_rz[threadIdx.x] = rz;
    __syncthreads();
    double *part = B.partials + (size_t)kBMaxBlocks * 64 * 2;
    for (int c = threadIdx.x; c < K; c += blockDim.x) {
        double a1 = 0.0, a2 = 0.0;
        for (int t = c; t < (int)blockDim.x; t += K) { a1 += s_rr[t]; a2 += s_rz[t]; }
        part[((size_t)blockIdx.x * K + c) * 2] = a1;
        part[((size_t)blockIdx.x * K + c) * 2 + 1] = a2;
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&B.tickets[64], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int c = threadIdx.x; c < K; c += blockDim.x) {
        double a1 = 0.0, a2 = 0.0;
        for (unsigned bb = 0; bb < gridDim.x; bb++) {
            a1 += __ldcg(&part[((size_t)bb * K + c) * 2]);
            a2 += __ldcg(&part[((size_t)bb * K + c) * 2 + 1]);
        }
        const double r0 = sqrt(a1);
        B.res[c] = r0;
        B.maxr[c] = r0;
        B.tol[c] = r0 * rtol;
        B.rz_cur[c] = a2;
        B.rz_prev[c] = 0.0;
        B.nits[c] = 0;
        B.status[c] = 0;
        B.done[c] = !(r0 > r0 * rtol) || B.flags[4] <= 0 || !isfinite(a2);
        if (!isfinite(a2)) B.status[c] = 2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        B.tickets[64] = 0u;
        int open = 0;
        for (int c = 0; c < K; c++) open |= !B.done[c];
        B.flags[0] = !open;
        B.flags[1] = 0;
        B.flags[2] = 0;
        B.flags[3] = 1;
    }
}

cudaError_t launch_block_init(const BlockPtrs &B, bool mixed, const double *R, const double *D, float *R32,
                              float *D32, float *Y32, double rtol, cudaStream_t s) {
    const int nb = blocks_for(B.n * B.K);
    if (mixed) binit_kernel<true><<<nb, kBT, 0, s>>>(B, R, D, R32, D32, Y32, rtol);
    else binit_kernel<false><<<nb, kBT, 0, s>>>(B, R, D, R32, D32, Y32, rtol);
    return cudaGetLastError();
}

// R[i*K + k] = k < m ? Bin[i*m + k] : 0  (and the reverse for the output)
__global__ void pack_kernel(int64_t n, int m, int K, const double *__restrict__ in, double *__restrict__ out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % K);
        out[t] = k < m ? in[(t / K) * m + k] : 0.0;
    }
}
__global__ void unpack_kernel(int64_t n, int m, int K, const double *__restrict__ in, double *__restrict__ out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n * m; t += (int64_t)gridDim.x * blockDim.x)
        out[t] = in[(t / m) * K + t % m];
}
__global__ void sub_kernel(int64_t total, const double *__restrict__ a, double *__restrict__ b) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x)
        b[t] = a[t] - b[t];
}
__global__ void to_float_kernel(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        b[t] = (float)a[t];
}

cudaError_t launch_block_pack(int64_t n, int m, int K, const double *in, double *out, cudaStream_t s) {
    pack_kernel<<<blocks_for(n * K), kBT, 0, s>>>(n, m, K, in, out);
    return cudaGetLastError();
}
cudaError_t launch_block_unpack(int64_t n, int m, int K, const double *in, double *out, cudaStream_t s) {
    unpack_kernel<<<blocks_for(n * m), kBT, 0, s>>>(n, m, K, in, out);
    return cudaGetLastError();
}
cudaError_t launch_block_sub(int64_t total, const double *a, double *b, cudaStream_t s) {
    sub_kernel<<<blocks_for(total), kBT, 0, s>>>(total, a, b);
    return cudaGetLastError();
}
cudaError_t launch_to_float(int64_t n, const double *a, float *b, cudaStream_t s) {
    to_float_kernel<<<blocks_for(n), kBT, 0, s>>>(n, a, b);
    return cudaGetLastError();
}

}  // namespace phgb
