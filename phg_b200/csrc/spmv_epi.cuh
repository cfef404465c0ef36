// SpMV over the autotuned layout (CSR rows, SELL-C-sigma or q16 slices) with a
// per-row epilogue and a grid-wide reduction of two sums, for the Krylov
// solvers whose dot products follow a matrix-vector product (BiCGstab,
// GMRES).  An epilogue type E provides
//   bool skip() const                     the solver is done: return at once
//   void row(int64_t r, double acc, double &sa, double &sb) const
//                                         store (A x)_r = acc, add to the sums
//   void final(double sa, double sb) const  one thread, with the grid totals
//   double *partials; unsigned *ticket;   reduction workspace
#pragma once
#include "q16.cuh"
#include "reduce.cuh"
#include "solve.h"

namespace phgb {

constexpr int kEpiThreads = 256;

template <class E, int U>
__global__ void __launch_bounds__(kEpiThreads)
sell_epi_kernel(int64_t nslices, const int32_t *__restrict__ perm, const uint16_t *__restrict__ len,
                const int32_t *__restrict__ sptr, const int32_t *__restrict__ cols, const double *__restrict__ vals,
                const double *__restrict__ x, E epi) {
    if (epi.skip()) return;
    grid_sum_init();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kEpiThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kEpiThreads) >> 5;
    double sa = 0.0, sb = 0.0;
    for (int64_t s = warp; s < nslices; s += nwarps) {
        const int64_t pos = s * 32 + lane;
        const int32_t row = perm[pos];
        const int l = len[pos];
        const int wl = __shfl_sync(0xffffffffu, l, 0);
        const int64_t b = (int64_t)sptr[s] + lane;
        double acc = 0.0;
        for (int j = 0; j < wl; j += U) {
            int32_t c[U];
            double v[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const bool ok = j + u < l;
                c[u] = ok ? __ldcs(&cols[b + 32 * (j + u)]) : 0;
                v[u] = ok ? __ldcs(&vals[b + 32 * (j + u)]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; u++)
                if (j + u < l) acc += v[u] * __ldg(&x[c[u]]);
        }
        if (row >= 0) epi.row(row, acc, sa, sb);
    }
    if (grid_sum2(sa, sb, epi.partials, epi.ticket)) epi.final(sa, sb);
}

template <class E, int LPR>
__global__ void __launch_bounds__(kEpiThreads)
csr_epi_kernel(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
               const double *__restrict__ va, const double *__restrict__ x, E epi) {
    if (epi.skip()) return;
    grid_sum_init();
    const int lane = threadIdx.x % LPR;
    constexpr int RPW = 32 / LPR;
    const int64_t warp = ((int64_t)blockIdx.x * kEpiThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kEpiThreads) >> 5;
    const int sub = (threadIdx.x & 31) / LPR;
    double sa = 0.0, sb = 0.0;
    // uniform loop bound: every lane reaches the shuffles
    for (int64_t base = warp * RPW; base < n; base += nwarps * RPW) {
        const int64_t row = base + sub;
        double s = 0.0;
        if (row < n) {
            const int32_t b = rp[row], e = rp[row + 1];
            for (int32_t j = b + lane; j < e; j += LPR) s += va[j] * __ldg(&x[ci[j]]);
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LPR);
        if (lane == 0 && row < n) epi.row(row, s, sa, sb);
    }
    if (grid_sum2(sa, sb, epi.partials, epi.ticket)) epi.final(sa, sb);
}

template <class E>
__global__ void __launch_bounds__(kEpiThreads)
q16_epi_kernel(const Q16View Q, const double *__restrict__ x, E epi) {
    if (epi.skip()) return;
    grid_sum_init();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kEpiThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kEpiThreads) >> 5;
    double sa = 0.0, sb = 0.0;
    for (int64_t s = warp; s < Q.nslices; s += nwarps) {
        const int64_t pos = s * 32 + lane;
        const int32_t row = Q.perm[pos];
        const double acc = q16_row64(Q, s, lane, Q.len[pos], Q.split[pos], Q.base0[pos], Q.base1[pos], x);
        if (row >= 0) epi.row(row, acc, sa, sb);
    }
    if (grid_sum2(sa, sb, epi.partials, epi.ticket)) epi.final(sa, sb);
}

// Grid of an epilogue product: a grid-stride loop over slices or rows, so
// the grid is the blocks that are resident at once (at most 8 per SM; the
// epilogues differ in register use), no more than the work needs.
template <typename K>
inline int epi_grid(K kernel, int64_t threads) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kEpiThreads, 0) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 1;
    }
    per_sm = per_sm < 1 ? 1 : per_sm > 8 ? 8 : per_sm;
    int64_t b = ceil_div(threads, kEpiThreads);
    if (b > 148 * per_sm) b = 148 * per_sm;
    if (b < 1) b = 1;
    return (int)b;
}

// y = A x with epilogue `epi` on the plan's layout; the partials buffer
// needs 2 * 148 * 8 + 64 doubles.
template <class E>
void launch_spmv_epi(const SpmvPlan &P, const double *x, const E &epi, cudaStream_t s) {
    if (P.kind == SPMV_CSR) {
        const CsrView &A = P.csr;
        switch (P.lpr) {
        case 4: csr_epi_kernel<E, 4><<<epi_grid(csr_epi_kernel<E, 4>, A.n * 4), kEpiThreads, 0, s>>>(A.n, A.rp, A.ci, A.va, x, epi); break;
        case 8: csr_epi_kernel<E, 8><<<epi_grid(csr_epi_kernel<E, 8>, A.n * 8), kEpiThreads, 0, s>>>(A.n, A.rp, A.ci, A.va, x, epi); break;
        case 16: csr_epi_kernel<E, 16><<<epi_grid(csr_epi_kernel<E, 16>, A.n * 16), kEpiThreads, 0, s>>>(A.n, A.rp, A.ci, A.va, x, epi); break;
        default: csr_epi_kernel<E, 32><<<epi_grid(csr_epi_kernel<E, 32>, A.n * 32), kEpiThreads, 0, s>>>(A.n, A.rp, A.ci, A.va, x, epi); break;
        }
        return;
    }
    if (P.kind == SPMV_Q16) {
        q16_epi_kernel<E><<<epi_grid(q16_epi_kernel<E>, P.q16.nslices * 32), kEpiThreads, 0, s>>>(P.q16, x, epi);
        return;
    }
    const SellView &S = P.sell;
    const int64_t t = S.nslices * 32;
    switch (P.unroll) {
    case 2: sell_epi_kernel<E, 2><<<epi_grid(sell_epi_kernel<E, 2>, t), kEpiThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, S.vals, x, epi); break;
    case 8: sell_epi_kernel<E, 8><<<epi_grid(sell_epi_kernel<E, 8>, t), kEpiThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, S.vals, x, epi); break;
    default: sell_epi_kernel<E, 4><<<epi_grid(sell_epi_kernel<E, 4>, t), kEpiThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, S.vals, x, epi); break;
    }
}

}  // namespace phgb
