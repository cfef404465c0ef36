// Sparse matrix-vector product and the Jacobi-PCG iteration on the device.
//
// One PCG iteration (solver_pcg, solver-phg.c:535-590) is three kernels:
//   dir     p = z + beta p, z = r / diag           (jacobi_pc + phgVecAXPBY)
//   spmv    Ap = A p, and p.Ap                      (phgMatVec + phgVecDot)
//   update  x += alpha p, r -= alpha Ap, ||r||^2 and r.z for the next step
// The scalars of the recurrence live in a device-resident state block; each
// reduction finishes in the last block to arrive (a ticket counter, no
// waiting), summing the per-block partials in block order so that results do
// not depend on scheduling.  Every kernel first checks the state's `done`
// flag, so a captured graph of many iterations turns into no-ops once the
// stopping rule of the reference (||r|| <= tol or nits == maxit) is met.
#include "common.cuh"
#include "pcg_final.cuh"
#include "q16.h"
#include "reduce.cuh"
#include "solve.h"

#include <math.h>

namespace phgb {


// ---------------------------------------------------------------------------
// SpMV: LPR lanes per row (CSR vector form).  With DOT, also p.y -> state.
template <int LPR, bool DOT, typename VT>
__global__ void __launch_bounds__(kVecThreads, kResidentBlocks)
spmv_kernel(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
            const VT *__restrict__ va, const VT *__restrict__ x, VT *__restrict__ y,
            double *partials, PcgState *st) {
    if (DOT && st->done) return;
    if (DOT) grid_sum_init();
    const int lane = threadIdx.x % LPR;
    constexpr int RPW = 32 / LPR;   // rows per warp per step
    const int64_t warp = ((int64_t)blockIdx.x * kVecThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kVecThreads) >> 5;
    const int sub = (threadIdx.x & 31) / LPR;
    double dot = 0.0, dummy = 0.0;
    // the loop bound is uniform across the warp so every lane reaches the
    // shuffles below
    for (int64_t base = warp * RPW; base < n; base += nwarps * RPW) {
        const int64_t row = base + sub;
        double s = 0.0;
        if (row < n) {
            const int32_t b = rp[row], e = rp[row + 1];
            for (int32_t j = b + lane; j < e; j += LPR) s += (double)va[j] * (double)__ldg(&x[ci[j]]);
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LPR);
        if (lane == 0 && row < n) {
            y[row] = (VT)s;
            if (DOT) dot += (double)x[row] * (double)(VT)s;
        }
    }
    if (!DOT) return;
    if (grid_sum2(dot, dummy, partials, st->ticket)) pcg_pap_final(dot, st);
}

// p = r / D (first iteration) or p = z + beta p; 16-byte vectors of rows.
template <typename VT>
__global__ void __launch_bounds__(kVecThreads)
pcg_dir_kernel(int64_t n, const VT *__restrict__ r, const VT *__restrict__ dinv_or_d, VT *__restrict__ p,
               PcgState *st) {
    if (st->done) return;
    const int k = st->nits + 1;
    double beta = 0.0;
    if (k > 1) {
        if (st->rz_prev == 0.0) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                st->done = 1;
                st->status = PCG_BREAKDOWN;
                st->nits = k;
            }
            return;
        }
        beta = st->rz_cur / st->rz_prev;
    }
    const VT vb = (VT)beta;
    constexpr int V = Vec16<VT>::V, UN = 2;   // UN vectors per thread in flight
    const int nfull = aligned16(r, dinv_or_d, p) ? (int)(n / V) : 0;   // n < 2^31
    const int stride = gridDim.x * blockDim.x;
    for (int c0 = blockIdx.x * blockDim.x + threadIdx.x; c0 < nfull; c0 += UN * stride) {
        VArr<VT> rr[UN], dd[UN], pp[UN];
#pragma unroll
        for (int u = 0; u < UN; u++) {
            const int c = c0 + u * stride;
            if (c < nfull) {
                rr[u] = vload_ro(r + c * V);
                dd[u] = vload_ro(dinv_or_d + c * V);
                if (k > 1) pp[u] = vload(p + c * V);
            }
        }
#pragma unroll
        for (int u = 0; u < UN; u++) {
            const int c = c0 + u * stride;
            if (c < nfull) {
#pragma unroll
                for (int q = 0; q < V; q++)
                    pp[u].v[q] = k == 1 ? rr[u].v[q] / dd[u].v[q] : vb * pp[u].v[q] + rr[u].v[q] / dd[u].v[q];
                vstore(p + c * V, pp[u]);
            }
        }
    }
    for (int64_t i = nfull * V + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const VT z = r[i] / dinv_or_d[i];
        p[i] = k == 1 ? z : vb * p[i] + z;
    }
}

// x += alpha p, r -= alpha Ap; sums ||r||^2 and r.(r/D); closes the iteration.
// Each thread handles 16-byte vectors of consecutive rows.
template <typename VT, typename XT>
__global__ void __launch_bounds__(kVecThreads)
pcg_update_kernel(int64_t n, XT *__restrict__ x, VT *__restrict__ r, const VT *__restrict__ p,
                  const VT *__restrict__ Ap, const VT *__restrict__ D, double *partials, PcgState *st,
                  double *hist) {
    if (st->done) return;
    grid_sum_init();
    const double alpha = st->alpha;
    const VT va = (VT)alpha;
    double rr = 0.0, rz = 0.0;
    constexpr int V = Vec16<VT>::V, UN = 2;   // UN vectors per thread in flight
    const int nfull = aligned16(x, r, p, Ap, D) ? (int)(n / V) : 0;   // n < 2^31
    const int stride = gridDim.x * blockDim.x;
    for (int c0 = blockIdx.x * blockDim.x + threadIdx.x; c0 < nfull; c0 += UN * stride) {
        VArr<VT> pp[UN], aa[UN], dd[UN], rv[UN];
        VArr<XT> xv[UN];
#pragma unroll
        for (int u = 0; u < UN; u++) {
            const int c = c0 + u * stride;
            if (c < nfull) {
                const int i = c * V;
                pp[u] = vload_ro(p + i);
                aa[u] = vload_ro(Ap + i);
                dd[u] = vload_ro(D + i);
                rv[u] = vload(r + i);
                xv[u] = vload(x + i);
            }
        }
#pragma unroll
        for (int u = 0; u < UN; u++) {
            const int c = c0 + u * stride;
            if (c < nfull) {
#pragma unroll
                for (int q = 0; q < V; q++) {
                    xv[u].v[q] += (XT)(alpha * (double)pp[u].v[q]);
                    const VT ri = rv[u].v[q] - va * aa[u].v[q];
                    rv[u].v[q] = ri;
                    const double rd = (double)ri;
                    rr += rd * rd;
                    rz += rd * (double)(ri / dd[u].v[q]);
                }
                vstore(r + c * V, rv[u]);
                vstore(x + c * V, xv[u]);
            }
        }
    }
    for (int64_t i = nfull * V + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += (XT)(alpha * (double)p[i]);
        const VT ri = r[i] - va * Ap[i];
        r[i] = ri;
        const double rd = (double)ri;
        rr += rd * rd;
        rz += rd * (double)(ri / D[i]);
    }
    if (grid_sum2(rr, rz, partials, st->ticket)) {
        const int k = st->nits + 1;
        const double res = sqrt(rr);
        st->nits = k;
        st->residual = res;
        st->rz_prev = st->rz_cur;
        st->rz_cur = rz;
        if (hist != nullptr) hist[k] = res;
        if (!isfinite(res)) {
            st->done = 1;
            st->status = PCG_NONFINITE;
        } else if (!(res > st->tol) || k >= st->maxit) {
            st->done = 1;
        }
    }
}

// Sums (|x|_1, ||b||^2) or (||r||^2, r.(r/D)) for the solver's start.
template <typename VT, typename XT>
__global__ void __launch_bounds__(kVecThreads)
init_sums_kernel(int64_t n, int mode, const XT *__restrict__ x, const VT *__restrict__ b,
                 const VT *__restrict__ D, double *partials, unsigned *ticket, double *out) {
    grid_sum_init();
    double s0 = 0.0, s1 = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double bi = (double)b[i];
        if (mode == 0) {
            s0 += fabs((double)x[i]);
            s1 += bi * bi;
        } else {
            s0 += bi * bi;
            s1 += bi * (double)(b[i] / D[i]);
        }
    }
    if (grid_sum2(s0, s1, partials, ticket)) { out[0] = s0; out[1] = s1; }
}

// r = b - y  (y = A x)
template <typename VT>
__global__ void residual_kernel(int64_t n, const VT *__restrict__ b, const VT *__restrict__ y, VT *__restrict__ r) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - y[i];
}

// ---------------------------------------------------------------------------
static_assert(148 * 8 <= kRedMaxBlocks, "grids of reducing kernels must fit the grid-sum workspace");

int vec_blocks(int64_t n) {
    int64_t b = ceil_div(n, kVecThreads);
    if (b > kVecMaxBlocks) b = kVecMaxBlocks;
    if (b < 1) b = 1;
    return (int)b;
}

// Grid of the vectorised element-wise kernels: 16-byte vectors, two per
// thread and step, at most 3 blocks per SM (all resident at once with up to
// 80 registers per thread; fewer partial sums to combine).
static int vvec_blocks(int64_t n, int V) {
    int64_t b = ceil_div(ceil_div(n, 2 * V), kVecThreads);
    if (b > 148 * 3) b = 148 * 3;
    if (b < 1) b = 1;
    return (int)b;
}

int spmv_lanes_for(double avg_nnz_per_row) {
    if (avg_nnz_per_row <= 6) return 4;
    if (avg_nnz_per_row <= 16) return 8;
    if (avg_nnz_per_row <= 40) return 16;
    return 32;
}

template <bool DOT, typename VT>
static void spmv_dispatch(int lpr, int64_t n, const int32_t *rp, const int32_t *ci, const VT *va, const VT *x,
                          VT *y, double *partials, PcgState *st, cudaStream_t s) {
    const int blocks = vec_blocks(n * lpr);
    switch (lpr) {
    case 4: spmv_kernel<4, DOT, VT><<<blocks, kVecThreads, 0, s>>>(n, rp, ci, va, x, y, partials, st); break;
    case 8: spmv_kernel<8, DOT, VT><<<blocks, kVecThreads, 0, s>>>(n, rp, ci, va, x, y, partials, st); break;
    case 16: spmv_kernel<16, DOT, VT><<<blocks, kVecThreads, 0, s>>>(n, rp, ci, va, x, y, partials, st); break;
    default: spmv_kernel<32, DOT, VT><<<blocks, kVecThreads, 0, s>>>(n, rp, ci, va, x, y, partials, st); break;
    }
}

cudaError_t launch_spmv(const CsrView &A, int lpr, const double *x, double *y, cudaStream_t s) {
    spmv_dispatch<false, double>(lpr, A.n, A.rp, A.ci, A.va, x, y, nullptr, nullptr, s);
    return cudaGetLastError();
}

cudaError_t launch_pcg_iteration(const PcgBuffers &B, int lpr, cudaStream_t s) {
    const int vb = vvec_blocks(B.A.n, 2);
    pcg_dir_kernel<double><<<vb, kVecThreads, 0, s>>>(B.A.n, B.r, B.D, B.p, B.st);
    spmv_dispatch<true, double>(lpr, B.A.n, B.A.rp, B.A.ci, B.A.va, B.p, B.Ap, B.partials, B.st, s);
    pcg_update_kernel<double, double><<<vb, kVecThreads, 0, s>>>(B.A.n, B.x, B.r, B.p, B.Ap, B.D, B.partials,
                                                                B.st, B.hist);
    return cudaGetLastError();
}

cudaError_t launch_init_sums(int64_t n, int mode, const double *x, const double *b, const double *D,
                             double *partials, unsigned *ticket, double *out, cudaStream_t s) {
    init_sums_kernel<double, double><<<vec_blocks(n), kVecThreads, 0, s>>>(n, mode, x, b, D, partials, ticket, out);
    return cudaGetLastError();
}

cudaError_t launch_residual(int64_t n, const double *b, const double *y, double *r, cudaStream_t s) {
    residual_kernel<double><<<vec_blocks(n), kVecThreads, 0, s>>>(n, b, y, r);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// SELL-C-sigma layout (C = 32 rows per slice, rows sorted by length inside
// windows of sigma = 256 rows).  Slice s stores entry j of its lane l at
// sptr[s] + 32 j + l: a warp reads 32 consecutive values (one 256-byte
// stream for FP64) per step, one thread per row, no shuffles.  Each thread
// stops at its own row length, so the padding is never read.
constexpr int kSellWin = 256;

__global__ void __launch_bounds__(kSellWin)
sell_sort_kernel(int64_t n, const int32_t *__restrict__ rp, int32_t *__restrict__ perm,
                 uint16_t *__restrict__ len, int32_t *__restrict__ slice_size) {
    __shared__ int32_t key[kSellWin];
    const int i = threadIdx.x;
    const int64_t base = (int64_t)blockIdx.x * kSellWin, row = base + i;
    const int32_t l = row < n ? rp[row + 1] - rp[row] : 0;
    key[i] = l * kSellWin + (kSellWin - 1 - i);   // unique; descending = long rows first, then row order
    __syncthreads();
    // bitonic sort, descending
    for (int k = 2; k <= kSellWin; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int p = i ^ j;
            if (p > i) {
                const bool desc = (i & k) == 0;
                const int32_t a = key[i], b = key[p];
                if (desc ? (a < b) : (a > b)) { key[i] = b; key[p] = a; }
            }
            __syncthreads();
        }
    }
    const int32_t kk = key[i];
    const int src = kSellWin - 1 - (kk % kSellWin);
    const int32_t li = kk / kSellWin;
    perm[base + i] = base + src < n ? (int32_t)(base + src) : -1;
    len[base + i] = (uint16_t)li;
    if ((i & 31) == 0) slice_size[(base + i) >> 5] = 32 * li;   // the slice's first row is its longest
}

template <typename VT>
__global__ void sell_fill_kernel(int64_t npos, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                 const double *__restrict__ va, const int32_t *__restrict__ perm,
                                 const uint16_t *__restrict__ len, const int32_t *__restrict__ sptr,
                                 int32_t *__restrict__ cols, VT *__restrict__ vals, float *__restrict__ vals32) {
    for (int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < npos;
         pos += (int64_t)gridDim.x * blockDim.x) {
        const int32_t row = perm[pos];
        if (row < 0) continue;
        const int l = len[pos];
        const int64_t b = (int64_t)sptr[pos >> 5] + (pos & 31);
        const int32_t r0 = rp[row];
        for (int j = 0; j < l; j++) {
            cols[b + 32 * j] = ci[r0 + j];
            const double v = va[r0 + j];
            vals[b + 32 * j] = (VT)v;
            if (vals32 != nullptr) vals32[b + 32 * j] = (float)v;
        }
    }
}

template <typename VT, bool DOT, int U>
__global__ void __launch_bounds__(kVecThreads, kResidentBlocks)
sell_spmv_kernel(int64_t nslices, const int32_t *__restrict__ perm, const uint16_t *__restrict__ len,
                 const int32_t *__restrict__ sptr, const int32_t *__restrict__ cols, const VT *__restrict__ vals,
                 const VT *__restrict__ x, VT *__restrict__ y, double *partials, PcgState *st) {
    if (DOT && st->done) return;
    if (DOT) grid_sum_init();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kVecThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kVecThreads) >> 5;
    double dot = 0.0, dummy = 0.0;
    for (int64_t s = warp; s < nslices; s += nwarps) {
        const int64_t pos = s * 32 + lane;
        const int32_t row = perm[pos];
        const int l = len[pos];
        const int w = __shfl_sync(0xffffffffu, l, 0);
        const int64_t b = (int64_t)sptr[s] + lane;
        VT acc = (VT)0;   // FP32: products and sums rounded on their own; FP64 in FP64
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
                    if constexpr (sizeof(VT) == 4) acc = fma_free(acc, v[u], __ldg(&x[c[u]]));
                    else acc += v[u] * __ldg(&x[c[u]]);
                }
        }
        if (row >= 0) {
            y[row] = (VT)acc;
            if (DOT) dot += (double)x[row] * (double)(VT)acc;
        }
    }
    if (!DOT) return;
    if (grid_sum2(dot, dummy, partials, st->ticket)) pcg_pap_final(dot, st);
}

int64_t sell_positions(int64_t n) { return ceil_div(n, kSellWin) * kSellWin; }

cudaError_t launch_sell_sort(int64_t n, const int32_t *rp, int32_t *perm, uint16_t *len, int32_t *slice_size,
                             cudaStream_t s) {
    sell_sort_kernel<<<(unsigned)ceil_div(n, kSellWin), kSellWin, 0, s>>>(n, rp, perm, len, slice_size);
    return cudaGetLastError();
}

cudaError_t launch_sell_fill(int64_t n, const int32_t *rp, const int32_t *ci, const double *va, const int32_t *perm,
                             const uint16_t *len, const int32_t *sptr, int32_t *cols, double *vals, float *vals32,
                             cudaStream_t s) {
    const int64_t npos = sell_positions(n);
    sell_fill_kernel<double><<<vec_blocks(npos), kVecThreads, 0, s>>>(npos, rp, ci, va, perm, len, sptr, cols,
                                                                      vals, vals32);
    return cudaGetLastError();
}

template <bool DOT, typename VT>
static void plan_spmv(const SpmvPlan &P, const VT *vals, const VT *x, VT *y, double *partials, PcgState *st,
                      cudaStream_t s) {
    if (P.kind == SPMV_CSR) {
        spmv_dispatch<DOT, VT>(P.lpr, P.csr.n, P.csr.rp, P.csr.ci, vals, x, y, partials, st, s);
        return;
    }
    const SellView &S = P.sell;
    const int blocks = vec_blocks(S.nslices * 32);
    switch (P.unroll) {
    case 2: sell_spmv_kernel<VT, DOT, 2><<<blocks, kVecThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, vals, x, y, partials, st); break;
    case 8: sell_spmv_kernel<VT, DOT, 8><<<blocks, kVecThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, vals, x, y, partials, st); break;
    default: sell_spmv_kernel<VT, DOT, 4><<<blocks, kVecThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, vals, x, y, partials, st); break;
    }
}

cudaError_t launch_spmv_plan(const SpmvPlan &P, const double *x, double *y, cudaStream_t s) {
    if (P.kind == SPMV_Q16) return launch_q16_spmv64(P.q16, x, y, s);
    plan_spmv<false, double>(P, P.kind == SPMV_CSR ? P.csr.va : P.sell.vals, x, y, nullptr, nullptr, s);
    return cudaGetLastError();
}

cudaError_t launch_pcg_iteration_plan(const PcgBuffers &B, const SpmvPlan &P, cudaStream_t s) {
    const int vb = vvec_blocks(B.A.n, 2);
    pcg_dir_kernel<double><<<vb, kVecThreads, 0, s>>>(B.A.n, B.r, B.D, B.p, B.st);
    if (P.kind == SPMV_Q16) {
        const cudaError_t e = launch_q16_spmv64_dot(P.q16, B.p, B.Ap, B.partials, B.st, s);
        if (e != cudaSuccess) return e;
    } else {
        plan_spmv<true, double>(P, P.kind == SPMV_CSR ? P.csr.va : P.sell.vals, B.p, B.Ap, B.partials, B.st, s);
    }
    pcg_update_kernel<double, double><<<vb, kVecThreads, 0, s>>>(B.A.n, B.x, B.r, B.p, B.Ap, B.D, B.partials,
                                                                B.st, B.hist);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FP32 values in "pair" SELL: the same slices as SELL-C-sigma, but each lane
// keeps two consecutive entries of its row side by side, so a warp moves
// 256 bytes of values and 256 bytes of column indices per load instruction
// (float2 / int2).  Slice s holds ceil(w_s / 2) pairs of 64 entries.  The
// slices are stored widest first (order[k] = SELL slice stored k-th): warps
// take slices k, k + nwarps, ..., so every warp gets a similar share of the
// work and no long slices are left for the end of the launch.
__global__ void sell2_heads_kernel(int64_t nslices, const uint16_t *__restrict__ len, uint16_t *__restrict__ width) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nslices; s += (int64_t)gridDim.x * blockDim.x)
        width[s] = len[s * 32];   // rows are sorted by length: position 0 is the slice's widest
}

__global__ void sell2_sizes_kernel(int64_t nslices, const uint16_t *__restrict__ len, const int32_t *__restrict__ order,
                                   int32_t *__restrict__ size) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nslices; k += (int64_t)gridDim.x * blockDim.x)
        size[k] = 64 * ((len[(int64_t)order[k] * 32] + 1) / 2);
}

__global__ void sell2_fill_kernel(int64_t npos, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                                  const double *__restrict__ va, const int32_t *__restrict__ perm,
                                  const uint16_t *__restrict__ len, const int32_t *__restrict__ order,
                                  const int32_t *__restrict__ sptr2, int32_t *__restrict__ perm2,
                                  uint16_t *__restrict__ len2, int32_t *__restrict__ cols2, float *__restrict__ vals2) {
    for (int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < npos;
         pos += (int64_t)gridDim.x * blockDim.x) {
        const int64_t src = (int64_t)order[pos >> 5] * 32 + (pos & 31);
        const int32_t row = perm[src];
        const int l = len[src];
        perm2[pos] = row;
        len2[pos] = (uint16_t)l;
        const int64_t b = (int64_t)sptr2[pos >> 5] + 2 * (pos & 31);
        const int32_t r0 = row >= 0 ? rp[row] : 0;
        const int lp = (l + 1) & ~1;
        for (int j = 0; j < lp; j++) {
            const int64_t idx = b + (int64_t)(j >> 1) * 64 + (j & 1);
            if (j < l) {
                cols2[idx] = ci[r0 + j];
                vals2[idx] = (float)va[r0 + j];
            } else {   // odd-length row: a harmless pad (never added)
                cols2[idx] = 0;
                vals2[idx] = 0.0f;
            }
        }
    }
}

template <bool DOT, int U>
__global__ void __launch_bounds__(kVecThreads, kResidentBlocks)
sell2_spmv_kernel(int64_t nslices, const int32_t *__restrict__ perm, const uint16_t *__restrict__ len,
                  const int32_t *__restrict__ sptr2, const int32_t *__restrict__ cols2,
                  const float *__restrict__ vals2, const float *__restrict__ x, float *__restrict__ y,
                  double *partials, PcgState *st) {
    if (DOT && st->done) return;
    if (DOT) grid_sum_init();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kVecThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kVecThreads) >> 5;
    double dot = 0.0, dummy = 0.0;
    for (int64_t s = warp; s < nslices; s += nwarps) {
        const int64_t pos = s * 32 + lane;
        const int32_t row = perm[pos];
        const int l = len[pos];
        const int wp = (__shfl_sync(0xffffffffu, l, 0) + 1) >> 1;
        const int2 *cp = reinterpret_cast<const int2 *>(cols2 + sptr2[s]) + lane;
        const float2 *vp = reinterpret_cast<const float2 *>(vals2 + sptr2[s]) + lane;
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
        if (row >= 0) {
            const float yr = acc;
            y[row] = yr;
            if (DOT) dot += (double)x[row] * (double)yr;
        }
    }
    if (!DOT) return;
    if (grid_sum2(dot, dummy, partials, st->ticket)) pcg_pap_final(dot, st);
}

cudaError_t launch_sell2_heads(const SellView &S, uint16_t *width, cudaStream_t s) {
    sell2_heads_kernel<<<vec_blocks(S.nslices), kVecThreads, 0, s>>>(S.nslices, S.len, width);
    return cudaGetLastError();
}

cudaError_t launch_sell2_sizes(const SellView &S, const int32_t *order, int32_t *sizes, cudaStream_t s) {
    sell2_sizes_kernel<<<vec_blocks(S.nslices), kVecThreads, 0, s>>>(S.nslices, S.len, order, sizes);
    return cudaGetLastError();
}

cudaError_t launch_sell2_fill(const SellView &S, const int32_t *rp, const int32_t *ci, const double *va,
                              const int32_t *order, const int32_t *sptr2, int32_t *perm2, uint16_t *len2,
                              int32_t *cols2, float *vals2, cudaStream_t s) {
    const int64_t npos = S.nslices * 32;
    sell2_fill_kernel<<<vec_blocks(npos), kVecThreads, 0, s>>>(npos, rp, ci, va, S.perm, S.len, order, sptr2, perm2,
                                                               len2, cols2, vals2);
    return cudaGetLastError();
}

// FP32 product for the mixed solver: kind 0 = SELL (unroll u), 1 = pair SELL (unroll u pairs)
template <bool DOT>
static void spmv32_dispatch(const SellView &S, const Sell2View &S2, int kind, int u, const float *x, float *y,
                            double *partials, PcgState *st, cudaStream_t s) {
    const int sb = vec_blocks(S.nslices * 32);
    if (kind == 0) {
        switch (u) {
        case 2: sell_spmv_kernel<float, DOT, 2><<<sb, kVecThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, S.vals32, x, y, partials, st); break;
        case 8: sell_spmv_kernel<float, DOT, 8><<<sb, kVecThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, S.vals32, x, y, partials, st); break;
        case 16: sell_spmv_kernel<float, DOT, 16><<<sb, kVecThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, S.vals32, x, y, partials, st); break;
        default: sell_spmv_kernel<float, DOT, 4><<<sb, kVecThreads, 0, s>>>(S.nslices, S.perm, S.len, S.sptr, S.cols, S.vals32, x, y, partials, st); break;
        }
    } else {
        switch (u) {
        case 2: sell2_spmv_kernel<DOT, 2><<<sb, kVecThreads, 0, s>>>(S.nslices, S2.perm2, S2.len2, S2.sptr2, S2.cols2, S2.vals2, x, y, partials, st); break;
        case 8: sell2_spmv_kernel<DOT, 8><<<sb, kVecThreads, 0, s>>>(S.nslices, S2.perm2, S2.len2, S2.sptr2, S2.cols2, S2.vals2, x, y, partials, st); break;
        default: sell2_spmv_kernel<DOT, 4><<<sb, kVecThreads, 0, s>>>(S.nslices, S2.perm2, S2.len2, S2.sptr2, S2.cols2, S2.vals2, x, y, partials, st); break;
        }
    }
}

cudaError_t launch_spmv32k(const SellView &S, const Sell2View &S2, int kind, int u, const float *x, float *y,
                           cudaStream_t s) {
    spmv32_dispatch<false>(S, S2, kind, u, x, y, nullptr, nullptr, s);
    return cudaGetLastError();
}

}  // namespace phgb
