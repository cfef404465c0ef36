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
#include "solve.h"

#include <math.h>

namespace phgb {

constexpr int kVecThreads = 256;

// Block-wide sum of two values; thread 0 gets the result.  Fixed tree order.
__device__ __forceinline__ void block_sum2(double &a, double &b) {
    __shared__ double sa[32], sb[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
    }
    __syncthreads();
}

// Publishes this block's partial sums; returns true in the last block to
// arrive, which then holds the grid totals in (a, b) on thread 0.
__device__ __forceinline__ bool grid_sum2(double &a, double &b, double *partials, unsigned *ticket) {
    __shared__ bool last;
    block_sum2(a, b);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double ta = 0.0, tb = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
        ta += __ldcg(&partials[2 * i]);
        tb += __ldcg(&partials[2 * i + 1]);
    }
    block_sum2(ta, tb);
    if (threadIdx.x == 0) { a = ta; b = tb; *ticket = 0u; }
    return true;
}

// ---------------------------------------------------------------------------
// SpMV: LPR lanes per row (CSR vector form).  With DOT, also p.y -> state.
template <int LPR, bool DOT, typename VT>
__global__ void __launch_bounds__(kVecThreads)
spmv_kernel(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
            const VT *__restrict__ va, const VT *__restrict__ x, VT *__restrict__ y,
            double *partials, PcgState *st) {
    if (DOT && st->done) return;
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
    if (grid_sum2(dot, dummy, partials, &st->ticket) && threadIdx.x == 0) {
        const int k = st->nits + 1;
        st->pAp = dot;
        if (dot == 0.0) {
            st->done = 1;
            st->status = PCG_BREAKDOWN;
            st->nits = k;
        } else {
            st->alpha = st->rz_cur / dot;
        }
    }
}

// p = r / D (first iteration) or p = z + beta p.
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
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const VT z = r[i] / dinv_or_d[i];
        p[i] = k == 1 ? z : vb * p[i] + z;
    }
}

// x += alpha p, r -= alpha Ap; sums ||r||^2 and r.(r/D); closes the iteration.
template <typename VT, typename XT>
__global__ void __launch_bounds__(kVecThreads)
pcg_update_kernel(int64_t n, XT *__restrict__ x, VT *__restrict__ r, const VT *__restrict__ p,
                  const VT *__restrict__ Ap, const VT *__restrict__ D, double *partials, PcgState *st,
                  double *hist) {
    if (st->done) return;
    const double alpha = st->alpha;
    const VT va = (VT)alpha;
    double rr = 0.0, rz = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += (XT)(alpha * (double)p[i]);
        const VT ri = r[i] - va * Ap[i];
        r[i] = ri;
        const double rd = (double)ri;
        rr += rd * rd;
        rz += rd * (double)(ri / D[i]);
    }
    if (grid_sum2(rr, rz, partials, &st->ticket) && threadIdx.x == 0) {
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
    if (grid_sum2(s0, s1, partials, ticket) && threadIdx.x == 0) { out[0] = s0; out[1] = s1; }
}

// r = b - y  (y = A x)
template <typename VT>
__global__ void residual_kernel(int64_t n, const VT *__restrict__ b, const VT *__restrict__ y, VT *__restrict__ r) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = b[i] - y[i];
}

// ---------------------------------------------------------------------------
int vec_blocks(int64_t n) {
    int64_t b = ceil_div(n, kVecThreads);
    if (b > 148 * 8) b = 148 * 8;
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
    const int vb = vec_blocks(B.A.n);
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

}  // namespace phgb
