// Launch interfaces of the SpMV / PCG kernels (solve.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace phgb {

enum { PCG_RUNNING = 0, PCG_BREAKDOWN = 1, PCG_NONFINITE = 2 };

// Device-resident scalars of one PCG run.
struct PcgState {
    double rz_cur, rz_prev, pAp, alpha, residual, tol;
    int nits, done, status, maxit;
    unsigned ticket;
    int pad;
};

struct CsrView {
    int64_t n;
    const int32_t *rp, *ci;
    const double *va;
};

struct PcgBuffers {
    CsrView A;
    double *x, *r, *p, *Ap;
    const double *D;
    double *partials;     // 2 * vec_blocks
    PcgState *st;
    double *hist;         // may be null
};

int vec_blocks(int64_t n);
int spmv_lanes_for(double avg_nnz_per_row);
cudaError_t launch_spmv(const CsrView &A, int lpr, const double *x, double *y, cudaStream_t s);
cudaError_t launch_pcg_iteration(const PcgBuffers &B, int lpr, cudaStream_t s);
cudaError_t launch_init_sums(int64_t n, int mode, const double *x, const double *b, const double *D,
                             double *partials, unsigned *ticket, double *out, cudaStream_t s);
cudaError_t launch_residual(int64_t n, const double *b, const double *y, double *r, cudaStream_t s);

}  // namespace phgb
