// Launch interfaces of the block (many right-hand sides) PCG (block.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace phgb {

// Device state of a block solve (all arrays in device memory, one entry per
// padded column unless noted).
struct BlockPtrs {
    int64_t n;
    int K;                        // padded column count: a power of two <= 64
    const int32_t *rp, *ci;       // CSR structure
    double *rz_cur, *rz_prev, *alpha, *res, *tol, *maxr, *pAp;
    int *nits, *done, *status;    // status: 1 breakdown, 2 non-finite
    int *flags;                   // [0] all done [1] reliable update [2] final check [3] reset y [4] maxit
    double delta;                 // reliable-update trigger (mixed)
    double *partials;             // block_partials_doubles()
    unsigned *tickets;            // block_ticket_count(), zeroed once
};

struct BlockVecs {
    const double *va, *D;         // FP64 CSR values, Jacobi diagonal
    double *X, *R, *P, *AP;       // n x K, row major
    const float *va32;            // FP32 CSR values (mixed)
    float *D32, *Y32, *R32, *P32, *AP32;
};

size_t block_partials_doubles();
size_t block_ticket_count();
cudaError_t launch_block_init(const BlockPtrs &B, bool mixed, const double *R, const double *D, float *R32,
                              float *D32, float *Y32, double rtol, cudaStream_t s);
cudaError_t launch_block_iteration(const BlockPtrs &B, int T, bool mixed, const BlockVecs &V, cudaStream_t s);
cudaError_t launch_block_spmm64(const BlockPtrs &B, int T, const double *va, const double *P, double *AP,
                                cudaStream_t s);
cudaError_t launch_block_spmm32(const BlockPtrs &B, int T, const float *va, const float *P, float *AP,
                                cudaStream_t s);
cudaError_t launch_block_pack(int64_t n, int m, int K, const double *in, double *out, cudaStream_t s);
cudaError_t launch_block_unpack(int64_t n, int m, int K, const double *in, double *out, cudaStream_t s);
cudaError_t launch_block_sub(int64_t total, const double *a, double *b, cudaStream_t s);   // b = a - b
cudaError_t launch_to_float(int64_t n, const double *a, float *b, cudaStream_t s);

}  // namespace phgb
