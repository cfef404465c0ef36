// Launch interfaces of the SpMV / PCG kernels (solve.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace phgb {

constexpr int kVecThreads = 256;   // threads per block of the solver kernels
// Grid-stride kernels launched on vec_blocks() grids (148 x 8 blocks) declare
// 8 resident blocks per SM (at most 32 registers a thread): with fewer, the
// grid runs as two waves and the second leaves most of the GPU idle.
constexpr int kResidentBlocks = 8;

enum { PCG_RUNNING = 0, PCG_BREAKDOWN = 1, PCG_NONFINITE = 2 };

// Device-resident scalars of one PCG run.
// Grid-wide sums (reduce.cuh) combine block sums in groups of kRedGroup
// blocks, then the group sums; grids have at most kRedMaxBlocks blocks and a
// sum needs kRedTickets counters.
constexpr int kRedGroup = 64;
constexpr int kRedMaxBlocks = 2048;   // at most 32 groups: one load per lane
constexpr int kRedTickets = 1 + kRedMaxBlocks / kRedGroup;
// Doubles of grid-sum workspace (reduce.cuh) a grid of `blocks` blocks uses.
constexpr int64_t red_partials_doubles(int64_t blocks) {
    return 2 * (blocks + (blocks + kRedGroup - 1) / kRedGroup);
}
// Largest grid vec_blocks() returns; every grid-sum launch stays within
// kRedMaxBlocks.
constexpr int kVecMaxBlocks = 148 * kResidentBlocks;
static_assert(kVecMaxBlocks <= kRedMaxBlocks, "grid sums take at most kRedMaxBlocks blocks");

struct PcgState {
    double rz_cur, rz_prev, pAp, alpha, residual, tol;
    int nits, done, status, maxit;
    unsigned ticket[kRedTickets];
    int passes, max_passes;   // passes of a graph loop, and their bound
};

// Status of a solve whose graph loop ran out of passes (a safeguard).
constexpr int kStatusPassLimit = 3;

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

// SpMV layouts: CSR with `lpr` lanes per row, or SELL-C-sigma (C = 32,
// sigma = 256) with the inner loop unrolled `unroll` times.
// SPMV_Q16: the 16-bit-column layout with FP64 values (FP64 products read
// 10 bytes per stored entry instead of 12).
enum { SPMV_CSR = 0, SPMV_SELL = 1, SPMV_Q16 = 2 };

struct SellView {
    int64_t n, nslices;
    const int32_t *perm;      // sorted position -> row, -1 for padding positions
    const uint16_t *len;      // row length at each sorted position
    const int32_t *sptr;      // slice offsets (nslices + 1)
    const int32_t *cols;
    const double *vals;
    const float *vals32;      // FP32 copy of the values (mixed precision), may be null
};

// FP32 pair layout of the same slices (see solve.cu).
struct Sell2View {
    const int32_t *sptr2;     // slice offsets in entries (nslices + 1), slices stored widest first
    const int32_t *cols2;
    const float *vals2;
    const int32_t *perm2;     // row of each position in the stored slice order
    const uint16_t *len2;     // its length
};

// The 16-bit-column layout ("q16", q16.cu): the same slices as SELL-C-sigma (C = 32, sigma = 256), stored widest first.
// Each lane holds four consecutive entries of its row per step (one 16-byte
// load of FP32 values, one 8-byte load of four 16-bit column offsets), so an
// entry costs 6 bytes in the FP32 product instead of 8.  A row's entries are
// split into two column windows of 65536: entries [0, split) are offsets
// from base0 (the row's smallest column), the rest from base1 (the smallest
// column outside the first window).  Rows of Lagrange P1-P3 matrices numbered
// vertices first, then edges and faces, fit; a matrix with a row that does
// not fit does not get this layout.
struct Q16View {
    int64_t nslices;
    const int32_t *sptr;       // stored slice offsets in entries (nslices + 1), multiples of 128
    const int32_t *perm;       // row of each stored position, -1 for padding
    const uint16_t *len;       // its length
    const uint16_t *split;     // entries of the first window
    const int32_t *base0, *base1;
    const uint16_t *cols;      // column offsets
    const float *vals32;       // FP32 values (mixed solver's product)
    const double *vals64;      // FP64 values (reliable updates, residuals)
};

struct SpmvPlan {
    int kind = SPMV_CSR, lpr = 8, unroll = 4;
    CsrView csr{};
    SellView sell{};
    Q16View q16{};
};

int vec_blocks(int64_t n);
cudaError_t launch_sell2_heads(const SellView &S, uint16_t *width, cudaStream_t s);
cudaError_t launch_sell2_sizes(const SellView &S, const int32_t *order, int32_t *sizes, cudaStream_t s);
cudaError_t launch_sell2_fill(const SellView &S, const int32_t *rp, const int32_t *ci, const double *va,
                              const int32_t *order, const int32_t *sptr2, int32_t *perm2, uint16_t *len2,
                              int32_t *cols2, float *vals2, cudaStream_t s);
cudaError_t launch_spmv32k(const SellView &S, const Sell2View &S2, int kind, int u, const float *x, float *y,
                           cudaStream_t s);
int64_t sell_positions(int64_t n);   // perm/len entries = slices * 32
cudaError_t launch_sell_sort(int64_t n, const int32_t *rp, int32_t *perm, uint16_t *len, int32_t *slice_size,
                             cudaStream_t s);
cudaError_t launch_sell_fill(int64_t n, const int32_t *rp, const int32_t *ci, const double *va, const int32_t *perm,
                             const uint16_t *len, const int32_t *sptr, int32_t *cols, double *vals, float *vals32,
                             cudaStream_t s);
cudaError_t launch_spmv_plan(const SpmvPlan &P, const double *x, double *y, cudaStream_t s);
cudaError_t launch_pcg_iteration_plan(const PcgBuffers &B, const SpmvPlan &P, cudaStream_t s);
int spmv_lanes_for(double avg_nnz_per_row);
cudaError_t launch_spmv(const CsrView &A, int lpr, const double *x, double *y, cudaStream_t s);
cudaError_t launch_pcg_iteration(const PcgBuffers &B, int lpr, cudaStream_t s);
cudaError_t launch_init_sums(int64_t n, int mode, const double *x, const double *b, const double *D,
                             double *partials, unsigned *ticket, double *out, cudaStream_t s);
cudaError_t launch_residual(int64_t n, const double *b, const double *y, double *r, cudaStream_t s);

}  // namespace phgb
