// Mixed-precision Jacobi-PCG with one grid reduction per iteration
// (mixed.cu): FP32 matrix, Krylov vectors and products, FP64 dot products,
// FP64 reliable updates, the whole solve in one CUDA graph launch.
#pragma once
#include "solve.h"

namespace phgb {

// Device-resident scalars of one solve.
struct GearState {
    double alpha, beta;             // scalars of the step the update kernel takes next
    double gamma_prev, alpha_prev;  // r.u and alpha of the previous step
    double gamma_cur, rr_cur;       // r.u and r.r of the current FP32 r and u (the update kernel's sums)
    double tol, maxr, delta, residual;
    int nits, maxit, done, status, first, y_reset, final_check, nupdates, passes, max_passes;
    int ru_due;                     // the last update asked for a reliable update
    unsigned ticket[kRedTickets];
};

enum { GEAR_PASS_LIMIT = kStatusPassLimit };   // status: the graph loop ran out of passes

// Working vectors: x, the right-hand side b and the initial residual rtrue
// FP64; r, u = r / D, w = A u, p, s = A p and the correction y (not yet
// folded into x) FP32.
struct GearBuffers {
    int64_t n;
    double *x, *rtrue;
    const double *b;
    float *r, *u, *w, *p, *s, *y, *D;
    double *partials;   // red_partials3_doubles(kRedMaxBlocks)
    GearState *st;
};

// The FP32 product layout of the iteration (kind 0 SELL, 1 pair SELL, 2 q16,
// with its unroll) and the FP64 values the reliable updates use (the q16
// layout's for kind 2, the SELL copy's otherwise).
struct GearLayouts {
    int kind, unroll;
    SellView S;
    Sell2View S2;
    Q16View Q;
};

// Grid-sum workspace of three sums (reduce.cuh) for `blocks` blocks.
constexpr int64_t red_partials3_doubles(int64_t blocks) {
    return 3 * (blocks + (blocks + kRedGroup - 1) / kRedGroup);
}

// r = (float) rtrue, u = r / D, D32 = (float) D64, y = p = s = 0, and
// (||rtrue||^2, r.u, r.r) into out[0..2].
cudaError_t launch_gear_init(const GearBuffers &B, const double *D64, unsigned *ticket, double *out,
                             cudaStream_t s);
// Builds the executable graph of a whole solve: a loop (conditional WHILE
// node) over `chunk` iterations, each the FP32 product with its dot products,
// a conditional reliable update, and the vector update; the loop ends when the
// state says done.  Graph construction uses `stream` for capture.
// With `plain` the graph is one chunk of iterations without conditional
// nodes (the reliable-update kernels run every iteration and return at once
// unless due) and the host relaunches it until the state says done: for
// profilers that do not see kernels inside conditional graph nodes.
cudaError_t build_gear_graph(const GearBuffers &B, const GearLayouts &L, int chunk, bool plain, cudaStream_t stream,
                             cudaGraphExec_t *exec, int *kernels_per_iteration);
// x += y at the end of a solve, unless a reliable update folded y last.
cudaError_t launch_gear_fold(const GearBuffers &B, cudaStream_t s);

// A graph that repeats `body` (launches on `stream`, captured) in a
// conditional WHILE loop until st->done, at most st->max_passes passes (then
// st->status = kStatusPassLimit): one graph launch runs a whole solve.
cudaError_t build_pcg_loop_graph(cudaStream_t stream, void (*body)(void *ctx, cudaStream_t s), void *ctx,
                                 PcgState *st, bool plain, cudaGraphExec_t *exec);

}  // namespace phgb
