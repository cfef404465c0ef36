// Jacobi-preconditioned BiCGstab on the device (solver_BiCGstab,
// solver-phg.c:606-781), on the same SpMV layouts as the PCG.
#pragma once
#include "solve.h"

namespace phgb {

// Device-resident scalars of the BiCGstab recurrence.
struct BicgState {
    double rho0, rho1, alpha, omega, rhv, residual, tol, snorm;
    int nits, done, status, maxit;
    unsigned ticket[kRedTickets];
    int pad;
};

// status values
enum {
    BICG_OK = 0,
    BICG_RHO_ZERO = 1,     // rho = r.rh = 0: the reference's "method failed" break
    BICG_SMALL_S = 2,      // ||s|| <= 1e-60: x += alpha p^, residual recomputed (host)
    BICG_BREAKDOWN = 3,    // rh.v = 0 or t.t = 0 (the reference would divide by zero)
    BICG_NONFINITE = 4,
};

struct BicgBuffers {
    int64_t n;
    double *x, *rg, *rh, *pg, *ph, *sg, *sh, *tg, *vg;   // 16-byte aligned
    const double *D;
    double *partials;
    BicgState *st;
    double *hist;   // optional: ||r|| after each iteration
};

// Distance between the working vectors of one buffer (keeps each 16-byte aligned).
int64_t bicg_stride(int64_t n);
constexpr int kBicgVectors = 7;   // rh, pg, ph, sg, sh, tg, vg

cudaError_t launch_bicg_iteration(const BicgBuffers &B, const SpmvPlan &P, cudaStream_t s);
// x += alpha p^ after a small-s stop (solver-phg.c:705-716)
cudaError_t launch_bicg_small_s(const BicgBuffers &B, cudaStream_t s);

}  // namespace phgb
