// Restarted right-preconditioned GMRES on the device (solver_GMRES_r,
// solver-phg.c:1050-1260), Jacobi preconditioner, on the SpMV layout the
// PCG autotuner chose.
#pragma once
#include "solve.h"

namespace phgb {

constexpr int kGmresMaxRestart = 64;

// Device-resident state of the solve.  H, c1, c2, s, y point to a device
// array laid out as H[(R + 2) * (R + 2)] (row i = inner iteration, column k),
// then c1, c2, s, y with R + 2 entries each (R = restart).
struct GmresState {
    double r_norm, tol, residual, rtol, btol_bnorm, atol;
    int nits, maxit, restart, ninner;
    int run, cycle_done, finished, first, status;
    // FLGMRES_r: base restart mk, augmenting corrections augk, cycle count,
    // and for the cycle's update the slot its correction goes to and the
    // number of corrections its basis used
    int flexible, mk, augk, itr_out, zi, ak;
    unsigned ticket[kRedTickets];
    double *H, *c1, *c2, *s, *y;
};

enum { GMRES_OK = 0, GMRES_NONFINITE = 1 };

struct GmresBuffers {
    int64_t n;
    double *x;
    const double *b, *D;
    double *z;          // residual b - A x, then the correction V y
    double *V;          // restart + 2 vectors at distance `stride`: V_0 = M^-1 v_i, V_1.. the basis
    int64_t stride;
    double *partials;
    GmresState *st;
    // FLGMRES_r only: F_1..F_R the preconditioned vectors of the steps (F_i
    // at F + i * stride), Z_0..Z_(augk-1) the stored corrections
    double *F, *Z;
};

inline int64_t gmres_small_doubles(int restart) { return (int64_t)(restart + 2) * (restart + 2) + 4 * (restart + 2); }

// One restart cycle: b - A x and its norm, `restart` Arnoldi steps (each a
// no-op once the cycle is over), the triangular solve and x += M^-1 V y.
// With st->flexible (FLGMRES_r, solver-phg.c:2063-2340) `restart` is mk +
// augk, the most steps a cycle takes; the cycle's own length is set by the
// state.
cudaError_t launch_gmres_cycle(const GmresBuffers &B, const SpmvPlan &P, int restart, cudaStream_t s);

}  // namespace phgb
