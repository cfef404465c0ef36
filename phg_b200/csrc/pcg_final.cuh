// Scalar steps of the PCG recurrences, run by the one thread that finishes a
// grid-wide sum (reduce.cuh).  Shared by every SpMV layout.
#pragma once
#include "solve.h"

namespace phgb {

// p.Ap of iteration nits + 1 is known: alpha = (r.z) / (p.Ap), or a
// breakdown when p.Ap is zero (the reference would divide by zero).
__device__ __forceinline__ void pcg_pap_final(double dot, PcgState *st) {
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

// The reliable update of the mixed solver is done: ||r_true||^2 = rr and
// r32.(r32 / D) = rz.  The FP64 residual becomes the reference point of the
// next update; a pending final check stops the iteration when it meets the
// tolerance.
__device__ __forceinline__ void mixed_reliable_final(double rr, double rz, MixedState *ms, double *hist) {
    PcgState *st = &ms->pcg;
    const double res = sqrt(rr);
    st->residual = res;
    st->rz_cur = rz;
    ms->maxr = res;
    ms->y_reset = 1;
    ms->ru_flag = 0;
    ms->nupdates += 1;
    if (hist != nullptr) hist[st->nits] = res;
    if (ms->final_check) {
        ms->final_check = 0;
        if (!(res > st->tol) || st->nits >= st->maxit) st->done = 1;
    }
}

}  // namespace phgb
