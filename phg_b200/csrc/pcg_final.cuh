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

}  // namespace phgb
