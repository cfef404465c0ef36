// Launch interfaces of the adjoint-gradient kernels (adjoint.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace phgb {

// rhs_adj[i] = u[i] - u_obs[i] on free DOFs, 0 on Dirichlet DOFs;
// out[0] = J = 1/2 sum_i (u[i] - u_obs[i])^2.  partials: >= 2 * 1184 doubles.
cudaError_t launch_adjoint_rhs(int64_t n, const double *u, const double *uobs, const uint8_t *bdry,
                               double *rhs_adj, double *partials, double *out, cudaStream_t s);
// grad[e] = dJ / dlog kappa_e = -lambda_e^T Ke[e] u_e.
cudaError_t launch_adjoint_grad(int p, int64_t nelem, const int32_t *e2l, const double *Ke, const double *lambda,
                                const double *u, double *grad, cudaStream_t s);

}  // namespace phgb
