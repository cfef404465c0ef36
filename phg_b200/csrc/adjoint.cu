// Adjoint gradient of a data-misfit functional with respect to the log of a
// piecewise-constant coefficient.
//
// With the assembled system A(kappa) u = b (Dirichlet rows diagonal, their
// columns lifted into b) and J(u) = 1/2 ||u - u_obs||^2, the adjoint state
// lambda solves A lambda = dJ/du on the free DOFs (lambda = 0 on Dirichlet
// DOFs; A is symmetric), and because each element matrix is linear in its
// coefficient, K_e(kappa_e) = kappa_e K_e^0,
//     dJ/dlog kappa_e = kappa_e dJ/dkappa_e = -kappa_e lambda_e^T K_e^0 u_e
//                     = -lambda_e^T K_e u_e,
// with the element matrix K_e the assembly kernel left in Ke.  No counterpart
// in the reference; it reuses the reference-equivalent assembly and PCG.
#include "common.cuh"
#include "adjoint.h"

namespace phgb {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;

__global__ void __launch_bounds__(kThreads)
adjoint_rhs_kernel(int64_t n, const double *__restrict__ u, const double *__restrict__ uobs,
                   const uint8_t *__restrict__ bdry, double *__restrict__ rhs, double *__restrict__ partials) {
    __shared__ double sw[kThreads / 32];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = u[i] - uobs[i];
        acc += d * d;
        rhs[i] = bdry[i] ? 0.0 : d;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; w++) s += sw[w];
        partials[blockIdx.x] = s;
    }
}

// sums the block partials in block order (deterministic), J = sum / 2
__global__ void sum_partials_kernel(int nb, const double *__restrict__ partials, double *__restrict__ out) {
    __shared__ double s[kThreads];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += partials[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)blockDim.x; i++) t += s[i];
        out[0] = 0.5 * t;
    }
}

template <int N>
__global__ void __launch_bounds__(128)
adjoint_grad_kernel(int64_t nelem, const int32_t *__restrict__ e2l, const double *__restrict__ Ke,
                    const double *__restrict__ lambda, const double *__restrict__ u, double *__restrict__ grad) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t e = warp; e < nelem; e += nwarps) {
        double ub = 0.0, la = 0.0;
        if (lane < N) {
            const int32_t d = e2l[(size_t)e * N + lane];
            ub = u[d];
            la = lambda[d];
        }
        // lane a: lambda_a * sum_b K[a][b] u_b
        double row = 0.0;
        const double *K = Ke + (size_t)e * N * N;
        for (int b = 0; b < N; b++) {
            const double ubb = __shfl_sync(0xffffffffu, ub, b);
            if (lane < N) row += K[lane * N + b] * ubb;
        }
        const double t = warp_sum(lane < N ? la * row : 0.0);
        if (lane == 0) grad[e] = -t;
    }
}

cudaError_t launch_adjoint_rhs(int64_t n, const double *u, const double *uobs, const uint8_t *bdry,
                               double *rhs_adj, double *partials, double *out, cudaStream_t s) {
    int64_t nb = (n + kThreads - 1) / kThreads;
    if (nb > kMaxBlocks) nb = kMaxBlocks;
    adjoint_rhs_kernel<<<(unsigned)nb, kThreads, 0, s>>>(n, u, uobs, bdry, rhs_adj, partials);
    sum_partials_kernel<<<1, kThreads, 0, s>>>((int)nb, partials, out);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_grad(int p, int64_t nelem, const int32_t *e2l, const double *Ke, const double *lambda,
                                const double *u, double *grad, cudaStream_t s) {
    int64_t nb = (nelem * 32 + 127) / 128;
    if (nb > 148 * 64) nb = 148 * 64;
    if (p == 1) adjoint_grad_kernel<4><<<(unsigned)nb, 128, 0, s>>>(nelem, e2l, Ke, lambda, u, grad);
    else if (p == 2) adjoint_grad_kernel<10><<<(unsigned)nb, 128, 0, s>>>(nelem, e2l, Ke, lambda, u, grad);
    else adjoint_grad_kernel<20><<<(unsigned)nb, 128, 0, s>>>(nelem, e2l, Ke, lambda, u, grad);
    return cudaGetLastError();
}

}  // namespace phgb
