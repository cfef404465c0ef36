// Restarted right-preconditioned GMRES (solver_GMRES_r, solver-phg.c:
// 1050-1260) and PHG's default flexible augmented variant (solver_FLGMRES_r,
// solver-phg.c:2063-2340) with the Jacobi preconditioner.  One restart cycle is
//   resid     z = b - A x, ||z|| -> s_1 (and the tolerance, first cycle)
//   per inner step i = 1..restart:
//     pc      v_i = v_i / h_(i-1,i) (v_1 = z / ||z||), V_0 = v_i / diag
//     spmv    v_(i+1) = A V_0, h_(i,1) = v_(i+1) . v_1
//     mgs k   v_(i+1) -= h_(i,k-1) v_(k-1), h_(i,k) = v_(i+1) . v_k   (k = 2..i)
//     norm    v_(i+1) -= h_(i,i) v_i, h_(i,i+1) = ||v_(i+1)||, Givens rotations
//   solve     H y = s (back substitution)
//   update    x += (V y) / diag
// The modified Gram-Schmidt steps are pipelined: each kernel applies the
// previous projection and sums the next dot product in one pass.  The small
// dense work (rotations, back substitution) runs in one thread with the
// reference's operation order (explicit round-to-nearest, no contraction);
// the element-wise vector updates do the same.  A step whose cycle has
// ended (convergence, restart length, maxit, happy breakdown) returns at once.
#include "common.cuh"
#include "reduce.cuh"
#include "spmv_epi.cuh"
#include "gmres.h"

#include <float.h>
#include <math.h>

namespace phgb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ bool is_zero(double a) { return fabs(a) < 10.0 * DBL_MIN; }   // utils.h:451

int vgrid(int64_t n) {
    int64_t b = ceil_div(n, kThreads);
    if (b > 148 * 4) b = 148 * 4;
    if (b < 1) b = 1;
    return (int)b;
}

__device__ __forceinline__ double &Hat(const GmresState *st, int i, int k) {
    return st->H[(size_t)i * (st->restart + 2) + k];
}

// z = b - A x (solver-phg.c:1104-1106, 1244-1245) and ||z||.
struct EpiResid {
    double *z;
    const double *b;
    double *partials;
    unsigned *ticket;
    GmresState *st;
    __device__ bool skip() const { return st->finished != 0; }
    __device__ void row(int64_t r, double acc, double &sa, double &) const {
        const double v = rn_sub(b[r], acc);
        z[r] = v;
        sa += v * v;
    }
    __device__ void final(double a, double) const {
        const double rn = sqrt(a);
        st->r_norm = rn;
        st->s[1] = rn;
        st->s[0] = 1.0;
        if (st->first) {   // get_tol (solver-phg.c:104-115) with ||r0||
            double tol = rn * st->rtol;
            if (tol < st->btol_bnorm) tol = st->btol_bnorm;
            if (tol < st->atol) tol = st->atol;
            st->tol = tol;
            st->residual = rn;
            st->first = 0;
        }
        st->ninner = 0;
        if (st->flexible)   // cycle k takes mk + min(k, augk) steps (solver-phg.c:2160-2164)
            st->restart = st->mk + (st->itr_out <= st->augk ? st->itr_out : st->augk);
        if (!isfinite(rn)) {
            st->status = GMRES_NONFINITE;
            st->finished = 1;
            st->run = 0;
            return;
        }
        if (st->nits >= st->maxit) {   // while (nits < max_its) ends
            st->finished = 1;
            st->run = 0;
            return;
        }
        st->run = 1;
        st->cycle_done = !(rn > st->tol);
    }
};

// v_(i+1) = A V_0 and h_(i,1) = v_(i+1) . v_1.
struct EpiArnoldi {
    double *y;
    const double *v1;
    double *partials;
    unsigned *ticket;
    GmresState *st;
    int i;
    __device__ bool skip() const { return !st->run || st->cycle_done; }
    __device__ void row(int64_t r, double acc, double &sa, double &) const {
        y[r] = acc;
        sa += acc * v1[r];
    }
    __device__ void final(double a, double) const { Hat(st, i, 1) = a; }
};

// v_i = scale * src (scale = 1 / ||z|| for i = 1, 1 / h_(i-1,i) after; src is
// v_i itself for i > 1), V_0 = v_i / diag.
__global__ void __launch_bounds__(kThreads)
gmres_pc_kernel(int64_t n, int i, const double *src, double *vi, double *__restrict__ v0,
                const double *__restrict__ D, const GmresState *st) {
    if (!st->run || st->cycle_done) return;
    const double scale = __ddiv_rn(1.0, i == 1 ? st->r_norm : Hat(st, i - 1, i));
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
        const double v = rn_mul(scale, src[l]);
        vi[l] = v;
        v0[l] = __ddiv_rn(v, D[l]);
    }
}

// FLGMRES_r: v_i = scale * v_i as above; the step preconditions v_i (i <= mk)
// or the stored correction Z_(i-mk-1) (solver-phg.c:2183-2188) into F_i, the
// vector the product takes and the update keeps.
__global__ void __launch_bounds__(kThreads)
flgmres_pc_kernel(int64_t n, int64_t stride, int i, const double *src, double *vi, const double *Z,
                  double *__restrict__ fi, const double *__restrict__ D, const GmresState *st) {
    if (!st->run || st->cycle_done) return;
    const double scale = __ddiv_rn(1.0, i == 1 ? st->r_norm : Hat(st, i - 1, i));
    const bool aug = i > st->mk;
    const double *za = aug ? Z + (int64_t)(i - st->mk - 1) * stride : vi;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
        const double v = rn_mul(scale, src[l]);
        vi[l] = v;
        fi[l] = __ddiv_rn(aug ? za[l] : v, D[l]);
    }
}

// v_(i+1) += (-h_(i,k-1)) v_(k-1); then h_(i,k) = v_(i+1) . v_k, or for
// k = i + 1 the norm and the rotations of step i.
__global__ void __launch_bounds__(kThreads)
gmres_mgs_kernel(int64_t n, int i, int k, double *__restrict__ w, const double *__restrict__ vprev,
                 const double *__restrict__ vk, double *partials, GmresState *st) {
    if (!st->run || st->cycle_done) return;
    grid_sum_init();
    const double mh = -Hat(st, i, k - 1);
    double sa = 0.0, dummy = 0.0;
    const bool last = k == i + 1;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
        const double v = rn_add(w[l], rn_mul(mh, vprev[l]));
        w[l] = v;
        sa += v * (last ? v : vk[l]);
    }
    if (!grid_sum2(sa, dummy, partials, st->ticket)) return;
    if (!last) {
        Hat(st, i, k) = sa;
        return;
    }
    // the rest of Arnoldi step i (solver-phg.c:1147-1182), one thread
    st->nits += 1;
    const double hn = sqrt(sa);
    Hat(st, i, i + 1) = hn;
    if (is_zero(hn)) {   // happy breakdown: step i is not used
        st->ninner = i - 1;
        st->cycle_done = 1;
        return;
    }
    double *c1 = st->c1, *c2 = st->c2, *s = st->s;
    for (int j = 1; j < i; j++) {
        const double a = Hat(st, i, j), b = Hat(st, i, j + 1);
        Hat(st, i, j) = rn_add(rn_mul(c1[j], a), rn_mul(c2[j], b));
        Hat(st, i, j + 1) = rn_add(rn_mul(-c2[j], a), rn_mul(c1[j], b));
    }
    const double hii = Hat(st, i, i), hi1 = Hat(st, i, i + 1);
    double tmp = sqrt(rn_add(rn_mul(hii, hii), rn_mul(hi1, hi1)));
    if (is_zero(tmp)) tmp = 1.e-16;
    c1[i] = __ddiv_rn(hii, tmp);
    c2[i] = __ddiv_rn(hi1, tmp);
    s[i + 1] = rn_mul(-c2[i], s[i]);
    s[i] = rn_mul(c1[i], s[i]);
    Hat(st, i, i) = rn_add(rn_mul(c1[i], hii), rn_mul(c2[i], hi1));
    const double rn = fabs(s[i + 1]);
    st->r_norm = rn;
    st->ninner = i;
    if (!isfinite(rn)) {
        st->status = GMRES_NONFINITE;
        st->cycle_done = 1;
        return;
    }
    if (rn <= st->tol || i >= st->restart || st->nits >= st->maxit) st->cycle_done = 1;
}

// H y = s by back substitution (solver-phg.c:1201-1207); decides whether the
// solve ends after this cycle's update.
__global__ void gmres_solve_kernel(GmresState *st) {
    if (!st->run || threadIdx.x != 0 || blockIdx.x != 0) return;
    const int i = st->ninner;
    double *s = st->s, *y = st->y;
    for (int j = i; j > 0; j--) {
        y[j] = __ddiv_rn(s[j], Hat(st, j, j));
        for (int k = j - 1; k > 0; k--) s[k] = rn_sub(s[k], rn_mul(Hat(st, j, k), y[j]));
    }
    if (st->flexible) {
        st->zi = st->itr_out % st->augk;
        st->ak = st->itr_out < st->augk ? st->itr_out : st->augk;
        st->itr_out += 1;
    }
    if (st->status != GMRES_OK) {
        st->finished = 1;
    } else if (st->r_norm <= st->tol) {
        st->residual = st->r_norm;
        st->finished = 1;
    } else if (st->nits >= st->maxit) {
        st->finished = 1;
    }
}

// x += (V y) / diag, or x += z / diag when the cycle made no step
// (solver-phg.c:1209-1225).
__global__ void __launch_bounds__(kThreads)
gmres_update_kernel(int64_t n, int64_t stride, const double *__restrict__ V, const double *__restrict__ z,
                    const double *__restrict__ D, double *__restrict__ x, const GmresState *st) {
    if (!st->run) return;
    const int i = st->ninner;
    const double *y = st->y;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
        double c;
        if (i > 0) {
            c = rn_mul(y[1], V[stride + l]);
            for (int j = 2; j <= i; j++) c = rn_add(c, rn_mul(y[j], V[(int64_t)j * stride + l]));
        } else {
            c = z[l];
        }
        x[l] = rn_add(x[l], __ddiv_rn(c, D[l]));
    }
}

// FLGMRES_r's update (solver-phg.c:2250-2290): x += sum_j y_j F_j (the
// cycle's starting residual z when it made no step), and the cycle's
// correction sum_j y_j v_j (j <= mk) + sum_j y_(mk+j) Z_(j-1) (j <= ak) --
// z itself when there was no step -- is stored in Z_zi.
__global__ void __launch_bounds__(kThreads)
flgmres_update_kernel(int64_t n, int64_t stride, const double *__restrict__ V, const double *__restrict__ F,
                      double *Z, const double *__restrict__ z, double *__restrict__ x, const GmresState *st) {
    if (!st->run) return;
    const int i = st->ninner, mk = st->mk;
    const double *y = st->y;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
        double c, w;
        if (i > 0) {
            c = rn_mul(y[1], F[stride + l]);
            for (int j = 2; j <= i; j++) c = rn_add(c, rn_mul(y[j], F[(int64_t)j * stride + l]));
            const int top = i <= mk ? i : mk;
            w = rn_mul(y[1], V[stride + l]);
            for (int j = 2; j <= top; j++) w = rn_add(w, rn_mul(y[j], V[(int64_t)j * stride + l]));
            if (i > mk)
                for (int j = 1; j <= st->ak; j++) w = rn_add(w, rn_mul(y[j + mk], Z[(int64_t)(j - 1) * stride + l]));
        } else {
            c = z[l];
            w = c;
        }
        x[l] = rn_add(c, x[l]);
        Z[(int64_t)st->zi * stride + l] = w;
    }
}

}  // namespace

cudaError_t launch_gmres_cycle(const GmresBuffers &B, const SpmvPlan &P, int restart, cudaStream_t s) {
    const int64_t n = B.n;
    const int vb = vgrid(n);
    double *V0 = B.V;
    auto Vi = [&](int i) { return B.V + (int64_t)i * B.stride; };
    const bool flex = B.F != nullptr;
    launch_spmv_epi(P, B.x, EpiResid{B.z, B.b, B.partials, B.st->ticket, B.st}, s);
    for (int i = 1; i <= restart; i++) {
        double *in = V0;
        if (flex) {
            in = B.F + (int64_t)i * B.stride;
            flgmres_pc_kernel<<<vb, kThreads, 0, s>>>(n, B.stride, i, i == 1 ? B.z : Vi(i), Vi(i), B.Z, in, B.D,
                                                      B.st);
        } else {
            gmres_pc_kernel<<<vb, kThreads, 0, s>>>(n, i, i == 1 ? B.z : Vi(i), Vi(i), V0, B.D, B.st);
        }
        launch_spmv_epi(P, in, EpiArnoldi{Vi(i + 1), Vi(1), B.partials, B.st->ticket, B.st, i}, s);
        for (int k = 2; k <= i + 1; k++)
            gmres_mgs_kernel<<<vb, kThreads, 0, s>>>(n, i, k, Vi(i + 1), Vi(k - 1), k <= i ? Vi(k) : nullptr,
                                                     B.partials, B.st);
    }
    gmres_solve_kernel<<<1, 32, 0, s>>>(B.st);
    if (flex)
        flgmres_update_kernel<<<vb, kThreads, 0, s>>>(n, B.stride, B.V, B.F, B.Z, B.z, B.x, B.st);
    else
        gmres_update_kernel<<<vb, kThreads, 0, s>>>(n, B.stride, B.V, B.z, B.D, B.x, B.st);
    return cudaGetLastError();
}

}  // namespace phgb
