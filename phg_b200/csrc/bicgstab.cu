// Jacobi-preconditioned BiCGstab on the device: the recurrence of
// solver_BiCGstab (solver-phg.c:606-781), one iteration as five kernels
//   dir      p = r + beta (p - omega v), p^ = p / diag           (:682-700)
//   spmv     v = A p^, and rh.v -> alpha = rho / rh.v            (:707-713)
//   s        s = r - alpha v, ||s||, s^ = s / diag               (:714-734)
//   spmv     t = A s^, and t.s, t.t -> omega = t.s / t.t         (:736-740)
//   update   p^ = alpha p^ + omega s^, x += p^, r = s - omega t,
//            ||r|| and r.rh (rho of the next iteration)           (:742-750)
// with the scalars in a device-resident state block and the reductions
// finished by the last block to arrive, as in the PCG (solve.cu).  Every
// kernel returns at once when the state says `done`, so a captured graph of
// several iterations becomes a no-op after the stopping rule is met.
#include "common.cuh"
#include "reduce.cuh"
#include "spmv_epi.cuh"
#include "bicgstab.h"

#include <math.h>

namespace phgb {

namespace {

constexpr int kThreads = 256;

int vgrid(int64_t n) {
    int64_t b = ceil_div(ceil_div(n, 2), kThreads);
    if (b > 148 * 4) b = 148 * 4;
    if (b < 1) b = 1;
    return (int)b;
}

int sgrid(int64_t threads) {
    int64_t b = ceil_div(threads, kThreads);
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) b = 1;
    return (int)b;
}

__global__ void __launch_bounds__(kThreads)
bicg_dir_kernel(int64_t n, const double *__restrict__ rg, const double *__restrict__ vg,
                const double *__restrict__ D, double *__restrict__ pg, double *__restrict__ ph, BicgState *st) {
    if (st->done) return;
    const int k = st->nits + 1;
    const double rho1 = st->rho1;
    if (rho1 == 0.0) {   // solver-phg.c:676-680: counted, then the loop ends
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->done = 1;
            st->status = BICG_RHO_ZERO;
            st->nits = k;
        }
        return;
    }
    const bool first = k == 1;
    const double beta = first ? 0.0 : (rho1 * st->alpha) / (st->rho0 * st->omega);
    const double mo = -st->omega;
    const int64_t nfull = aligned16(rg, vg, D, pg, ph) ? n / 2 : 0;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nfull; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = 2 * c;
        const VArr<double> r = vload_ro(rg + i), d = vload_ro(D + i);
        VArr<double> p = first ? r : vload(pg + i), q;
        if (!first) {
            const VArr<double> v = vload_ro(vg + i);
#pragma unroll
            for (int u = 0; u < 2; u++) p.v[u] = r.v[u] + beta * (p.v[u] + mo * v.v[u]);
        }
#pragma unroll
        for (int u = 0; u < 2; u++) q.v[u] = p.v[u] / d.v[u];
        vstore(pg + i, p);
        vstore(ph + i, q);
    }
    for (int64_t i = 2 * nfull + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double p = first ? rg[i] : rg[i] + beta * (pg[i] + mo * vg[i]);
        pg[i] = p;
        ph[i] = p / D[i];
    }
}

// SpMV epilogues (spmv_epi.cuh).  Alpha: v = A p^, sums rh.v and sets
// alpha = rho / rh.v.  Omega: t = A s^, sums t.s and t.t and sets
// omega = t.s / t.t.  A zero denominator, where the reference would divide
// by zero, ends the solve with BICG_BREAKDOWN.
struct EpiAlpha {
    double *y;
    const double *w;
    double *partials;
    unsigned *ticket;
    BicgState *st;
    __device__ bool skip() const { return st->done != 0; }
    __device__ void row(int64_t r, double acc, double &sa, double &) const {
        y[r] = acc;
        sa += w[r] * acc;
    }
    __device__ void final(double a, double) const {
        st->rhv = a;
        if (a == 0.0 || !isfinite(a)) {
            st->done = 1;
            st->status = a == 0.0 ? BICG_BREAKDOWN : BICG_NONFINITE;
            st->nits = st->nits + 1;
        } else {
            st->alpha = st->rho1 / a;
            st->rho0 = st->rho1;
        }
    }
};

struct EpiOmega {
    double *y;
    const double *w;
    double *partials;
    unsigned *ticket;
    BicgState *st;
    __device__ bool skip() const { return st->done != 0; }
    __device__ void row(int64_t r, double acc, double &sa, double &sb) const {
        y[r] = acc;
        sa += w[r] * acc;
        sb += acc * acc;
    }
    __device__ void final(double a, double b) const {
        if (b == 0.0 || !isfinite(a) || !isfinite(b)) {
            st->done = 1;
            st->status = b == 0.0 ? BICG_BREAKDOWN : BICG_NONFINITE;
            st->nits = st->nits + 1;
        } else {
            st->omega = a / b;
        }
    }
};

__global__ void __launch_bounds__(kThreads)
bicg_s_kernel(int64_t n, const double *__restrict__ rg, const double *__restrict__ vg, const double *__restrict__ D,
              double *__restrict__ sg, double *__restrict__ sh, double *partials, BicgState *st) {
    if (st->done) return;
    grid_sum_init();
    const double ma = -st->alpha;
    double ss = 0.0, dummy = 0.0;
    const int64_t nfull = aligned16(rg, vg, D, sg, sh) ? n / 2 : 0;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nfull; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = 2 * c;
        const VArr<double> r = vload_ro(rg + i), v = vload_ro(vg + i), d = vload_ro(D + i);
        VArr<double> sv, hv;
#pragma unroll
        for (int u = 0; u < 2; u++) {
            sv.v[u] = r.v[u] + ma * v.v[u];
            hv.v[u] = sv.v[u] / d.v[u];
            ss += sv.v[u] * sv.v[u];
        }
        vstore(sg + i, sv);
        vstore(sh + i, hv);
    }
    for (int64_t i = 2 * nfull + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double sv = rg[i] + ma * vg[i];
        sg[i] = sv;
        sh[i] = sv / D[i];
        ss += sv * sv;
    }
    if (grid_sum2(ss, dummy, partials, st->ticket)) {
        const double s = sqrt(ss);
        st->snorm = s;
        if (s <= 1e-60) {   // solver-phg.c:717-729; the host finishes the step
            st->done = 1;
            st->status = BICG_SMALL_S;
            st->nits = st->nits + 1;
        }
    }
}

__global__ void __launch_bounds__(kThreads)
bicg_update_kernel(int64_t n, double *__restrict__ x, double *__restrict__ ph, const double *__restrict__ sh,
                   const double *__restrict__ sg, const double *__restrict__ tg, double *__restrict__ rg,
                   const double *__restrict__ rh, double *partials, BicgState *st, double *hist) {
    if (st->done) return;
    grid_sum_init();
    const double al = st->alpha, om = st->omega, mo = -om;
    double rr = 0.0, rrh = 0.0;
    const int64_t nfull = aligned16(x, ph, sh, sg, tg, rg, rh) ? n / 2 : 0;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nfull; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = 2 * c;
        const VArr<double> h = vload_ro(sh + i), s = vload_ro(sg + i), t = vload_ro(tg + i), w = vload_ro(rh + i);
        VArr<double> p = vload(ph + i), xv = vload(x + i), r;
#pragma unroll
        for (int u = 0; u < 2; u++) {
            p.v[u] = al * p.v[u] + om * h.v[u];
            xv.v[u] = xv.v[u] + p.v[u];
            r.v[u] = s.v[u] + mo * t.v[u];
            rr += r.v[u] * r.v[u];
            rrh += r.v[u] * w.v[u];
        }
        vstore(ph + i, p);
        vstore(x + i, xv);
        vstore(rg + i, r);
    }
    for (int64_t i = 2 * nfull + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double p = al * ph[i] + om * sh[i];
        ph[i] = p;
        x[i] = x[i] + p;
        const double r = sg[i] + mo * tg[i];
        rg[i] = r;
        rr += r * r;
        rrh += r * rh[i];
    }
    if (grid_sum2(rr, rrh, partials, st->ticket)) {
        const int k = st->nits + 1;
        const double res = sqrt(rr);
        st->residual = res;
        st->rho1 = rrh;
        st->nits = k;
        if (hist != nullptr) hist[k] = res;
        if (!isfinite(res)) {
            st->done = 1;
            st->status = BICG_NONFINITE;
        } else if (!(res > st->tol) || k >= st->maxit) {
            st->done = 1;
        }
    }
}

__global__ void bicg_small_s_kernel(int64_t n, double *__restrict__ x, const double *__restrict__ ph,
                                    const BicgState *st) {
    const double al = st->alpha;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = x[i] + al * ph[i];
}

}  // namespace

int64_t bicg_stride(int64_t n) { return (n + 31) / 32 * 32; }

cudaError_t launch_bicg_iteration(const BicgBuffers &B, const SpmvPlan &P, cudaStream_t s) {
    const int vb = vgrid(B.n);
    bicg_dir_kernel<<<vb, kThreads, 0, s>>>(B.n, B.rg, B.vg, B.D, B.pg, B.ph, B.st);
    launch_spmv_epi(P, B.ph, EpiAlpha{B.vg, B.rh, B.partials, B.st->ticket, B.st}, s);
    bicg_s_kernel<<<vb, kThreads, 0, s>>>(B.n, B.rg, B.vg, B.D, B.sg, B.sh, B.partials, B.st);
    launch_spmv_epi(P, B.sh, EpiOmega{B.tg, B.sg, B.partials, B.st->ticket, B.st}, s);
    bicg_update_kernel<<<vb, kThreads, 0, s>>>(B.n, B.x, B.ph, B.sh, B.sg, B.tg, B.rg, B.rh, B.partials, B.st,
                                               B.hist);
    return cudaGetLastError();
}

cudaError_t launch_bicg_small_s(const BicgBuffers &B, cudaStream_t s) {
    bicg_small_s_kernel<<<sgrid(B.n), kThreads, 0, s>>>(B.n, B.x, B.ph, B.st);
    return cudaGetLastError();
}

}  // namespace phgb
