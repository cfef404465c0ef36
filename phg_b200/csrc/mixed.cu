// Mixed-precision Jacobi-PCG with one grid-wide reduction per iteration.
//
// The recurrence is the single-reduction form of preconditioned CG
// (Chronopoulos and Gear): with u = D^-1 r, w = A u and s = A p kept by
// recurrence,
//   gamma = r.u, delta = w.u
//   beta  = gamma / gamma_prev,  alpha = gamma / (delta - beta gamma / alpha_prev)
//   p = u + beta p,  s = w + beta s,  y += alpha p,  r -= alpha s,  u = D^-1 r
// In exact arithmetic it produces the iterates of solver_pcg
// (solver-phg.c:485-604).  An iteration is two kernels, each with one grid
// sum in its epilogue:
//   K1  w = A u (FP32 values and vectors) and delta = w.u in FP64; the last
//       block takes the step's alpha and beta from delta and the gamma the
//       update left
//   K2  the vector update above, and the next gamma = r.u and r.r in FP64
//       from the new r and u while they are in registers; the last block
//       tests the FP32 residual and decides whether a reliable update is due
// A reliable update (the FP32 residual has fallen tenfold since the last one,
// or the iteration looks converged) runs inside a conditional graph node
// after K2, before the next product:
//   R0  x += y (FP64)
//   R1  rtrue = b - A x with the FP64 matrix values (the explicit residual of
//       the FP64 iterate), r = (float) rtrue, u = D^-1 r, ||rtrue||^2 -> the
//       stopping test (the reference's rule, get_tol solver-phg.c:104), and
//       r.u, r.r for the next step
// and the next K1 takes its product on the new u; the K2 after it restarts
// y.  The stopping test thus sees the residual of the iterate it returns,
// not a recurrence that may have drifted from it.
// The iterations run in a conditional WHILE loop of `chunk` iterations per
// pass, so a solve is one graph launch and the host waits once.
#include "common.cuh"
#include "mixed.h"
#include "reduce.cuh"
#include "rows.cuh"

#include <math.h>

namespace phgb {

// ---------------------------------------------------------------------------
// The scalar decisions, taken by the one thread that finishes a grid sum.

__device__ __forceinline__ void gear_breakdown(GearState *st) {
    st->done = 1;
    st->status = PCG_BREAKDOWN;
    st->nits += 1;   // the reference counts the step it breaks down in (solver-phg.c:537)
}

// The step from gamma = r.u (the update kernel's, or the reliable update's)
// and delta = w.u.
__device__ __forceinline__ void gear_step(GearState *st, double gamma, double delta) {
    if (!(isfinite(gamma) && isfinite(delta))) {
        st->done = 1;
        st->status = PCG_NONFINITE;
        return;
    }
    double alpha, beta;
    if (st->first) {
        if (delta == 0.0) { gear_breakdown(st); return; }
        beta = 0.0;
        alpha = gamma / delta;
    } else {
        if (st->gamma_prev == 0.0) { gear_breakdown(st); return; }
        beta = gamma / st->gamma_prev;
        const double den = delta - beta * gamma / st->alpha_prev;
        if (den == 0.0) { gear_breakdown(st); return; }
        alpha = gamma / den;
    }
    st->alpha = alpha;
    st->beta = beta;
    st->gamma_prev = gamma;
    st->alpha_prev = alpha;
    st->first = 0;
    st->nits += 1;
}

// After an update: the FP32 recurrence's residual (rr = r.r) against the
// tolerance and the last reliable update.  Returns whether a reliable
// update is due.
__device__ __forceinline__ bool gear_check(GearState *st, double rr) {
    const double res = sqrt(rr);
    st->residual = res;
    st->y_reset = 0;   // this update restarted y if it had to
    if (!isfinite(res)) {
        st->done = 1;
        st->status = PCG_NONFINITE;
        return false;
    }
    const bool conv = !(res > st->tol) || st->nits >= st->maxit;
    st->final_check = conv ? 1 : 0;
    return conv || res < st->delta * st->maxr;
}

// ---------------------------------------------------------------------------
// K1: w = A u and delta = w.u.  Grid-stride over slices on a grid of
// kGearBlocksPerSM blocks of 256 threads per SM.
constexpr int kGearBlocksPerSM = 8;

template <class L>
__global__ void __launch_bounds__(kVecThreads, kGearBlocksPerSM)
gear_spmv_kernel(const L lay, const GearBuffers B) {
    GearState *st = B.st;
    if (st->done) return;
    grid_sum_init();
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * kVecThreads + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * kVecThreads) >> 5);
    double delta = 0.0, dummy = 0.0;
    const int nsl = (int)lay.nslices();   // < 2^26 (rows < 2^31)
    for (int s = warp; s < nsl; s += nwarps) {
        const int64_t pos = (int64_t)s * 32 + lane;
        const int32_t row = lay.row(pos);
        // the row's own u, loaded before the row sum so that it arrives
        // behind it (after it, it would add a memory round trip to every
        // slice a warp takes)
        const float uf = row >= 0 ? __ldg(&B.u[row]) : 0.0f;
        const float acc = lay.sum(s, lane, pos, B.u);
        if (row >= 0) {
            B.w[row] = acc;
            delta += (double)acc * (double)uf;
        }
    }
    if (grid_sum2(delta, dummy, B.partials, st->ticket)) gear_step(st, st->gamma_cur, delta);
}

// R0: x += y before the explicit residual.
__global__ void __launch_bounds__(kVecThreads)
gear_fold_ru_kernel(const GearBuffers B) {
    if (B.st->done || !B.st->ru_due) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += (int64_t)gridDim.x * blockDim.x)
        B.x[i] += (double)B.y[i];
}

// R1: the reliable update with the FP64 matrix values.
template <class L64>
__global__ void __launch_bounds__(kVecThreads, 6)
gear_reliable_kernel(const L64 lay, const GearBuffers B) {
    GearState *st = B.st;
    if (st->done || !st->ru_due) return;
    grid_sum3_init();
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * kVecThreads + threadIdx.x) >> 5);
    const int nwarps = (int)((gridDim.x * kVecThreads) >> 5);
    double v[3] = {0.0, 0.0, 0.0};   // ||rtrue||^2, r.u, r.r
    const int nsl = (int)lay.nslices();
    for (int s = warp; s < nsl; s += nwarps) {
        const int64_t pos = (int64_t)s * 32 + lane;
        const int32_t row = lay.row(pos);
        double bi = 0.0;
        float di = 1.0f;
        if (row >= 0) {   // loaded before the row sum, as in K1
            bi = __ldg(&B.b[row]);
            di = __ldg(&B.D[row]);
        }
        const double acc = lay.sum_x(s, lane, pos, B.x);
        if (row >= 0) {
            const double rt = bi - acc;
            const float rf = (float)rt, uf = rf / di;
            B.r[row] = rf;
            B.u[row] = uf;
            v[0] += rt * rt;
            v[1] += (double)rf * (double)uf;
            v[2] += (double)rf * (double)rf;
        }
    }
    if (grid_sum3(v, B.partials, st->ticket)) {
        const double res = sqrt(v[0]);
        st->residual = res;
        st->maxr = res;
        st->gamma_cur = v[1];
        st->rr_cur = v[2];
        st->y_reset = 1;
        st->nupdates += 1;
        st->final_check = 0;
        if (!isfinite(res)) {
            st->done = 1;
            st->status = PCG_NONFINITE;
        } else if (!(res > st->tol) || st->nits >= st->maxit) {
            st->done = 1;   // the FP64 residual meets the tolerance, or maxit
        }
    }
}

// K2: the vector update, V rows a thread and step (16-byte vectors: 2.5% to
// 7% faster solves at P2 64^3 than 8-byte ones at 5 blocks an SM), with the
// next gamma = r.u and r.r summed from the new r and u.  After a reliable
// update (whose R0 folded y into x) it restarts y.
template <int V> struct FVec;
template <> struct FVec<2> { using T = float2; };
template <> struct FVec<4> { using T = float4; };

template <int V>
struct FArr {
    float v[V];
};
template <int V> __device__ __forceinline__ FArr<V> fload(const float *p) {
    FArr<V> a;
    *reinterpret_cast<typename FVec<V>::T *>(a.v) = *reinterpret_cast<const typename FVec<V>::T *>(p);
    return a;
}
template <int V> __device__ __forceinline__ FArr<V> fload_ro(const float *p) {
    FArr<V> a;
    *reinterpret_cast<typename FVec<V>::T *>(a.v) = __ldg(reinterpret_cast<const typename FVec<V>::T *>(p));
    return a;
}
template <int V> __device__ __forceinline__ void fstore(float *p, const FArr<V> &a) {
    *reinterpret_cast<typename FVec<V>::T *>(p) = *reinterpret_cast<const typename FVec<V>::T *>(a.v);
}

constexpr int kUpdateV = 4;

// COND: the graph has conditional nodes and K2 sets the reliable update's
// condition (a kernel that sets a graph condition is one that profilers do
// not see, so the plain graphs launch an instance without the call).
template <int V, bool COND = true>
__global__ void __launch_bounds__(kVecThreads, V == 2 ? 5 : 4)
gear_update_kernel(const GearBuffers B, cudaGraphConditionalHandle hif) {
    GearState *st = B.st;
    if (st->done) return;
    grid_sum_init();
    const float a = (float)st->alpha, b = (float)st->beta;
    const bool reset = st->y_reset != 0;
    const int64_t n = B.n;
    const int nfull = aligned16(B.r, B.u, B.w, B.p, B.s, B.y, B.D) ? (int)(n / V) : 0;   // n < 2^31
    const int stride = gridDim.x * blockDim.x;
    double ru = 0.0, rr = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nfull; c += stride) {
        const int i = V * c;
        // u = r / D is not read: the stored u is that same correctly rounded
        // quotient (K2, R1 and the set-up all form it so), recomputed here
        FArr<V> p = fload<V>(B.p + i), w = fload_ro<V>(B.w + i), s = fload<V>(B.s + i);
        FArr<V> y;
        if (reset) {
#pragma unroll
            for (int q = 0; q < V; q++) y.v[q] = 0.0f;
        } else {
            y = fload<V>(B.y + i);
        }
        FArr<V> r = fload<V>(B.r + i), u;
        const FArr<V> d = fload_ro<V>(B.D + i);
#pragma unroll
        for (int q = 0; q < V; q++) {
            p.v[q] = r.v[q] / d.v[q] + b * p.v[q];
            s.v[q] = w.v[q] + b * s.v[q];
            y.v[q] = y.v[q] + a * p.v[q];
            r.v[q] = r.v[q] - a * s.v[q];
            u.v[q] = r.v[q] / d.v[q];
            ru += (double)r.v[q] * (double)u.v[q];
            rr += (double)r.v[q] * (double)r.v[q];
        }
        fstore<V>(B.p + i, p);
        fstore<V>(B.s + i, s);
        fstore<V>(B.y + i, y);
        fstore<V>(B.r + i, r);
        fstore<V>(B.u + i, u);
    }
    for (int64_t i = (int64_t)nfull * V + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float p = B.r[i] / B.D[i] + b * B.p[i], s = B.w[i] + b * B.s[i];
        B.p[i] = p;
        B.s[i] = s;
        B.y[i] = (reset ? 0.0f : B.y[i]) + a * p;
        const float r = B.r[i] - a * s, u = r / B.D[i];
        B.r[i] = r;
        B.u[i] = u;
        ru += (double)r * (double)u;
        rr += (double)r * (double)r;
    }
    if (grid_sum2(ru, rr, B.partials, st->ticket)) {
        st->gamma_cur = ru;
        st->rr_cur = rr;
        const bool due = gear_check(st, rr);
        st->ru_due = due ? 1 : 0;
        if constexpr (COND) cudaGraphSetConditional(hif, due ? 1u : 0u);
    }
}

// One pass of the graph loop is over: stop when done, or when the passes
// exceed the bound the iteration limit gives (a safeguard: every pass takes
// `chunk` steps until done).
__global__ void gear_loop_kernel(GearState *st, cudaGraphConditionalHandle hwhile) {
    st->passes += 1;
    if (!st->done && st->passes > st->max_passes) {
        st->done = 1;
        st->status = GEAR_PASS_LIMIT;
    }
    cudaGraphSetConditional(hwhile, st->done ? 0u : 1u);
}

// The same for the FP64 PCG's state.
__global__ void pcg_loop_kernel(PcgState *st, cudaGraphConditionalHandle hwhile) {
    st->passes += 1;
    if (!st->done && st->passes > st->max_passes) {
        st->done = 1;
        st->status = kStatusPassLimit;
    }
    cudaGraphSetConditional(hwhile, st->done ? 0u : 1u);
}

__global__ void __launch_bounds__(kVecThreads)
gear_init_kernel(const GearBuffers B, const double *__restrict__ D64, unsigned *ticket, double *out) {
    grid_sum3_init();
    double v[3] = {0.0, 0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += (int64_t)gridDim.x * blockDim.x) {
        const double rt = B.rtrue[i];
        const float rf = (float)rt, df = (float)D64[i];
        const float uf = rf / df;
        B.r[i] = rf;
        B.u[i] = uf;
        B.D[i] = df;
        B.y[i] = 0.0f;
        B.p[i] = 0.0f;
        B.s[i] = 0.0f;
        v[0] += rt * rt;
        v[1] += (double)rf * (double)uf;
        v[2] += (double)rf * (double)rf;
    }
    if (grid_sum3(v, B.partials, ticket)) {
        out[0] = v[0];
        out[1] = v[1];
        out[2] = v[2];
    }
}

// The solve is over: x += y, unless a reliable update (R0) folded y last.
__global__ void gear_fold_kernel(const GearBuffers B) {
    if (B.st->y_reset) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B.n; i += (int64_t)gridDim.x * blockDim.x)
        B.x[i] += (double)B.y[i];
}

// ---------------------------------------------------------------------------
// Host side.

static int update_blocks(int64_t n) {
    constexpr int per_sm = kUpdateV == 2 ? 5 : 4;
    int64_t b = ceil_div(ceil_div(n, kUpdateV), kVecThreads);
    if (b > 148 * per_sm) b = 148 * per_sm;
    return b < 1 ? 1 : (int)b;
}

cudaError_t launch_gear_init(const GearBuffers &B, const double *D64, unsigned *ticket, double *out,
                             cudaStream_t s) {
    gear_init_kernel<<<vec_blocks(B.n), kVecThreads, 0, s>>>(B, D64, ticket, out);
    return cudaGetLastError();
}

cudaError_t launch_gear_fold(const GearBuffers &B, cudaStream_t s) {
    gear_fold_kernel<<<vec_blocks(B.n), kVecThreads, 0, s>>>(B);
    return cudaGetLastError();
}

// Captures the launches `f` makes on `st` into `g` after `dep` (none if
// null); *last gets the node the capture ended with.
template <typename F>
static cudaError_t capture_into(cudaStream_t st, cudaGraph_t g, cudaGraphNode_t dep, F &&f, cudaGraphNode_t *last) {
    cudaError_t e = cudaStreamBeginCaptureToGraph(st, g, dep != nullptr ? &dep : nullptr, nullptr, dep != nullptr ? 1 : 0,
                                                  cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    f();
    cudaError_t le = cudaGetLastError();
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    cudaError_t ie = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd);
    cudaGraphNode_t ln = (ie == cudaSuccess && nd == 1) ? deps[0] : nullptr;
    cudaGraph_t out = nullptr;
    e = cudaStreamEndCapture(st, &out);
    if (le != cudaSuccess) return le;
    if (ie != cudaSuccess) return ie;
    if (e != cudaSuccess) return e;
    if (ln == nullptr) return cudaErrorStreamCaptureUnjoined;
    *last = ln;
    return cudaSuccess;
}

// Adds a conditional node of `type` on handle h after dep; *body gets its graph.
static cudaError_t add_conditional(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h,
                                   cudaGraphConditionalNodeType type, cudaGraphNode_t *node, cudaGraph_t *body) {
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = type;
    np.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(node, g, dep != nullptr ? &dep : nullptr, dep != nullptr ? 1 : 0, &np);
    if (e != cudaSuccess) return e;
    *body = np.conditional.phGraph_out[0];
    return cudaSuccess;
}

// The iteration's kernels for FP32 layout L32 and FP64 layout L64.
template <class L32, class L64>
static cudaError_t build_body(const GearBuffers &B, const L32 &l32, const L64 &l64, int chunk, cudaStream_t stream,
                              cudaGraph_t body, cudaGraphConditionalHandle hwhile, bool plain) {
    int sb = vec_blocks(l32.nslices_host * 32);
    if (sb > 148 * kGearBlocksPerSM) sb = 148 * kGearBlocksPerSM;
    const int rb = sb < 148 * 6 ? sb : 148 * 6;   // the reliable kernel holds 6 blocks per SM
    const int ub = update_blocks(B.n);
    cudaGraphNode_t prev = nullptr;
    if (plain) {   // every kernel every iteration; R0 and R1 return unless K2 asked for them
        for (int i = 0; i < chunk; i++) {
            cudaGraphNode_t last;
            const cudaGraphConditionalHandle none{};
            cudaError_t e = capture_into(stream, body, prev, [&] {
                gear_spmv_kernel<typename L32::Dev><<<sb, kVecThreads, 0, stream>>>(l32.dev, B);
                gear_update_kernel<kUpdateV, false><<<ub, kVecThreads, 0, stream>>>(B, none);
                gear_fold_ru_kernel<<<vec_blocks(B.n), kVecThreads, 0, stream>>>(B);
                gear_reliable_kernel<L64><<<rb, kVecThreads, 0, stream>>>(l64, B);
            }, &last);
            if (e != cudaSuccess) return e;
            prev = last;
        }
        return cudaSuccess;
    }
    for (int i = 0; i < chunk; i++) {
        cudaGraphConditionalHandle hif;
        cudaError_t e = cudaGraphConditionalHandleCreate(&hif, body, 0, 0);
        if (e != cudaSuccess) return e;
        cudaGraphNode_t k2, ifn;
        e = capture_into(stream, body, prev, [&] {
            gear_spmv_kernel<typename L32::Dev><<<sb, kVecThreads, 0, stream>>>(l32.dev, B);
            gear_update_kernel<kUpdateV><<<ub, kVecThreads, 0, stream>>>(B, hif);
        }, &k2);
        if (e != cudaSuccess) return e;
        cudaGraph_t ifbody;
        e = add_conditional(body, k2, hif, cudaGraphCondTypeIf, &ifn, &ifbody);
        if (e != cudaSuccess) return e;
        cudaGraphNode_t r1;
        e = capture_into(stream, ifbody, nullptr, [&] {
            gear_fold_ru_kernel<<<vec_blocks(B.n), kVecThreads, 0, stream>>>(B);
            gear_reliable_kernel<L64><<<rb, kVecThreads, 0, stream>>>(l64, B);
        }, &r1);
        if (e != cudaSuccess) return e;
        prev = ifn;
    }
    cudaGraphNode_t lk;
    return capture_into(stream, body, prev, [&] { gear_loop_kernel<<<1, 1, 0, stream>>>(B.st, hwhile); }, &lk);
}

// A device layout functor with the slice count known on the host.
template <class D>
struct HostLayout {
    using Dev = D;
    D dev;
    int64_t nslices_host;
};

cudaError_t build_gear_graph(const GearBuffers &B, const GearLayouts &L, int chunk, bool plain, cudaStream_t stream,
                             cudaGraphExec_t *exec, int *kernels_per_iteration) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle hw{};
    cudaGraph_t body = g;
    if (!plain) {
        cudaGraphNode_t wnode;
        e = cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) e = add_conditional(g, nullptr, hw, cudaGraphCondTypeWhile, &wnode, &body);
    }
    if (e == cudaSuccess) {
        const int64_t nsl = L.S.nslices;
        const SellRows<double, double, 4> sell64{nsl, L.S.perm, L.S.len, L.S.sptr, L.S.cols, L.S.vals};
        if (L.kind == 2) {
            const Q16Rows64 q64{L.Q};
            if (L.unroll == 2)
                e = build_body(B, HostLayout<Q16Rows32<2>>{{L.Q}, L.Q.nslices}, q64, chunk, stream, body, hw, plain);
            else
                e = build_body(B, HostLayout<Q16Rows32<1>>{{L.Q}, L.Q.nslices}, q64, chunk, stream, body, hw, plain);
        } else if (L.kind == 1) {
            switch (L.unroll) {
            case 2: e = build_body(B, HostLayout<PairRows32<2>>{{nsl, L.S2}, nsl}, sell64, chunk, stream, body, hw, plain); break;
            case 8: e = build_body(B, HostLayout<PairRows32<8>>{{nsl, L.S2}, nsl}, sell64, chunk, stream, body, hw, plain); break;
            default: e = build_body(B, HostLayout<PairRows32<4>>{{nsl, L.S2}, nsl}, sell64, chunk, stream, body, hw, plain); break;
            }
        } else {
            using S32_4 = SellRows<float, float, 4>;
            using S32_8 = SellRows<float, float, 8>;
            using S32_16 = SellRows<float, float, 16>;
            switch (L.unroll) {
            case 8: e = build_body(B, HostLayout<S32_8>{{nsl, L.S.perm, L.S.len, L.S.sptr, L.S.cols, L.S.vals32}, nsl}, sell64, chunk, stream, body, hw, plain); break;
            case 16: e = build_body(B, HostLayout<S32_16>{{nsl, L.S.perm, L.S.len, L.S.sptr, L.S.cols, L.S.vals32}, nsl}, sell64, chunk, stream, body, hw, plain); break;
            default: e = build_body(B, HostLayout<S32_4>{{nsl, L.S.perm, L.S.len, L.S.sptr, L.S.cols, L.S.vals32}, nsl}, sell64, chunk, stream, body, hw, plain); break;
            }
        }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (kernels_per_iteration != nullptr) *kernels_per_iteration = 2;
    return e;
}

cudaError_t build_pcg_loop_graph(cudaStream_t stream, void (*body)(void *ctx, cudaStream_t s), void *ctx,
                                 PcgState *st, bool plain, cudaGraphExec_t *exec) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    if (plain) {   // the chunk alone; the host loops
        cudaGraphNode_t last;
        e = capture_into(stream, g, nullptr, [&] { body(ctx, stream); }, &last);
        if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
        cudaGraphDestroy(g);
        return e;
    }
    cudaGraphConditionalHandle hw;
    cudaGraphNode_t wnode, last;
    cudaGraph_t wbody = nullptr;
    e = cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) e = add_conditional(g, nullptr, hw, cudaGraphCondTypeWhile, &wnode, &wbody);
    if (e == cudaSuccess)
        e = capture_into(stream, wbody, nullptr, [&] {
            body(ctx, stream);
            pcg_loop_kernel<<<1, 1, 0, stream>>>(st, hw);
        }, &last);
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    return e;
}

}  // namespace phgb
