// Element assembly on the device: element matrices and vectors, the DOF ->
// element incidence lists, and the deterministic row-owner assembly into CSR.
//
// Data layout in HBM (one system):
//   verts   f64 [nvert][3]           coordinates (PHG g->verts)
//   elems   i32 [nelem][4]           element vertices (PHG e->verts)
//   e2l     i32 [nelem][N]           vector index of each element basis
//   bdry    u8  [ndof]               Dirichlet flag per DOF
//   inc_ptr i32 [ndof+1], inc i32    per DOF, the incident (element, basis)
//                                    pairs as keys e*N+a, ascending
//   Ke      f64 [nelem][N][N]        element matrices (row a = basis a)
//   Km      u32 [nelem][ceil(N*N/32)] nonzero bits of Ke
//   Re      f64 [nelem][N]           element right-hand sides
//   ptr/cols/vals                    CSR (rows in first-touch order)
//   bptr/bcols/bvals                 saved boundary columns
//   rhs, diag                        f64 [ndof]
//
// The element kernel repeats the reference's floating-point operations one by
// one (explicit round-to-nearest intrinsics, no fused multiply-adds), so the
// element entries -- and therefore which entries are exactly zero and get
// dropped -- are identical to the reference's.  The row walk then visits each
// row's contributions in element order, which is the order the reference's
// element loop adds them in, so the assembled values are identical as well.
#include "common.cuh"
#include "assemble.h"

namespace phgb {

// ---------------------------------------------------------------------------
// Geometry: compute_jacobian (geom.c:103-169) and the volume
// (geom.c:46-78), operation for operation.
__device__ __forceinline__ void jacobian_vol(const double *x, double *J, double &vol) {
    double a[4][8];
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
        for (int i = 0; i < 3; i++) a[j][i] = x[3 * j + i];
        a[j][3] = 1.0;
#pragma unroll
        for (int i = 0; i < 4; i++) a[j][4 + i] = (i == j) ? 1.0 : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        double d = fabs(a[j][j]);
        int k = j;
#pragma unroll
        for (int i = j + 1; i < 4; i++) {
            const double t = fabs(a[i][j]);
            if (d < t) { d = t; k = i; }
        }
        // row swap, written as selects so the array stays in registers
#pragma unroll
        for (int r = j + 1; r < 4; r++) {
            const bool sw = (r == k);
#pragma unroll
            for (int i = j; i < 8; i++) {
                const double t = a[j][i], u = a[r][i];
                a[j][i] = sw ? u : t;
                a[r][i] = sw ? t : u;
            }
        }
        const double t = a[j][j];
        d = __ddiv_rn(1.0, t == 0. ? 1. : t);
#pragma unroll
        for (int i = j + 1; i < 8; i++) a[j][i] = rn_mul(a[j][i], d);
#pragma unroll
        for (int i = j + 1; i < 4; i++) {
            const double m = a[i][j];
#pragma unroll
            for (int c = j + 1; c < 8; c++) a[i][c] = rn_sub(a[i][c], rn_mul(m, a[j][c]));
        }
    }
#pragma unroll
    for (int j = 2; j >= 0; j--)
#pragma unroll
        for (int i = j + 1; i < 4; i++) {
            const double d = a[j][i];
#pragma unroll
            for (int c = 4; c < 8; c++) a[j][c] = rn_sub(a[j][c], rn_mul(d, a[i][c]));
        }
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int i = 0; i < 4; i++) J[4 * j + i] = a[i][j + 4];

    const double x0 = x[0], y0 = x[1], z0 = x[2];
    const double x1 = rn_sub(x[3], x0), y1 = rn_sub(x[4], y0), z1 = rn_sub(x[5], z0);
    const double x2 = rn_sub(x[6], x0), y2 = rn_sub(x[7], y0), z2 = rn_sub(x[8], z0);
    const double x3 = rn_sub(x[9], x0), y3 = rn_sub(x[10], y0), z3 = rn_sub(x[11], z0);
    const double s1 = rn_add(rn_add(rn_mul(rn_mul(x1, y2), z3), rn_mul(rn_mul(x2, y3), z1)),
                           rn_mul(rn_mul(y1, z2), x3));
    const double s2 = rn_add(rn_add(rn_mul(rn_mul(z1, y2), x3), rn_mul(rn_mul(y1, x2), z3)),
                           rn_mul(rn_mul(z2, y3), x1));
    vol = rn_mul(fabs(rn_sub(s1, s2)), 0x1.5555555555555p-3 /* 1/6 */);
}

// ---------------------------------------------------------------------------
// Element kernel.  A warp takes 32 elements at a time:
//   phase A  one thread per element: vertex gather, Jacobian and volume
//            (the long serial part), written to shared memory;
//   phase B  the warp walks its 32 elements one by one, lanes spread over
//            (basis, point) for the gradients and over basis pairs for the
//            matrix, then a coalesced store of the N x N element matrix.
// Outputs per element e:
//   Ke[e]   N x N stiffness, integral of grad phi_b . kappa grad phi_a with the
//           order-2(p-1) rule (phgQuadGradBasAGradBas, quad.c:5260-5344, basis
//           gradients as phgQuadGetBasisGradient, quad.c:3314-3421)
//           plus, when c = mass != 0, c times the mass matrix, integral of
//           phi_b phi_a with the order-2p rule (phgQuadBasABas with A = NULL,
//           quad.c:5582-5625), added as stiffness + c * mass the way
//           examples/simplest.c:68-72 writes the element matrix
//   Re[e]   N right-hand side entries, integral of f_h phi_a with the order-2p
//           rule (phgQuadDofTimesBas, quad.c:5481-5530; f_h at the points as
//           phgDofEval_, dof-utils.c:59-300)
template <int P>
struct ElemDims {
    static constexpr int N = P == 1 ? 4 : P == 2 ? 10 : 20;
    static constexpr int QK = P == 1 ? 1 : P == 2 ? 4 : 14;
    static constexpr int QR = P == 1 ? 4 : P == 2 ? 14 : 24;
    static constexpr int WARPS = 4;                       // warps per block
};

constexpr int kGeo = 18;   // doubles of geometry per element: J (16), volume, pad

// Row a of symmetric pair idx = a (a + 1) / 2 + b (b <= a), for N <= 20.
__device__ const unsigned char g_pair_a[210] = {
    0, 1, 1, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 4, 5, 5, 5, 5, 5, 5,
    6, 6, 6, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7, 7, 7, 8, 8, 8, 8, 8, 8, 8, 8, 8,
    9, 9, 9, 9, 9, 9, 9, 9, 9, 9, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10, 10,
    11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 11, 12, 12, 12, 12, 12, 12, 12, 12, 12, 12, 12, 12, 12,
    13, 13, 13, 13, 13, 13, 13, 13, 13, 13, 13, 13, 13, 13,
    14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14, 14,
    15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15,
    16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16,
    17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17, 17,
    18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18, 18,
    19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19, 19,
};

// Geometry: one thread per element, J (16) and the volume into geo[e][0..16].
__global__ void __launch_bounds__(128)
geometry_kernel(int64_t nelem, int64_t nvert, const double *__restrict__ verts, const int32_t *__restrict__ elems,
                double *__restrict__ geo, int *status) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += (int64_t)gridDim.x * blockDim.x) {
        double x[12];
        bool ok = true;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int32_t v = elems[4 * e + j];
            if (v < 0 || v >= nvert) {
                ok = false;
                x[3 * j] = x[3 * j + 1] = x[3 * j + 2] = 0.0;
            } else {
                x[3 * j] = verts[3 * (int64_t)v];
                x[3 * j + 1] = verts[3 * (int64_t)v + 1];
                x[3 * j + 2] = verts[3 * (int64_t)v + 2];
            }
        }
        if (!ok) atomicExch(status, PHGB_DEV_BAD_INDEX);
        bool fin = true;
#pragma unroll
        for (int t = 0; t < 12; t++) fin = fin && isfinite(x[t]);
        if (!fin) atomicExch(status, PHGB_DEV_NONFINITE);
        double J[16], vol;
        jacobian_vol(x, J, vol);
        double *o = geo + (size_t)e * kGeo;
#pragma unroll
        for (int t = 0; t < 16; t++) o[t] = J[t];
        o[16] = vol;
    }
}

// Quadrature weights, passed by value: every lane reads the same weight at
// the same time, so they are read from the kernel's parameter (constant)
// bank instead of through the load/store pipe the kernel is bound by.
struct ElemWeights {
    double wk[kElemMaxQK];
    double wr[kElemMaxQR];
};

// Element matrices and vectors: one warp per element.
template <int P>
__global__ void __launch_bounds__(ElemDims<P>::WARPS * 32)
element_kernel(int64_t nelem, int64_t ndof, const double *__restrict__ geo, const int32_t *__restrict__ e2l,
               const double *__restrict__ kappa, const double mass, const double *__restrict__ f,
               const ElemWeights Wt, const double *__restrict__ gk, const double *__restrict__ br,
               const double *__restrict__ brt,
               double *__restrict__ Ke, double *__restrict__ Re, int *status) {
    using D = ElemDims<P>;
    constexpr int N = D::N, QK = D::QK, QR = D::QR, W = D::WARPS;
    __shared__ double s_geo[W][kGeo + 1];       // J (16), volume, kappa
    // basis gradients at the stiffness points, component-major with the basis
    // index fastest (grad[(c * QK + q) * N + k]): lanes that read gradients
    // of different bases hit different banks
    __shared__ double s_grad[W][N * QK * 3];
    __shared__ double s_K[W][N * N];
    __shared__ double s_f[W][N];
    __shared__ double s_fq[W][QR];

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double *J = s_geo[w], *grad = s_grad[w], *K = s_K[w], *fl = s_f[w], *fq = s_fq[w];

    for (int64_t e = (int64_t)blockIdx.x * W + w; e < nelem; e += (int64_t)gridDim.x * W) {
        if (lane < 17) J[lane] = geo[(size_t)e * kGeo + lane];
        if (lane == 17) {
            const double kv = kappa != nullptr ? kappa[e] : 0.0;
            if (!isfinite(kv)) atomicExch(status, PHGB_DEV_NONFINITE);
            J[17] = kv;
        }
        // f_h at the element's nodes
        if (lane < N) {
            double fv = 0.0;
            if (f != nullptr) {
                const int32_t d = e2l[(size_t)e * N + lane];
                if (d < 0 || d >= ndof) atomicExch(status, PHGB_DEV_BAD_INDEX);
                else fv = f[d];
                if (!isfinite(fv)) atomicExch(status, PHGB_DEV_NONFINITE);
            }
            fl[lane] = fv;
        }
        __syncwarp();
        const double vol = J[16], kap = J[17];

        // basis gradients at the stiffness points
        constexpr int CS = QK * N;   // component stride of grad
        for (int idx = lane; idx < N * QK; idx += 32) {
            const int k = idx % N, q = idx / N;
            double *o = grad + q * N + k;
            if (P == 1) {
                o[0] = J[4 * k]; o[CS] = J[4 * k + 1]; o[2 * CS] = J[4 * k + 2];
            } else if (k < 4) {
                const double d = gk[(k * QK + q) * N + k];
                o[0] = rn_mul(d, J[4 * k]);
                o[CS] = rn_mul(d, J[4 * k + 1]);
                o[2 * CS] = rn_mul(d, J[4 * k + 2]);
            } else {
                const double *G = gk + q * N + k;
                const double g0 = G[0], g1 = G[CS], g2 = G[2 * CS], g3 = G[3 * CS];
#pragma unroll
                for (int c = 0; c < 3; c++)
                    o[c * CS] = rn_add(rn_add(rn_add(rn_mul(g0, J[c]), rn_mul(g1, J[4 + c])), rn_mul(g2, J[8 + c])),
                                       rn_mul(g3, J[12 + c]));
            }
        }
        for (int q = lane; q < QR; q += 32) {
            double v = 0.0;
            for (int k = 0; k < N; k++) v = rn_add(v, rn_mul(brt[k * QR + q], fl[k]));
            fq[q] = v;
        }
        __syncwarp();

        // symmetric pairs b <= a (pair idx = a (a + 1) / 2 + b, from a table)
        for (int idx = lane; idx < N * (N + 1) / 2; idx += 32) {
            const int a = __ldg(&g_pair_a[idx]);   // lanes read different entries: L1, not constant cache
            const int b = idx - a * (a + 1) / 2;
            double d = 0.;
#pragma unroll 4
            for (int q = 0; q < QK; q++) {
                const double *g1 = grad + q * N + b;
                const double *g2 = grad + q * N + a;
                const double d0 = rn_add(0., rn_add(rn_add(rn_mul(g1[0], g2[0]), rn_mul(g1[CS], g2[CS])),
                                                    rn_mul(g1[2 * CS], g2[2 * CS])));
                const double t = rn_mul(d0, Wt.wk[q]);
                d = rn_add(d, kappa != nullptr ? rn_mul(t, kap) : t);
            }
            double v = rn_mul(d, vol);
            if (mass != 0.0) {
                double dm = 0.;
                for (int q = 0; q < QR; q++) {
                    const double d0 = rn_add(0., rn_mul(br[q * N + b], br[q * N + a]));
                    dm = rn_add(dm, rn_mul(d0, Wt.wr[q]));
                }
                v = rn_add(v, rn_mul(mass, rn_mul(dm, vol)));
            }
            K[a * N + b] = v;
            K[b * N + a] = v;
        }
        if (lane < N) {
            double d = 0.0;
            for (int q = 0; q < QR; q++) d = rn_add(d, rn_mul(rn_mul(br[q * N + lane], Wt.wr[q]), fq[q]));
            Re[(size_t)e * N + lane] = rn_mul(d, vol);
        }
        __syncwarp();
        double *ke = Ke + (size_t)e * N * N;
        for (int t = lane; t < N * N; t += 32) ke[t] = K[t];
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Element kernel for P1 and P2: a lane per basis function, 32 / N elements
// per warp (P1 eight, P2 three).  Lane b computes the gradients of basis b
// at the stiffness points in registers and publishes them in shared memory;
// then it computes column b of the element matrix, reading the gradient of
// basis a (a = 0..N-1) with loads every lane of the element shares, and
// stores Ke[e][a][b] directly (the lanes of an element write a row's N
// consecutive entries).  Entry (a, b) and its mirror (b, a) come out bit for
// bit equal to the reference's single evaluation of the pair: each product of
// gradient components commutes and the sums run over the same components in
// the same order.  Every operation is the one the warp-per-element kernel
// performs (the reference's order, round-to-nearest, no contraction); what
// changes is where the operands live: the pair sums read 40 shared-memory
// words an element instead of hundreds, and the element matrix goes straight
// to global memory.
template <int P>
__global__ void __launch_bounds__(128, 6)   // 80 registers: 24 warps an SM (96 without the bound: 20)
element_lanes_kernel(int64_t nelem, int64_t ndof, const double *__restrict__ geo, const int32_t *__restrict__ e2l,
                     const double *__restrict__ kappa, const double mass, const double *__restrict__ f,
                     const ElemWeights Wt, const double *__restrict__ gk, const double *__restrict__ br,
                     const double *__restrict__ brt, double *__restrict__ Ke, double *__restrict__ Re, int *status) {
    using D = ElemDims<P>;
    constexpr int N = D::N, QK = D::QK, QR = D::QR, W = 4;
    constexpr int EPW = 32 / N;                  // elements per warp
    constexpr int CS = QK * N;                   // component stride of the gk table
    // gradient component c at point q of basis b at [b][q * 3 + c]: a basis'
    // gradients are one row of RW doubles, read with 16-byte loads; each
    // element's table is padded so that the EPW elements of a warp start in
    // different banks (a lane reads its element's row while the other
    // elements' lanes read theirs)
    constexpr int RW = (QK * 3 + 1) & ~1;               // doubles per basis row (even: 16-byte loads)
    constexpr int GW = RW * N;                          // doubles of one element's table
    constexpr int WANT = (32 / EPW) & ~3;               // bank offset (words) between elements
    constexpr int GPAD = ((((WANT - 2 * GW) % 32 + 32) % 32) / 2 + 1) & ~1;   // even: rows stay 16-byte aligned
    __shared__ __align__(16) double s_g[W][EPW][GW + GPAD];
    __shared__ double s_f[W][EPW][N];
    __shared__ double s_fq[W][EPW][QR];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sub = lane / N, b = lane - sub * N;
    const bool lane_ok = sub < EPW;
    const int sl = lane_ok ? sub : 0;
    double(*G)[RW] = reinterpret_cast<double(*)[RW]>(s_g[w][sl]);
    double *fl = s_f[w][sl], *fq = s_fq[w][sl];

    for (int64_t e0 = ((int64_t)blockIdx.x * W + w) * EPW; e0 < nelem; e0 += (int64_t)gridDim.x * W * EPW) {
        const int64_t e = e0 + sub;
        const bool act = lane_ok && e < nelem;
        const double *J = geo + (size_t)(act ? e : 0) * kGeo;
        double kap = 0.0;
        if (act && kappa != nullptr) {
            kap = kappa[e];
            if (b == 0 && !isfinite(kap)) atomicExch(status, PHGB_DEV_NONFINITE);
        }
        // gradients of basis b at the stiffness points
        double g[QK][3];
#pragma unroll
        for (int q = 0; q < QK; q++) {
            if (P == 1) {
#pragma unroll
                for (int c = 0; c < 3; c++) g[q][c] = act ? J[4 * b + c] : 0.0;
            } else if (b < 4) {
                const double d = gk[(b * QK + q) * N + b];
#pragma unroll
                for (int c = 0; c < 3; c++) g[q][c] = rn_mul(d, act ? J[4 * b + c] : 0.0);
            } else {
                const double *Gk = gk + q * N + b;
                const double g0 = Gk[0], g1 = Gk[CS], g2 = Gk[2 * CS], g3 = Gk[3 * CS];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const double j0 = act ? J[c] : 0.0, j1 = act ? J[4 + c] : 0.0;
                    const double j2 = act ? J[8 + c] : 0.0, j3 = act ? J[12 + c] : 0.0;
                    g[q][c] = rn_add(rn_add(rn_add(rn_mul(g0, j0), rn_mul(g1, j1)), rn_mul(g2, j2)), rn_mul(g3, j3));
                }
            }
        }
        double fv = 0.0;
        if (act && f != nullptr) {
            const int32_t d = e2l[(size_t)e * N + b];
            if (d < 0 || d >= ndof) atomicExch(status, PHGB_DEV_BAD_INDEX);
            else fv = f[d];
            if (!isfinite(fv)) atomicExch(status, PHGB_DEV_NONFINITE);
        }
        if (lane_ok) {
#pragma unroll
            for (int q = 0; q < QK; q++)
#pragma unroll
                for (int c = 0; c < 3; c++) G[b][q * 3 + c] = g[q][c];
            fl[b] = fv;
        }
        __syncwarp();
        // f_h at the RHS points (phgDofEval_: sum over the element's nodes)
        if (lane_ok)
            for (int q = b; q < QR; q += N) {
                double v = 0.0;
                for (int k = 0; k < N; k++) v = rn_add(v, rn_mul(brt[k * QR + q], fl[k]));
                fq[q] = v;
            }
        __syncwarp();
        const double vol = act ? J[16] : 0.0;
        // column b of the element matrix
        for (int a = 0; a < N; a++) {
            double ga[RW];   // basis a's gradients, RW / 2 16-byte loads
#pragma unroll
            for (int k = 0; k < RW; k += 2) {
                const double2 t2 = *reinterpret_cast<const double2 *>(&G[a][k]);
                ga[k] = t2.x;
                ga[k + 1] = t2.y;
            }
            double d = 0.;
#pragma unroll
            for (int q = 0; q < QK; q++) {
                const double d0 = rn_add(0., rn_add(rn_add(rn_mul(g[q][0], ga[q * 3]), rn_mul(g[q][1], ga[q * 3 + 1])),
                                                    rn_mul(g[q][2], ga[q * 3 + 2])));
                const double t = rn_mul(d0, Wt.wk[q]);
                d = rn_add(d, kappa != nullptr ? rn_mul(t, kap) : t);
            }
            double v = rn_mul(d, vol);
            if (mass != 0.0) {
                double dm = 0.;
                for (int q = 0; q < QR; q++) {
                    const double d0 = rn_add(0., rn_mul(br[q * N + b], br[q * N + a]));
                    dm = rn_add(dm, rn_mul(d0, Wt.wr[q]));
                }
                v = rn_add(v, rn_mul(mass, rn_mul(dm, vol)));
            }
            if (act) Ke[((size_t)e * N + a) * N + b] = v;
        }
        if (act) {
            double d = 0.0;
            for (int q = 0; q < QR; q++) d = rn_add(d, rn_mul(rn_mul(br[q * N + b], Wt.wr[q]), fq[q]));
            Re[(size_t)e * N + b] = rn_mul(d, vol);
        }
        __syncwarp();
    }
}

// Element matrices and vectors with N / 2 lanes per element (P2: six
// elements a warp): lane j owns the columns j and j + N / 2, so that each
// row of basis gradients it reads from shared memory serves two entries.
// Every entry takes the operations of element_lanes_kernel in the same order
// (round-to-nearest, no contraction) but one, so the matrices are the same
// bits: the dot products' leading "0 +" is left out, since it only turns a
// -0 into +0, and a -0 term added to the running sum (which starts at +0 and
// so never is -0) leaves the same sum.
template <int P>
__global__ void __launch_bounds__(128, 4)   // 128 registers, no spills (5 blocks: 96 registers, 1% slower)
element_cols2_kernel(int64_t nelem, int64_t ndof, const double *__restrict__ geo, const int32_t *__restrict__ e2l,
                     const double *__restrict__ kappa, const double mass, const double *__restrict__ f,
                     const ElemWeights Wt, const double *__restrict__ gk, const double *__restrict__ br,
                     const double *__restrict__ brt, double *__restrict__ Ke, double *__restrict__ Re, int *status) {
    using D = ElemDims<P>;
    constexpr int N = D::N, QK = D::QK, QR = D::QR, W = 4, H = N / 2;
    static_assert(N % 2 == 0, "columns are paired");
    constexpr int EPW = 32 / H;                  // elements per warp
    constexpr int CS = QK * N;                   // component stride of the gk table
    constexpr int RW = (QK * 3 + 1) & ~1;        // doubles per basis row (even: 16-byte loads)
    constexpr int GW = RW * N;
    constexpr int WANT = (32 / EPW) & ~3;
    constexpr int GPAD = ((((WANT - 2 * GW) % 32 + 32) % 32) / 2 + 1) & ~1;
    __shared__ __align__(16) double s_g[W][EPW][GW + GPAD];
    __shared__ double s_f[W][EPW][N];
    __shared__ double s_fq[W][EPW][QR];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sub = lane / H, j = lane - sub * H;
    const bool lane_ok = sub < EPW;
    const int sl = lane_ok ? sub : 0;
    const int b1 = j, b2 = j + H;
    double(*G)[RW] = reinterpret_cast<double(*)[RW]>(s_g[w][sl]);
    double *fl = s_f[w][sl], *fq = s_fq[w][sl];

    // gradients of basis b at the stiffness points (as element_lanes_kernel)
    auto grad = [&](const double *J, bool act, int b, double (&g)[QK][3]) {
#pragma unroll
        for (int q = 0; q < QK; q++) {
            if (P == 1) {
#pragma unroll
                for (int c = 0; c < 3; c++) g[q][c] = act ? J[4 * b + c] : 0.0;
            } else if (b < 4) {
                const double d = gk[(b * QK + q) * N + b];
#pragma unroll
                for (int c = 0; c < 3; c++) g[q][c] = rn_mul(d, act ? J[4 * b + c] : 0.0);
            } else {
                const double *Gk = gk + q * N + b;
                const double g0 = Gk[0], g1 = Gk[CS], g2 = Gk[2 * CS], g3 = Gk[3 * CS];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const double j0 = act ? J[c] : 0.0, j1 = act ? J[4 + c] : 0.0;
                    const double j2 = act ? J[8 + c] : 0.0, j3 = act ? J[12 + c] : 0.0;
                    g[q][c] = rn_add(rn_add(rn_add(rn_mul(g0, j0), rn_mul(g1, j1)), rn_mul(g2, j2)), rn_mul(g3, j3));
                }
            }
        }
    };

    for (int64_t e0 = ((int64_t)blockIdx.x * W + w) * EPW; e0 < nelem; e0 += (int64_t)gridDim.x * W * EPW) {
        const int64_t e = e0 + sub;
        const bool act = lane_ok && e < nelem;
        const double *J = geo + (size_t)(act ? e : 0) * kGeo;
        double kap = 0.0;
        if (act && kappa != nullptr) {
            kap = kappa[e];
            if (j == 0 && !isfinite(kap)) atomicExch(status, PHGB_DEV_NONFINITE);
        }
        double g1[QK][3], g2[QK][3];
        grad(J, act, b1, g1);
        grad(J, act, b2, g2);
        double fv1 = 0.0, fv2 = 0.0;
        if (act && f != nullptr) {
            const int32_t d1 = e2l[(size_t)e * N + b1], d2 = e2l[(size_t)e * N + b2];
            if (d1 < 0 || d1 >= ndof) atomicExch(status, PHGB_DEV_BAD_INDEX);
            else fv1 = f[d1];
            if (d2 < 0 || d2 >= ndof) atomicExch(status, PHGB_DEV_BAD_INDEX);
            else fv2 = f[d2];
            if (!isfinite(fv1) || !isfinite(fv2)) atomicExch(status, PHGB_DEV_NONFINITE);
        }
        if (lane_ok) {
#pragma unroll
            for (int q = 0; q < QK; q++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    G[b1][q * 3 + c] = g1[q][c];
                    G[b2][q * 3 + c] = g2[q][c];
                }
            fl[b1] = fv1;
            fl[b2] = fv2;
        }
        __syncwarp();
        // f_h at the RHS points (phgDofEval_: sum over the element's nodes)
        if (lane_ok)
            for (int q = j; q < QR; q += H) {
                double v = 0.0;
                for (int k = 0; k < N; k++) v = rn_add(v, rn_mul(brt[k * QR + q], fl[k]));
                fq[q] = v;
            }
        __syncwarp();
        const double vol = act ? J[16] : 0.0;
        double *Ke_e = Ke + (size_t)(act ? e : 0) * N * N;
        // columns b1 and b2 of the element matrix
        for (int a = 0; a < N; a++) {
            double ga[RW];
#pragma unroll
            for (int k = 0; k < RW; k += 2) {
                const double2 t2 = *reinterpret_cast<const double2 *>(&G[a][k]);
                ga[k] = t2.x;
                ga[k + 1] = t2.y;
            }
            double d1 = 0., d2 = 0.;
#pragma unroll
            for (int q = 0; q < QK; q++) {
                const double x1 = rn_add(rn_add(rn_mul(g1[q][0], ga[q * 3]), rn_mul(g1[q][1], ga[q * 3 + 1])),
                                         rn_mul(g1[q][2], ga[q * 3 + 2]));
                const double x2 = rn_add(rn_add(rn_mul(g2[q][0], ga[q * 3]), rn_mul(g2[q][1], ga[q * 3 + 1])),
                                         rn_mul(g2[q][2], ga[q * 3 + 2]));
                const double t1 = rn_mul(x1, Wt.wk[q]), t2 = rn_mul(x2, Wt.wk[q]);
                d1 = rn_add(d1, kappa != nullptr ? rn_mul(t1, kap) : t1);
                d2 = rn_add(d2, kappa != nullptr ? rn_mul(t2, kap) : t2);
            }
            double v1 = rn_mul(d1, vol), v2 = rn_mul(d2, vol);
            if (mass != 0.0) {
                double m1 = 0., m2 = 0.;
                for (int q = 0; q < QR; q++) {
                    const double ba = br[q * N + a];
                    m1 = rn_add(m1, rn_mul(rn_mul(br[q * N + b1], ba), Wt.wr[q]));
                    m2 = rn_add(m2, rn_mul(rn_mul(br[q * N + b2], ba), Wt.wr[q]));
                }
                v1 = rn_add(v1, rn_mul(mass, rn_mul(m1, vol)));
                v2 = rn_add(v2, rn_mul(mass, rn_mul(m2, vol)));
            }
            if (act) {
                Ke_e[a * N + b1] = v1;
                Ke_e[a * N + b2] = v2;
            }
        }
        if (act) {
            double r1 = 0.0, r2 = 0.0;
            for (int q = 0; q < QR; q++) {
                r1 = rn_add(r1, rn_mul(rn_mul(br[q * N + b1], Wt.wr[q]), fq[q]));
                r2 = rn_add(r2, rn_mul(rn_mul(br[q * N + b2], Wt.wr[q]), fq[q]));
            }
            Re[(size_t)e * N + b1] = rn_mul(r1, vol);
            Re[(size_t)e * N + b2] = rn_mul(r2, vol);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// DOF -> (element, basis) incidence lists.

__global__ void inc_count_kernel(int64_t nkeys, int N, int64_t ndof, const int32_t *__restrict__ e2l,
                                 int32_t *__restrict__ cnt, int *status) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nkeys;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = e2l[t];
        if (d < 0 || d >= ndof) { atomicExch(status, PHGB_DEV_BAD_INDEX); continue; }
        atomicAdd(&cnt[d], 1);
    }
}

__global__ void inc_fill_kernel(int64_t nkeys, int64_t ndof, const int32_t *__restrict__ e2l,
                                const int32_t *__restrict__ inc_ptr, int32_t *__restrict__ cursor,
                                int32_t *__restrict__ inc) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nkeys;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = e2l[t];
        if (d < 0 || d >= ndof) continue;
        const int32_t pos = atomicAdd(&cursor[d], 1);
        inc[inc_ptr[d] + pos] = (int32_t)t;   // key = e * N + a
    }
}

// Sorts each DOF's short incidence list ascending (element order).
__global__ void inc_sort_kernel(int64_t ndof, const int32_t *__restrict__ inc_ptr,
                                int32_t *__restrict__ inc) {
    for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < ndof;
         d += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = inc_ptr[d], n = inc_ptr[d + 1] - b;
        int32_t *v = inc + b;
        for (int i = 1; i < n; i++) {
            const int32_t key = v[i];
            int j = i - 1;
            while (j >= 0 && v[j] > key) { v[j + 1] = v[j]; j--; }
            v[j + 1] = key;
        }
    }
}

// ---------------------------------------------------------------------------
// Exclusive scan of int32 counts (three phases), with the total.
constexpr int kScanBlock = 1024;

__global__ void scan_local_kernel(int64_t n, const int32_t *__restrict__ in, int32_t *__restrict__ out,
                                  int64_t *__restrict__ block_sums) {
    __shared__ int64_t s[kScanBlock];
    const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
    const int64_t v = i < n ? in[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
        const int64_t t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) out[i] = (int32_t)(s[threadIdx.x] - v);   // block-local exclusive
    if (threadIdx.x == kScanBlock - 1) block_sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void scan_blocks_kernel(int64_t nb, int64_t *__restrict__ block_sums, int64_t *__restrict__ total) {
    // single block: serial per thread chunk, then across threads
    __shared__ int64_t s[1024];
    const int64_t chunk = (nb + blockDim.x - 1) / blockDim.x;
    const int64_t b0 = threadIdx.x * chunk, b1 = min(nb, b0 + chunk);
    int64_t acc = 0;
    for (int64_t b = b0; b < b1; b++) acc += block_sums[b];
    s[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t run = 0;
        for (int t = 0; t < (int)blockDim.x; t++) { const int64_t c = s[t]; s[t] = run; run += c; }
        *total = run;
    }
    __syncthreads();
    acc = s[threadIdx.x];
    for (int64_t b = b0; b < b1; b++) { const int64_t c = block_sums[b]; block_sums[b] = acc; acc += c; }
}

__global__ void scan_add_kernel(int64_t n, int32_t *__restrict__ out, const int64_t *__restrict__ block_sums,
                                const int64_t *__restrict__ total) {
    const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n) out[i] = (int32_t)(out[i] + block_sums[blockIdx.x]);
    if (i == n) out[n] = (int32_t)*total;
}

// ---------------------------------------------------------------------------
// Row walk: G lanes per row (G >= N; 32/G rows per warp side by side), one
// pass.  For an interior row the lane group visits the row's incidences in
// element order; lane j handles element column j, skips exact zeros
// (phgMatAddEntries_, matvec.c:5459-5461), finds or appends the column
// (add_columns_to_row, matvec.c:3286-3321: first-touch order) through the
// group's open-addressing table in shared memory, and accumulates the value.
// Boundary columns are then separated from the row as save_bdry_columns does
// (matvec.c:4430-4488) and lifted into the RHS as update_rhs does
// (solver.c:707-725).  A Dirichlet row is the sum of the unit rows of its
// elements (phgDofDirichletBC, dof-utils.c:1369-1392).
//
// The row's entries go to a scratch region sized by the row's incidences
// (incidences x N slots, at inc_ptr[d] * N; the row cannot be longer):
// kept entries from the front in first-touch order, saved boundary columns
// from the back in reverse.  The counts are scanned into the CSR row
// pointers and compact_kernel copies the regions into the CSR arrays.
template <int N>
struct WalkCfg {
    static constexpr int G = N <= 8 ? 8 : N <= 16 ? 16 : 32;   // lanes per row
    static constexpr int R = 32 / G;                            // rows per warp
    static constexpr int HS = N == 4 ? 128 : N == 10 ? 256 : 512;
    static constexpr int MAXROW = HS / 2;
    static constexpr int WARPS = 4;
    static constexpr bool LONG = false;   // overflowing rows go to the list
};

// The pattern a build records for the next ones (phgGpuBuildLinearSystem
// with the same mesh and DOF map): per contribution (row incidence, element
// column) its first-touch position in the row or kSlotZero (an exact zero,
// dropped); per first-touch position its place among the row's kept entries
// (k) or, with kTmapBdry set, among its saved boundary columns (j).
constexpr uint16_t kSlotZero = 0xffff;
constexpr uint16_t kTmapBdry = 0x8000;

// The second pass over the rows the first one could not hold (high-valence
// vertices of locally refined meshes): a warp per row, a table of 2048 slots
// for up to 1024 entries.
template <int N>
struct LongWalkCfg {
    static constexpr int G = 32;
    static constexpr int R = 1;
    static constexpr int HS = 2048;
    static constexpr int MAXROW = 1024;
    static constexpr int WARPS = 1;
    static constexpr bool LONG = true;    // an overflowing row is an error
};

__device__ __forceinline__ unsigned hash32(int32_t c) { return (unsigned)c * 2654435761u; }

// Sum of g_k added mult times (the Dirichlet row's RHS, phgVecAddEntries_).
__device__ __forceinline__ double bdry_rhs(const double *g, int32_t k, int mult) {
    if (g == nullptr) return 0.0;
    const double v = g[k];
    if (v == 0.0) return 0.0;
    double s = 0.0;
    for (int i = 0; i < mult; i++) s = rn_add(s, v);
    return s;
}

template <int N, class C>
__global__ void __launch_bounds__(C::WARPS * 32, C::LONG ? 1 : 8)
row_walk_kernel(int64_t ndof, const int32_t *__restrict__ inc_ptr, const int32_t *__restrict__ inc,
                const int32_t *__restrict__ e2l, const uint8_t *__restrict__ bdry,
                const double *__restrict__ Ke, const double *__restrict__ Re, const double *__restrict__ g,
                int32_t *__restrict__ cnt_keep, int32_t *__restrict__ cnt_bdry,
                int32_t *__restrict__ sc_cols, double *__restrict__ sc_vals,
                double *__restrict__ rhs, double *__restrict__ diag, int *status,
                int32_t *__restrict__ over_list, int *nover, uint16_t *__restrict__ slot,
                uint16_t *__restrict__ tmap, int32_t *__restrict__ dpos) {
    constexpr int G = C::G, R = C::R, HS = C::HS, MAXROW = C::MAXROW, W = C::WARPS;
    __shared__ int32_t s_key[W][R][HS];
    __shared__ int16_t s_pos[W][R][HS];
    __shared__ int32_t s_col[W][R][MAXROW];
    __shared__ double s_val[W][R][MAXROW];

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int grp = lane / G, gl = lane % G;
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (grp * G);
    const unsigned lt_mask = (1u << lane) - 1u;
    int32_t *key = s_key[w][grp];
    int16_t *hpos = s_pos[w][grp];
    int32_t *scol = s_col[w][grp];
    double *sval = s_val[w][grp];

    const int64_t nwarps = (int64_t)gridDim.x * W;
    // the first pass walks every row, the second the listed ones
    const int64_t nrows = C::LONG ? (int64_t)*nover : ndof;
    for (int64_t wb = ((int64_t)blockIdx.x * W + w) * R; wb < nrows; wb += nwarps * R) {
        const int64_t d = C::LONG ? (wb + grp < nrows ? (int64_t)over_list[wb + grp] : ndof) : wb + grp;
        const bool active = d < ndof;
        int32_t i0 = 0, i1 = 0;
        bool isb = false;
        if (active) {
            i0 = inc_ptr[d];
            i1 = inc_ptr[d + 1];
            isb = bdry[d] != 0;
        }
        // the scratch region of row d
        const int64_t rbase = (int64_t)i0 * N, rcap = (int64_t)(i1 - i0) * N;
        if (active && isb && gl == 0) {
            const int mult = i1 - i0;
            if (g != nullptr && !isfinite(g[d])) atomicExch(status, PHGB_DEV_NONFINITE);
            double m = 0.0;
            for (int i = 0; i < mult; i++) m = rn_add(m, 1.0);
            if (mult > 0) {
                sc_cols[rbase] = (int32_t)d;
                sc_vals[rbase] = m;
                sc_cols[rbase + rcap - 1] = (int32_t)d;
                sc_vals[rbase + rcap - 1] = m;
            }
            cnt_keep[d] = mult > 0 ? 1 : 0;
            cnt_bdry[d] = mult > 0 ? 1 : 0;
            diag[d] = m;
            rhs[d] = bdry_rhs(g, (int32_t)d, mult);
        }
        const bool walk = active && !isb;
        const int nwalk = walk ? i1 - i0 : 0;
        int maxwalk = nwalk;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) maxwalk = max(maxwalk, __shfl_xor_sync(0xffffffffu, maxwalk, o));
        if (maxwalk == 0) continue;   // warp-uniform

        for (int t = gl; t < HS; t += G) key[t] = -1;
        __syncwarp();
        int L = 0;
        bool overflow = false;

        // Incidence keys come G at a time: lane gl of the group holds entry
        // gl of the current chunk (incA) and of the next one (incB); a key is
        // read with a shuffle.  The element data of incidence ii + 3 is loaded
        // while incidence ii is processed; the loaded words are only
        // inspected when they are used, so the loads stay in flight.
        auto inc_at = [&](int j) -> int32_t { return j < nwalk ? __ldg(&inc[i0 + j]) : 0; };
        int32_t incA = inc_at(gl), incB = inc_at(G + gl);
        // the element RHS entries of the first two chunks, loaded now and
        // summed after the walk (their loads complete behind it)
        const double reA = gl < nwalk ? __ldg(&Re[incA]) : 0.0;
        const double reB = G + gl < nwalk ? __ldg(&Re[incB]) : 0.0;
        struct Pf {
            int32_t c;
            double v;
            int ok;
        };
        auto load = [&](int j, Pf &f) {
            const int32_t kk = __shfl_sync(0xffffffffu, incA, j % G, G);
            f.ok = (j < nwalk && gl < N) ? 1 : 0;
            f.c = -1;
            f.v = 0.0;
            if (f.ok) {
                const int32_t e = kk / N, a = kk - e * N;
                f.c = e2l[(size_t)e * N + gl];
                f.v = Ke[((size_t)e * N + a) * N + gl];
            }
        };
        constexpr int kPf = 3;   // prefetch distance (incidences)
        Pf f0, f1, f2;
        load(0, f0);
        load(1, f1);
        load(2, f2);
        for (int ii = 0; ii < maxwalk; ii++) {
            const int j = ii + kPf;
            if (j % G == 0) { incA = incB; incB = inc_at(j + G + gl); }
            Pf f3;
            load(j, f3);
            const int32_t col = f0.c;
            const double v = f0.v;
            const bool nz = f0.ok != 0 && v != 0.0;
            int pos = -1;
            if (nz) {
                unsigned h = hash32(col) & (HS - 1);
                for (int probe = 0; probe < HS; probe++) {
                    const int32_t k = key[h];
                    if (k == col) { pos = hpos[h]; break; }
                    if (k == -1) break;
                    h = (h + 1) & (HS - 1);
                }
            }
            const unsigned newm = __ballot_sync(0xffffffffu, nz && pos < 0) & gmask;
            if (nz && pos < 0) {
                pos = L + __popc(newm & lt_mask);
                if (pos < MAXROW) {
                    unsigned h = hash32(col) & (HS - 1);
                    for (int probe = 0; probe < HS; probe++) {
                        if (atomicCAS(&key[h], -1, col) == -1) { hpos[h] = (int16_t)pos; break; }
                        h = (h + 1) & (HS - 1);
                    }
                    scol[pos] = col;
                    sval[pos] = v;
                } else {
                    overflow = true;
                }
            } else if (nz) {
                sval[pos] = rn_add(sval[pos], v);
            }
            // the pattern of later builds: where this contribution went (its
            // first-touch position in the row), or that it was an exact zero
            if (slot != nullptr && f0.ok)
                slot[((int64_t)i0 + ii) * N + gl] = nz ? (uint16_t)min(pos, MAXROW) : kSlotZero;
            L += __popc(newm);
            f0 = f1; f1 = f2; f2 = f3;
            __syncwarp();
        }
        const bool bad = overflow || L > MAXROW;
        const unsigned badm = __ballot_sync(0xffffffffu, bad) & gmask;
        if (badm != 0 && gl == 0) {
            if (C::LONG) atomicExch(status, PHGB_DEV_ROW_OVERFLOW);
            else over_list[atomicAdd(nover, 1)] = (int32_t)d;   // assembled by the second pass
        }

        // emit kept columns (front) and saved boundary columns (back, reversed),
        // in first-touch order.  Lanes also evaluate, in parallel, the lift
        // term of each boundary column (rhs_k * a_dk / D_kk, solver.c:716-724);
        // it replaces the column's value in s_val once the value is emitted.
        const bool emit = walk && badm == 0;
        int nk = 0, nb = 0;
        double dg = 0.0;
        int maxL = emit ? L : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) maxL = max(maxL, __shfl_xor_sync(0xffffffffu, maxL, o));
        for (int base = 0; base < maxL; base += G) {
            const int t = base + gl;
            bool isbc = false;
            const bool valid = emit && t < L;
            int32_t c = 0;
            double val = 0.0;
            if (valid) {
                c = scol[t];
                val = sval[t];
                isbc = (c != d) && bdry[c];
                if (c == d) dg = val;
                double term = 0.0;
                if (isbc) {
                    const int mult = inc_ptr[c + 1] - inc_ptr[c];
                    double Dk = 0.0;
                    for (int m = 0; m < mult; m++) Dk = rn_add(Dk, 1.0);
                    const double rk = bdry_rhs(g, c, mult);
                    term = __ddiv_rn(rn_mul(rn_mul(1.0, rk), val), Dk);
                }
                sval[t] = term;
                if (!isbc) scol[t] = -1;   // only boundary columns remain for the lift below
            }
            const unsigned km = __ballot_sync(0xffffffffu, valid && !isbc) & gmask;
            const unsigned bm = __ballot_sync(0xffffffffu, valid && isbc) & gmask;
            if (valid && !isbc) {
                const int k = nk + __popc(km & lt_mask);
                const int64_t q = rbase + k;
                sc_cols[q] = c;
                sc_vals[q] = val;
                if (tmap != nullptr) tmap[rbase + t] = (uint16_t)k;
                if (dpos != nullptr && c == d) dpos[d] = k;
            }
            if (valid && isbc) {
                const int j = nb + __popc(bm & lt_mask);
                const int64_t q = rbase + rcap - 1 - j;
                sc_cols[q] = c;
                sc_vals[q] = val;
                if (tmap != nullptr) tmap[rbase + t] = (uint16_t)(kTmapBdry | j);
            }
            nk += __popc(km);
            nb += __popc(bm);
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) dg += __shfl_xor_sync(0xffffffffu, dg, o, G);   // one lane holds it
        // element right-hand sides of this row, loaded by the lanes in parallel
        // and added by the group's first lane in element order (zeros skipped)
        double r = 0.0;
        for (int t = 0; t < G; t++) {
            const double ba = __shfl_sync(0xffffffffu, reA, t, G);
            if (gl == 0 && t < nwalk && ba != 0.0) r = rn_add(r, ba);
        }
        for (int t = 0; t < G; t++) {
            const double bb = __shfl_sync(0xffffffffu, reB, t, G);
            if (gl == 0 && G + t < nwalk && bb != 0.0) r = rn_add(r, bb);
        }
        const int maxinc = __reduce_max_sync(0xffffffffu, (unsigned)(emit ? i1 - i0 : 0));
        for (int base = 2 * G; base < maxinc; base += G) {
            const int ii = base + gl;
            const double bb = (emit && ii < i1 - i0) ? Re[inc[i0 + ii]] : 0.0;
            for (int t = 0; t < G; t++) {
                const double bt = __shfl_sync(0xffffffffu, bb, t, G);
                if (gl == 0 && base + t < i1 - i0 && bt != 0.0) r = rn_add(r, bt);
            }
        }
        __syncwarp();
        if (emit && gl == 0) {
            cnt_keep[d] = nk;
            cnt_bdry[d] = nb;
            diag[d] = dg;
            // lift the boundary columns in first-touch order: r -= term
            // (rows without boundary columns, most of them, skip the scan)
            if (nb > 0)
                for (int t = 0; t < L; t++)
                    if (scol[t] >= 0) r = rn_sub(r, sval[t]);
            rhs[d] = r;
        }
        __syncwarp();
    }
}

// A later build on the same pattern: the rows' values from the recorded
// slots, without the column search.  Per row, the contributions are added in
// element order at their recorded first-touch positions (so every entry is
// the same sum in the same order as the full walk makes), then written to
// their places in the CSR and the saved boundary columns, with the RHS
// lifted as the walk does.  A contribution whose zero/non-zero status
// differs from the recorded one means the pattern changed (status
// PHGB_DEV_PATTERN_CHANGED): the caller runs the full walk instead.
template <int N, class C>
__global__ void __launch_bounds__(C::WARPS * 32, C::LONG ? 1 : 8)
value_walk_kernel(int64_t ndof, const int32_t *__restrict__ inc_ptr, const int32_t *__restrict__ inc,
                  const uint8_t *__restrict__ bdry, const double *__restrict__ Ke, const double *__restrict__ Re,
                  const double *__restrict__ g, const uint16_t *__restrict__ slot, const uint16_t *__restrict__ tmap,
                  const int32_t *__restrict__ dpos, const int32_t *__restrict__ ptr,
                  const int32_t *__restrict__ bptr, const int32_t *__restrict__ bcols, double *__restrict__ vals,
                  double *__restrict__ bvals, double *__restrict__ rhs, double *__restrict__ diag, int *status,
                  const int32_t *__restrict__ over_list, const int *nover) {
    constexpr int G = C::G, R = C::R, MAXROW = C::MAXROW, W = C::WARPS;
    constexpr int TPL = C::LONG ? 1 : MAXROW / G;   // first-touch places a lane prefetches
    static_assert(N % 2 == 0, "element rows are staged as 16-byte pairs");
    __shared__ double s_val[W][R][MAXROW];
    __shared__ uint8_t s_isb[W][R][MAXROW];
    __shared__ __align__(16) double s_ke[W][R][G][N];     // staged element rows of G incidences
    __shared__ __align__(4) uint16_t s_sl[W][R][G][N];    // and their recorded slots
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int grp = lane / G, gl = lane % G;
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (grp * G);
    double *sval = s_val[w][grp];
    uint8_t *sisb = s_isb[w][grp];

    const int64_t nwarps = (int64_t)gridDim.x * W;
    const int64_t nrows = C::LONG ? (int64_t)*nover : ndof;
    for (int64_t wb = ((int64_t)blockIdx.x * W + w) * R; wb < nrows; wb += nwarps * R) {
        const int64_t d = C::LONG ? (wb + grp < nrows ? (int64_t)over_list[wb + grp] : ndof) : wb + grp;
        const bool active = d < ndof;
        int32_t i0 = 0, i1 = 0, p0 = 0, nk = 0, b0 = 0, nb = 0, dk = -1;
        bool isb = false;
        if (active) {
            i0 = inc_ptr[d];
            i1 = inc_ptr[d + 1];
            isb = bdry[d] != 0;
            p0 = ptr[d];
            nk = ptr[d + 1] - p0;
            b0 = bptr[d];
            nb = bptr[d + 1] - b0;
            dk = dpos[d];
        }
        const int L = nk + nb;
        if (active && isb && gl == 0) {   // the Dirichlet row, as the walk makes it
            const int mult = i1 - i0;
            if (g != nullptr && !isfinite(g[d])) atomicExch(status, PHGB_DEV_NONFINITE);
            double m = 0.0;
            for (int i = 0; i < mult; i++) m = rn_add(m, 1.0);
            if (mult > 0) {
                vals[p0] = m;
                bvals[b0] = m;
            }
            diag[d] = m;
            rhs[d] = bdry_rhs(g, (int32_t)d, mult);
        }
        // rows the first pass cannot hold are the second pass's
        const bool mine = C::LONG ? true : L <= MAXROW;
        const bool walk = active && !isb && mine;
        const int nwalk = walk ? i1 - i0 : 0;
        const int maxwalk = __reduce_max_sync(0xffffffffu, (unsigned)nwalk);
        if (maxwalk == 0) continue;   // warp-uniform
        const int Lw = walk ? L : 0;
        // the row's first-touch map, fetched now so that it is here when the
        // values are (first pass: each lane's places gl, gl + G, ...)
        uint16_t tm[TPL];
        if (!C::LONG) {
#pragma unroll
            for (int k = 0; k < TPL; k++) {
                const int t = gl + k * G;
                tm[k] = t < Lw ? __ldg(&tmap[(int64_t)i0 * N + t]) : (uint16_t)0;
            }
        }
        for (int t = gl; t < Lw; t += G) sval[t] = 0.0;
        bool changed = false;
        double r = 0.0;   // the row's RHS: element contributions in element order
        for (int c0 = 0; c0 < maxwalk; c0 += G) {
            // lane gl stages incidence c0 + gl: its element row (N / 2 16-byte
            // loads), its N recorded slots and its element RHS entry, so a
            // group has G rows in flight
            const int ii = c0 + gl;
            double reb = 0.0;
            if (ii < nwalk) {
                const int32_t kk = __ldg(&inc[i0 + ii]);
                const int32_t e = kk / N, a = kk - e * N;
                const double2 *src = reinterpret_cast<const double2 *>(Ke + ((size_t)e * N + a) * N);
                const uint32_t *ssrc = reinterpret_cast<const uint32_t *>(slot + ((int64_t)i0 + ii) * N);
                double2 kv[N / 2];
                uint32_t sv[N / 2];
#pragma unroll
                for (int q = 0; q < N / 2; q++) kv[q] = __ldcs(src + q);
#pragma unroll
                for (int q = 0; q < N / 2; q++) sv[q] = __ldcs(ssrc + q);
                reb = __ldg(&Re[kk]);
                double2 *dst = reinterpret_cast<double2 *>(s_ke[w][grp][gl]);
                uint32_t *sdst = reinterpret_cast<uint32_t *>(s_sl[w][grp][gl]);
#pragma unroll
                for (int q = 0; q < N / 2; q++) {
                    dst[q] = kv[q];
                    sdst[q] = sv[q];
                }
            }
            __syncwarp();
            // add them in element order (lane gl: column gl of each row)
            const int nj = nwalk - c0 < G ? nwalk - c0 : G;
            const int maxj = __reduce_max_sync(0xffffffffu, (unsigned)(nj > 0 ? nj : 0));
            for (int j = 0; j < maxj; j++) {
                if (j < nj && gl < N) {
                    const double v = s_ke[w][grp][j][gl];
                    const uint16_t t = s_sl[w][grp][j][gl];
                    if ((v != 0.0) != (t != kSlotZero) || (t != kSlotZero && t >= L)) changed = true;
                    else if (t != kSlotZero) sval[t] = rn_add(sval[t], v);
                }
                __syncwarp();
            }
            // the chunk's element RHS entries, zeros skipped
            for (int t = 0; t < G; t++) {
                const double bt = __shfl_sync(0xffffffffu, reb, t, G);
                if (gl == 0 && c0 + t < nwalk && bt != 0.0) r = rn_add(r, bt);
            }
        }
        if (changed) atomicExch(status, PHGB_DEV_PATTERN_CHANGED);
        // write the entries; a boundary column's value is replaced in s_val by
        // its lift term
        double dg = 0.0;
        bool anyb = false;
#pragma unroll
        for (int k = 0; k < (C::LONG ? MAXROW / G : TPL); k++) {
            const int t = gl + k * G;
            if (t >= Lw) break;
            const uint16_t tmk = C::LONG ? __ldg(&tmap[(int64_t)i0 * N + t]) : tm[C::LONG ? 0 : k];
            const double val = sval[t];
            if (tmk & kTmapBdry) {
                const int j = tmk & ~kTmapBdry;
                const int32_t c = bcols[b0 + j];
                bvals[b0 + j] = val;
                const int mult = inc_ptr[c + 1] - inc_ptr[c];
                double Dk = 0.0;
                for (int m = 0; m < mult; m++) Dk = rn_add(Dk, 1.0);
                const double rk = bdry_rhs(g, c, mult);
                sval[t] = __ddiv_rn(rn_mul(rn_mul(1.0, rk), val), Dk);
                sisb[t] = 1;
                anyb = true;
            } else {
                vals[p0 + tmk] = val;
                if (tmk == dk) dg = val;
                sisb[t] = 0;
            }
        }
        const bool lift = (__ballot_sync(0xffffffffu, anyb) & gmask) != 0;
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) dg += __shfl_xor_sync(0xffffffffu, dg, o, G);
        __syncwarp();
        if (walk && gl == 0) {
            diag[d] = dg;
            // lift the boundary columns in first-touch order: r -= term
            if (lift)
                for (int t = 0; t < L; t++)
                    if (sisb[t]) r = rn_sub(r, sval[t]);
            rhs[d] = r;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Rows from recorded phgMatAddEntries_ calls (src/matvec.c:5348-5493): each
// record is one row segment (row, columns, values) in call order.  A lane
// group of 32 takes a row and its records in call order; within a record the
// entries are taken 32 at a time in their order.  As add_columns_to_row
// (matvec.c:3045-3332, SORT_COLUMNS 0) does, exact zeros and negative
// columns are skipped, a column's first appearance fixes its place and later
// ones add to it.  The reference copies a row's first non-empty segment
// verbatim, so a column repeated inside that segment would appear twice; the
// kernel flags that case (PHGB_DEV_DUPLICATE) rather than reproducing it.
template <int HS_, int MAXROW_, int WARPS_, bool LONG_>
struct RecCfg {
    static constexpr int HS = HS_, MAXROW = MAXROW_, WARPS = WARPS_;
    static constexpr bool LONG = LONG_;
};
using RecShort = RecCfg<512, 256, 4, false>;
using RecLong = RecCfg<2048, 1024, 1, true>;

template <class C>
__global__ void __launch_bounds__(C::WARPS * 32)
record_walk_kernel(int64_t n, const int32_t *__restrict__ rinc_ptr, const int32_t *__restrict__ rinc,
                   const int64_t *__restrict__ rec_ptr, const int32_t *__restrict__ rec_cols,
                   const double *__restrict__ rec_vals, const int32_t *__restrict__ cap_ptr,
                   int32_t *__restrict__ cnt, int32_t *__restrict__ sc_cols, double *__restrict__ sc_vals,
                   int *status, int32_t *__restrict__ over_list, int *nover) {
    constexpr int HS = C::HS, MAXROW = C::MAXROW, W = C::WARPS;
    __shared__ int32_t s_key[W][HS];
    __shared__ int16_t s_pos[W][HS];
    __shared__ int32_t s_col[W][MAXROW];
    __shared__ double s_val[W][MAXROW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    int32_t *key = s_key[w];
    int16_t *hpos = s_pos[w];
    int32_t *scol = s_col[w];
    double *sval = s_val[w];
    const int64_t nwarps = (int64_t)gridDim.x * W;
    const int64_t nrows = C::LONG ? (int64_t)*nover : n;
    for (int64_t k = (int64_t)blockIdx.x * W + w; k < nrows; k += nwarps) {
        const int64_t d = C::LONG ? (int64_t)over_list[k] : k;
        const int32_t r0 = rinc_ptr[d], r1 = rinc_ptr[d + 1];
        for (int t = lane; t < HS; t += 32) key[t] = -1;
        __syncwarp();
        int L = 0;
        bool overflow = false, dup = false;
        for (int ri = r0; ri < r1; ri++) {
            const int32_t rec = rinc[ri];
            const int64_t e0 = rec_ptr[rec], e1 = rec_ptr[rec + 1];
            const bool fresh = L == 0;   // the row's first non-empty segment
            for (int64_t b = e0; b < e1; b += 32) {
                const int64_t j = b + lane;
                int32_t col = -1;
                double v = 0.0;
                if (j < e1) {
                    col = rec_cols[j];
                    v = rec_vals[j];
                }
                const bool nz = j < e1 && col >= 0 && v != 0.0;
                int pos = -1;
                if (nz) {
                    unsigned h = hash32(col) & (HS - 1);
                    for (int probe = 0; probe < HS; probe++) {
                        const int32_t kk = key[h];
                        if (kk == col) { pos = hpos[h]; break; }
                        if (kk == -1) break;
                        h = (h + 1) & (HS - 1);
                    }
                    if (pos >= 0 && fresh) dup = true;
                }
                const unsigned newm = __ballot_sync(0xffffffffu, nz && pos < 0);
                if (nz && pos < 0) {
                    pos = L + __popc(newm & lt_mask);
                    if (pos < MAXROW) {
                        unsigned h = hash32(col) & (HS - 1);
                        for (int probe = 0; probe < HS; probe++) {
                            const int32_t old = atomicCAS(&key[h], -1, col);
                            if (old == -1) { hpos[h] = (int16_t)pos; break; }
                            if (old == col) { dup = true; break; }   // the same column twice in one chunk
                            h = (h + 1) & (HS - 1);
                        }
                        scol[pos] = col;
                        sval[pos] = v;
                    } else {
                        overflow = true;
                    }
                } else if (nz) {
                    sval[pos] = rn_add(sval[pos], v);
                }
                L += __popc(newm);
                __syncwarp();
            }
        }
        const bool bad = __any_sync(0xffffffffu, overflow) || L > MAXROW;
        if (__any_sync(0xffffffffu, dup) && lane == 0) atomicExch(status, PHGB_DEV_DUPLICATE);
        if (bad) {
            if (lane == 0) {
                if (C::LONG) atomicExch(status, PHGB_DEV_ROW_OVERFLOW);
                else over_list[atomicAdd(nover, 1)] = (int32_t)d;
            }
        } else {
            const int64_t base = cap_ptr[d];
            for (int t = lane; t < L; t += 32) {
                sc_cols[base + t] = scol[t];
                sc_vals[base + t] = sval[t];
            }
            if (lane == 0) cnt[d] = L;
        }
        __syncwarp();
    }
}

// Record lengths per row, for the rows' scratch capacities.
__global__ void record_len_kernel(int64_t nrec, const int32_t *__restrict__ rec_row, const int64_t *__restrict__ rec_ptr,
                                  int32_t *__restrict__ cap) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cap[rec_row[r]], (int32_t)(rec_ptr[r + 1] - rec_ptr[r]));
}

// Copies each row's scratch entries (at cap_ptr) to the CSR at ptr.
__global__ void __launch_bounds__(256)
record_compact_kernel(int64_t n, const int32_t *__restrict__ cap_ptr, const int32_t *__restrict__ sc_cols,
                      const double *__restrict__ sc_vals, const int32_t *__restrict__ ptr, int32_t *__restrict__ cols,
                      double *__restrict__ vals) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t d = warp; d < n; d += nwarps) {
        const int32_t src = cap_ptr[d], p0 = ptr[d], len = ptr[d + 1] - p0;
        for (int j = lane; j < len; j += 32) {
            cols[p0 + j] = sc_cols[src + j];
            vals[p0 + j] = sc_vals[src + j];
        }
    }
}

// Copies every row's scratch region into the CSR arrays: kept entries to
// ptr[d].., saved boundary columns (stored reversed at the region's end) to
// bptr[d]...  One warp per row.
__global__ void __launch_bounds__(256)
compact_kernel(int64_t ndof, int N, const int32_t *__restrict__ inc_ptr, const int32_t *__restrict__ sc_cols,
               const double *__restrict__ sc_vals, const int32_t *__restrict__ ptr, int32_t *__restrict__ cols,
               double *__restrict__ vals, const int32_t *__restrict__ bptr, int32_t *__restrict__ bcols,
               double *__restrict__ bvals) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t d = warp; d < ndof; d += nwarps) {
        const int64_t rbase = (int64_t)inc_ptr[d] * N, rcap = (int64_t)(inc_ptr[d + 1] - inc_ptr[d]) * N;
        const int32_t p0 = ptr[d], nk = ptr[d + 1] - p0, b0 = bptr[d], nb = bptr[d + 1] - b0;
        for (int j = lane; j < nk; j += 32) {
            cols[p0 + j] = sc_cols[rbase + j];
            vals[p0 + j] = sc_vals[rbase + j];
        }
        for (int j = lane; j < nb; j += 32) {
            bcols[b0 + j] = sc_cols[rbase + rcap - 1 - j];
            bvals[b0 + j] = sc_vals[rbase + rcap - 1 - j];
        }
    }
}

// ---------------------------------------------------------------------------
// Host-side launchers.

static int grid_for(int64_t work, int per_block, int max_blocks) {
    int64_t b = ceil_div(work, per_block);
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (int)b;
}

template <int P>
static void elem_launch(const ElemArgs &A, cudaStream_t s) {
    constexpr int W = ElemDims<P>::WARPS;
    if (!A.geometry_given)
        geometry_kernel<<<grid_for(A.nelem, 128, 148 * 64), 128, 0, s>>>(A.nelem, A.nvert, A.verts, A.elems,
                                                                        A.geo, A.status);
    ElemWeights Wt{};
    for (int q = 0; q < ElemDims<P>::QK; q++) Wt.wk[q] = A.wk_host[q];
    for (int q = 0; q < ElemDims<P>::QR; q++) Wt.wr[q] = A.wr_host[q];
    if constexpr (P == 1) {   // a lane per basis function
        constexpr int EPB = 4 * (32 / ElemDims<P>::N);   // elements per block
        const int blocks = grid_for(A.nelem, EPB, 148 * 64);
        element_lanes_kernel<P><<<blocks, 128, 0, s>>>(A.nelem, A.ndof, A.geo, A.e2l, A.kappa, A.mass, A.f, Wt,
                                                       A.gk, A.br, A.brt, A.Ke, A.Re, A.status);
    } else if constexpr (P == 2) {   // a lane per two basis functions
        constexpr int EPB = 4 * (32 / (ElemDims<P>::N / 2));
        const int blocks = grid_for(A.nelem, EPB, 148 * 64);
        element_cols2_kernel<P><<<blocks, 128, 0, s>>>(A.nelem, A.ndof, A.geo, A.e2l, A.kappa, A.mass, A.f, Wt,
                                                       A.gk, A.br, A.brt, A.Ke, A.Re, A.status);
    } else {          // P3: a warp per element
        const int blocks = grid_for(A.nelem, W, 148 * 64);
        element_kernel<P><<<blocks, W * 32, 0, s>>>(A.nelem, A.ndof, A.geo, A.e2l, A.kappa, A.mass, A.f, Wt, A.gk,
                                                    A.br, A.brt, A.Ke, A.Re, A.status);
    }
}

cudaError_t launch_element_kernel(int p, const ElemArgs &A, cudaStream_t s) {
    if (p == 1) elem_launch<1>(A, s);
    else if (p == 2) elem_launch<2>(A, s);
    else elem_launch<3>(A, s);
    return cudaGetLastError();
}

int64_t geometry_doubles(int64_t nelem) { return nelem * kGeo; }
int geometry_stride() { return kGeo; }


cudaError_t launch_incidence(int N, int64_t nelem, int64_t ndof, const int32_t *e2l, int32_t *cnt,
                             int32_t *inc_ptr, int32_t *cursor, int32_t *inc, int64_t *scan_ws,
                             int *status, cudaStream_t s) {
    const int64_t nkeys = nelem * N;
    cudaMemsetAsync(cnt, 0, sizeof(int32_t) * ndof, s);
    cudaMemsetAsync(cursor, 0, sizeof(int32_t) * ndof, s);
    const int bl = grid_for(nkeys, 256, 148 * 16);
    inc_count_kernel<<<bl, 256, 0, s>>>(nkeys, N, ndof, e2l, cnt, status);
    cudaError_t err = launch_scan(ndof, cnt, inc_ptr, scan_ws, s);
    if (err != cudaSuccess) return err;
    inc_fill_kernel<<<bl, 256, 0, s>>>(nkeys, ndof, e2l, inc_ptr, cursor, inc);
    inc_sort_kernel<<<grid_for(ndof, 128, 148 * 16), 128, 0, s>>>(ndof, inc_ptr, inc);
    return cudaGetLastError();
}

int64_t scan_workspace_elems(int64_t n) { return ceil_div(n + 1, kScanBlock) + 2; }

cudaError_t launch_scan(int64_t n, const int32_t *in, int32_t *out, int64_t *ws, cudaStream_t s) {
    // ws: block sums (nb) + total; out has n + 1 entries
    const int64_t nb = ceil_div(n + 1, kScanBlock);
    int64_t *total = ws + nb;
    scan_local_kernel<<<(unsigned)nb, kScanBlock, 0, s>>>(n, in, out, ws);
    scan_blocks_kernel<<<1, 1024, 0, s>>>(nb, ws, total);
    scan_add_kernel<<<(unsigned)nb, kScanBlock, 0, s>>>(n, out, ws, total);
    return cudaGetLastError();
}

template <int N>
static cudaError_t walk(const WalkArgs &A, cudaStream_t s) {
    constexpr int W = WalkCfg<N>::WARPS, R = WalkCfg<N>::R;
    const int blocks = grid_for(ceil_div(A.ndof, R), W, 148 * 32);
    cudaError_t e = cudaMemsetAsync(A.nover, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    row_walk_kernel<N, WalkCfg<N>><<<blocks, W * 32, 0, s>>>(
        A.ndof, A.inc_ptr, A.inc, A.e2l, A.bdry, A.Ke, A.Re, A.g, A.cnt_keep, A.cnt_bdry, A.sc_cols, A.sc_vals,
        A.rhs, A.diag, A.status, A.over_list, A.nover, A.slot, A.tmap, A.dpos);
    // the rows the first pass listed (none in most meshes: the blocks return
    // after reading the count)
    row_walk_kernel<N, LongWalkCfg<N>><<<148 * 4, 32, 0, s>>>(
        A.ndof, A.inc_ptr, A.inc, A.e2l, A.bdry, A.Ke, A.Re, A.g, A.cnt_keep, A.cnt_bdry, A.sc_cols, A.sc_vals,
        A.rhs, A.diag, A.status, A.over_list, A.nover, A.slot, A.tmap, A.dpos);
    return cudaGetLastError();
}

template <int N>
static cudaError_t value_walk(const WalkArgs &A, cudaStream_t s) {
    constexpr int W = WalkCfg<N>::WARPS, R = WalkCfg<N>::R;
    const int blocks = grid_for(ceil_div(A.ndof, R), W, 148 * 32);
    value_walk_kernel<N, WalkCfg<N>><<<blocks, W * 32, 0, s>>>(
        A.ndof, A.inc_ptr, A.inc, A.bdry, A.Ke, A.Re, A.g, A.slot, A.tmap, A.dpos, A.ptr, A.bptr, A.bcols, A.vals,
        A.bvals, A.rhs, A.diag, A.status, A.over_list, A.nover);
    // rows longer than the walk's table (listed by the recording walk)
    value_walk_kernel<N, LongWalkCfg<N>><<<148 * 4, 32, 0, s>>>(
        A.ndof, A.inc_ptr, A.inc, A.bdry, A.Ke, A.Re, A.g, A.slot, A.tmap, A.dpos, A.ptr, A.bptr, A.bcols, A.vals,
        A.bvals, A.rhs, A.diag, A.status, A.over_list, A.nover);
    return cudaGetLastError();
}

cudaError_t launch_record_lengths(int64_t nrec, const int32_t *rec_row, const int64_t *rec_ptr, int32_t *cap,
                                  cudaStream_t s) {
    record_len_kernel<<<grid_for(nrec, 256, 148 * 16), 256, 0, s>>>(nrec, rec_row, rec_ptr, cap);
    return cudaGetLastError();
}

cudaError_t launch_record_walk(const RecordArgs &A, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(A.nover, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    record_walk_kernel<RecShort><<<grid_for(A.n, RecShort::WARPS, 148 * 16), RecShort::WARPS * 32, 0, s>>>(
        A.n, A.rinc_ptr, A.rinc, A.rec_ptr, A.rec_cols, A.rec_vals, A.cap_ptr, A.cnt, A.sc_cols, A.sc_vals,
        A.status, A.over_list, A.nover);
    record_walk_kernel<RecLong><<<148 * 4, 32, 0, s>>>(A.n, A.rinc_ptr, A.rinc, A.rec_ptr, A.rec_cols, A.rec_vals,
                                                      A.cap_ptr, A.cnt, A.sc_cols, A.sc_vals, A.status,
                                                      A.over_list, A.nover);
    return cudaGetLastError();
}

cudaError_t launch_record_compact(const RecordArgs &A, const int32_t *ptr, int32_t *cols, double *vals,
                                  cudaStream_t s) {
    record_compact_kernel<<<grid_for(A.n * 32, 256, 148 * 16), 256, 0, s>>>(A.n, A.cap_ptr, A.sc_cols, A.sc_vals,
                                                                          ptr, cols, vals);
    return cudaGetLastError();
}

cudaError_t launch_value_walk(int p, const WalkArgs &A, cudaStream_t s) {
    if (p == 1) return value_walk<4>(A, s);
    if (p == 2) return value_walk<10>(A, s);
    return value_walk<20>(A, s);
}

cudaError_t launch_row_walk(int p, const WalkArgs &A, cudaStream_t s) {
    if (p == 1) return walk<4>(A, s);
    if (p == 2) return walk<10>(A, s);
    return walk<20>(A, s);
}

cudaError_t launch_compact(int N, const WalkArgs &A, cudaStream_t s) {
    compact_kernel<<<grid_for(A.ndof * 32, 256, 148 * 16), 256, 0, s>>>(A.ndof, N, A.inc_ptr, A.sc_cols, A.sc_vals,
                                                                      A.ptr, A.cols, A.vals, A.bptr, A.bcols,
                                                                      A.bvals);
    return cudaGetLastError();
}

int row_walk_max_row(int p) {
    return p == 1 ? LongWalkCfg<4>::MAXROW : p == 2 ? LongWalkCfg<10>::MAXROW : LongWalkCfg<20>::MAXROW;
}

}  // namespace phgb
