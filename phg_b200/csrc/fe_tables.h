// Host-side quadrature rules and Lagrange basis tables for P1/P2/P3 on the
// tetrahedron, evaluated once per order and uploaded to the device.
#pragma once
#include <vector>

namespace phgb {

// A symmetric tetrahedral quadrature rule: barycentric points (np x 4),
// weights summing to 1.
struct QuadRule {
    int np = 0;
    std::vector<double> pts, wts;
};

// The rule the reference selects for polynomial order `order` (0..6).
const QuadRule &quad_rule(int order);

int nbas(int p);                                    // 4, 10, 20
void basis_values(int p, const double *lam, double *v);      // N
void basis_grad_lambda(int p, const double *lam, double *G); // N x 4

// Per-order tables consumed by the element kernels.
struct ElementTables {
    int p = 0, N = 0;
    int nq_k = 0;                 // stiffness points: order 2(p-1)
    int nq_r = 0;                 // rhs / mass points: order 2p
    std::vector<double> wk;       // nq_k
    std::vector<double> gk;       // nq_k x N x 4   d phi / d lambda
    std::vector<double> wr;       // nq_r
    std::vector<double> br;       // nq_r x N       phi
};
ElementTables make_tables(int p);

}  // namespace phgb
