// Quadrature rules and P1/P2/P3 Lagrange bases on the tetrahedron.
//
// Compiled with -ffp-contract=off: the tables are built with the same
// operations as the reference (quad.c:1799-1988 with the orbit expansions
// of include/phg/quad-permu.h:81-115; lagrange.c:80-727), so every point,
// weight, basis value and gradient is the same double the reference uses.
#include "fe_tables.h"

#include <cstring>
#include <stdexcept>

namespace phgb {

namespace {

// Orbit of a symmetric rule: kind 0 = centroid, 1 = (c,a,a,a) with
// c = 1 - 3a, 2 = (a,a,h,h) with h = 1/2 - a, 3 = (a,a,b,c) with
// c = 1 - a - a - b.  Weight w per point.
struct Orbit { int kind; double a, b, w; };

const Orbit kP1[] = {{0, 0x1p-2, 0, 0x1p+0}};
const Orbit kP2[] = {{1, 0x1.1b06d1d200913p-3, 0, 0x1p-2}};
const Orbit kP3[] = {{1, 0x1.4fed9206b2f89p-2, 0, 0x1.1bb48cedffa77p-3},
                     {1, 0x1.b613966c6575dp-4, 0, 0x1.c896e62400b12p-4}};
const Orbit kP4[] = {{1, 0x1.7bd7f53458af6p-4, 0, 0x1.2d070a8ab1538p-4},
                     {1, 0x1.3e58e0e01751bp-2, 0, 0x1.cd91dab9ceaa5p-4},
                     {2, 0x1.74c42f2220fa2p-5, 0, 0x1.5c8978fa0002fp-5}};
const Orbit kP5[] = {{1, 0x1.3e58e0e01751bp-2, 0, 0x1.cd91dab9ceaa5p-4},
                     {1, 0x1.7bd7f53458af6p-4, 0, 0x1.2d070a8ab1538p-4},
                     {2, 0x1.74c42f2220fa2p-5, 0, 0x1.5c8978fa0002fp-5}};
const Orbit kP6[] = {{1, 0x1.b781b5cd7c6ddp-3, 0, 0x1.470c135734e1p-5},
                     {1, 0x1.4d3379368f7d6p-5, 0, 0x1.4a35c5f5705f2p-7},
                     {1, 0x1.4a12f1a1b0dbfp-2, 0, 0x1.c57c6c8a84f8ap-5},
                     {3, 0x1.04c1661157396p-4, 0x1.34bd28932a6e3p-1,
                      0x1.8af8af8af8af9p-5}};

void push(QuadRule &r, double l0, double l1, double l2, double l3, double w) {
    r.pts.insert(r.pts.end(), {l0, l1, l2, l3});
    r.wts.push_back(w);
    r.np++;
}

QuadRule build(const Orbit *orb, int n) {
    QuadRule r;
    for (int o = 0; o < n; o++) {
        const double a = orb[o].a, b = orb[o].b, w = orb[o].w;
        switch (orb[o].kind) {
        case 0:
            push(r, a, a, a, a, w);
            break;
        case 1: {
            const double c = 1.0 - 3.0 * a;
            push(r, c, a, a, a, w); push(r, a, c, a, a, w);
            push(r, a, a, c, a, w); push(r, a, a, a, c, w);
            break;
        }
        case 2: {
            const double h = 0.5 - a;
            push(r, a, a, h, h, w); push(r, a, h, a, h, w);
            push(r, a, h, h, a, w); push(r, h, a, h, a, w);
            push(r, h, a, a, h, w); push(r, h, h, a, a, w);
            break;
        }
        default: {
            const double c = 1.0 - a - a - b;
            push(r, a, a, b, c, w); push(r, a, a, c, b, w);
            push(r, a, b, a, c, w); push(r, a, b, c, a, w);
            push(r, a, c, a, b, w); push(r, a, c, b, a, w);
            push(r, b, a, a, c, w); push(r, b, a, c, a, w);
            push(r, b, c, a, a, w); push(r, c, a, a, b, w);
            push(r, c, a, b, a, w); push(r, c, b, a, a, w);
            break;
        }
        }
    }
    return r;
}

const int kEdge[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

}  // namespace

const QuadRule &quad_rule(int order) {
    // Order 0 is integrated with the order-1 rule (the reference fills empty
    // slots of its rule table with the next available rule).
    static const QuadRule rules[7] = {
        build(kP1, 1), build(kP1, 1), build(kP2, 1), build(kP3, 2),
        build(kP4, 3), build(kP5, 3), build(kP6, 4)};
    if (order < 0 || order > 6) throw std::invalid_argument("quadrature order");
    return rules[order];
}

int nbas(int p) { return p == 1 ? 4 : p == 2 ? 10 : p == 3 ? 20 : -1; }

void basis_values(int p, const double *l, double *v) {
    const double L0 = l[0], L1 = l[1], L2 = l[2], L3 = l[3];
    if (p == 1) {
        v[0] = L0; v[1] = L1; v[2] = L2; v[3] = L3;
        return;
    }
    if (p == 2) {
        v[0] = L0 * (L0 + L0 - 1.);
        v[1] = L1 * (L1 + L1 - 1.);
        v[2] = L2 * (L2 + L2 - 1.);
        v[3] = L3 * (L3 + L3 - 1.);
        for (int e = 0; e < 6; e++) v[4 + e] = 4. * l[kEdge[e][0]] * l[kEdge[e][1]];
        return;
    }
    for (int k = 0; k < 4; k++) {
        const double t = 3. * l[k];
        v[k] = .5 * (t - 1.) * (t - 2.) * l[k];
    }
    for (int e = 0; e < 6; e++) {
        const int a = kEdge[e][0], b = kEdge[e][1];
        const double d = l[a] * l[b];
        v[4 + 2 * e] = 4.5 * (3. * l[a] - 1.) * d;
        v[5 + 2 * e] = 4.5 * (3. * l[b] - 1.) * d;
    }
    v[16] = 27. * L1 * L2 * L3;
    v[17] = 27. * L0 * L2 * L3;
    v[18] = 27. * L0 * L1 * L3;
    v[19] = 27. * L0 * L1 * L2;
}

void basis_grad_lambda(int p, const double *l, double *G) {
    const int n = nbas(p);
    std::memset(G, 0, sizeof(double) * n * 4);
    if (p == 1) {
        for (int k = 0; k < 4; k++) G[4 * k + k] = 1.0;
        return;
    }
    if (p == 2) {
        for (int k = 0; k < 4; k++) G[4 * k + k] = 4. * l[k] - 1.;
        for (int e = 0; e < 6; e++) {
            const int a = kEdge[e][0], b = kEdge[e][1];
            G[4 * (4 + e) + a] = 4. * l[b];
            G[4 * (4 + e) + b] = 4. * l[a];
        }
        return;
    }
    for (int k = 0; k < 4; k++) G[4 * k + k] = (13.5 * l[k] - 9.) * l[k] + 1.;
    for (int e = 0; e < 6; e++) {
        const int a = kEdge[e][0], b = kEdge[e][1];
        G[4 * (4 + 2 * e) + a] = (27. * l[a] - 4.5) * l[b];
        G[4 * (4 + 2 * e) + b] = 4.5 * l[a] * (3. * l[a] - 1.);
        G[4 * (5 + 2 * e) + a] = 4.5 * l[b] * (3. * l[b] - 1.);
        G[4 * (5 + 2 * e) + b] = (27. * l[b] - 4.5) * l[a];
    }
    for (int k = 0; k < 4; k++) {
        int o[3], m = 0;
        for (int i = 0; i < 4; i++)
            if (i != k) o[m++] = i;
        G[4 * (16 + k) + o[0]] = 27. * l[o[1]] * l[o[2]];
        G[4 * (16 + k) + o[1]] = 27. * l[o[0]] * l[o[2]];
        G[4 * (16 + k) + o[2]] = 27. * l[o[0]] * l[o[1]];
    }
}

ElementTables make_tables(int p) {
    ElementTables t;
    t.p = p;
    t.N = nbas(p);
    if (t.N < 0) throw std::invalid_argument("Lagrange order must be 1, 2 or 3");
    const QuadRule &rk = quad_rule(2 * (p - 1));
    const QuadRule &rr = quad_rule(2 * p);
    t.nq_k = rk.np;
    t.nq_r = rr.np;
    t.wk = rk.wts;
    t.wr = rr.wts;
    t.gk.resize((size_t)rk.np * t.N * 4);
    for (int q = 0; q < rk.np; q++)
        basis_grad_lambda(p, &rk.pts[4 * q], &t.gk[(size_t)q * t.N * 4]);
    t.br.resize((size_t)rr.np * t.N);
    for (int q = 0; q < rr.np; q++)
        basis_values(p, &rr.pts[4 * q], &t.br[(size_t)q * t.N]);
    return t;
}

}  // namespace phgb
