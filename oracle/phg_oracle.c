/*
 * phg_oracle.c -- CPU restatement of the reference (PHG 0.9.7) arithmetic
 * for the P1/P2/P3 element assembly + Jacobi-PCG path.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle of tests/, smoke() and bench.py's
 * CPU-baseline leg.  The product never links, loads or calls it.
 *
 * Compiled with -ffp-contract=off: every expression below is evaluated with
 * the operand order and roundings of the reference routine it cites, so the
 * results agree with the reference's serial x86-64 build bit for bit.  The
 * parity tests pin this against outputs of the unmodified reference built
 * from its sources (tests/golden/).
 */
#include "phg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

/*------------------------------ geometry --------------------------------*/

void
pho_jacobian(const double *x, double *J)
/* Restates compute_jacobian (geom.c:103-169): Gauss-Jordan elimination with
 * partial pivoting on the 4x8 system [x_j y_j z_j 1 | I], then transpose of
 * the right half.  Same loop order and operations. */
{
    double a[4][8], d, t;
    int i, j, k;

    for (j = 0; j < 4; j++) {
	for (i = 0; i < 3; i++)
	    a[j][i] = x[3 * j + i];
	a[j][3] = 1.0;
	for (i = 0; i < 4; i++)
	    a[j][4 + i] = (i == j) ? 1.0 : 0.0;
    }
    for (j = 0; j < 4; j++) {
	d = fabs(a[j][j]);
	k = j;
	for (i = j + 1; i < 4; i++) {
	    t = fabs(a[i][j]);
	    if (d < t) {
		d = t;
		k = i;
	    }
	}
	if (k != j)
	    for (i = j; i < 8; i++) {
		t = a[j][i];
		a[j][i] = a[k][i];
		a[k][i] = t;
	    }
	t = a[j][j];
	d = 1.0 / (t == 0. ? 1. : t);
	for (i = j + 1; i < 8; i++)
	    a[j][i] *= d;
	for (i = j + 1; i < 4; i++) {
	    d = a[i][j];
	    for (k = j + 1; k < 8; k++)
		a[i][k] -= d * a[j][k];
	}
    }
    for (j = 2; j >= 0; j--)
	for (i = j + 1; i < 4; i++) {
	    d = a[j][i];
	    for (k = 4; k < 8; k++)
		a[j][k] -= d * a[i][k];
	}
    for (j = 0; j < 4; j++)
	for (i = 0; i < 4; i++)
	    J[4 * j + i] = a[i][j + 4];
}

double
pho_volume(const double *x)
/* Restates the volume part of _phg_compute_elem_data (geom.c:46-78). */
{
    const double oned6 = 1.0 / 6.0;
    double x0 = x[0], y0 = x[1], z0 = x[2];
    double x1 = x[3] - x0, y1 = x[4] - y0, z1 = x[5] - z0;
    double x2 = x[6] - x0, y2 = x[7] - y0, z2 = x[8] - z0;
    double x3 = x[9] - x0, y3 = x[10] - y0, z3 = x[11] - z0;

    return fabs(x1 * y2 * z3 + x2 * y3 * z1 + y1 * z2 * x3 -
		(z1 * y2 * x3 + y1 * x2 * z3 + z2 * y3 * x1)) * oned6;
}

/*----------------------------- quadrature --------------------------------*/

/* Symmetric tetrahedral rules, stored as orbit generators (exact doubles,
 * C99 hex) and expanded below.  The expansions follow the point order of the
 * reference's orbit macros (include/phg/quad-permu.h:81-115) and compute the
 * dependent coordinate the same way (1 - 3a, 1/2 - a, 1 - a - a - b), so the
 * expanded tables equal the reference's QUAD_3D_P1..P6 (quad.c:1799-1988)
 * bit for bit. */
enum { S4, S31, S22, S211 };
typedef struct { int kind; double a, b, w; } ORBIT;

static const ORBIT rule_p1[] = {{S4, 0x1p-2, 0, 0x1p+0}};
static const ORBIT rule_p2[] = {{S31, 0x1.1b06d1d200913p-3, 0, 0x1p-2}};
static const ORBIT rule_p3[] = {
    {S31, 0x1.4fed9206b2f89p-2, 0, 0x1.1bb48cedffa77p-3},
    {S31, 0x1.b613966c6575dp-4, 0, 0x1.c896e62400b12p-4}};
static const ORBIT rule_p4[] = {
    {S31, 0x1.7bd7f53458af6p-4, 0, 0x1.2d070a8ab1538p-4},
    {S31, 0x1.3e58e0e01751bp-2, 0, 0x1.cd91dab9ceaa5p-4},
    {S22, 0x1.74c42f2220fa2p-5, 0, 0x1.5c8978fa0002fp-5}};
static const ORBIT rule_p5[] = {
    {S31, 0x1.3e58e0e01751bp-2, 0, 0x1.cd91dab9ceaa5p-4},
    {S31, 0x1.7bd7f53458af6p-4, 0, 0x1.2d070a8ab1538p-4},
    {S22, 0x1.74c42f2220fa2p-5, 0, 0x1.5c8978fa0002fp-5}};
static const ORBIT rule_p6[] = {
    {S31, 0x1.b781b5cd7c6ddp-3, 0, 0x1.470c135734e1p-5},
    {S31, 0x1.4d3379368f7d6p-5, 0, 0x1.4a35c5f5705f2p-7},
    {S31, 0x1.4a12f1a1b0dbfp-2, 0, 0x1.c57c6c8a84f8ap-5},
    {S211, 0x1.04c1661157396p-4, 0x1.34bd28932a6e3p-1, 0x1.8af8af8af8af9p-5}};

static int
expand(const ORBIT *orb, int norb, double *pts, double *wts)
{
    int o, n = 0, i, k;
    for (o = 0; o < norb; o++) {
	double a = orb[o].a, b = orb[o].b, w = orb[o].w, c;
	double p[12][4];
	int np;
	switch (orb[o].kind) {
	case S4:
	    np = 1;
	    p[0][0] = p[0][1] = p[0][2] = p[0][3] = a;
	    break;
	case S31:
	    np = 4;
	    c = 1.0 - 3.0 * a;
	    for (i = 0; i < 4; i++)
		for (k = 0; k < 4; k++)
		    p[i][k] = (i == k) ? c : a;
	    break;
	case S22: {
	    /* positions holding `a` in each of the 6 points */
	    static const int pa[6][2] = {{0,1},{0,2},{0,3},{1,3},{1,2},{2,3}};
	    np = 6;
	    c = 0.5 - a;
	    for (i = 0; i < 6; i++)
		for (k = 0; k < 4; k++)
		    p[i][k] = (k == pa[i][0] || k == pa[i][1]) ? a : c;
	    break;
	}
	default: {		/* S211: two a's, one b, one c */
	    /* each point as (position of b, position of c) */
	    static const int pbc[12][2] = {
		{2,3},{3,2},{1,3},{1,2},{3,1},{2,1},
		{0,3},{0,2},{0,1},{3,0},{2,0},{1,0}};
	    np = 12;
	    c = 1.0 - a - a - b;
	    for (i = 0; i < 12; i++)
		for (k = 0; k < 4; k++)
		    p[i][k] = (k == pbc[i][0]) ? b : (k == pbc[i][1]) ? c : a;
	    break;
	}
	}
	for (i = 0; i < np; i++, n++) {
	    memcpy(pts + 4 * n, p[i], 4 * sizeof(double));
	    wts[n] = w;
	}
    }
    return n;
}

#define MAXQP 24
static double qpts[7][MAXQP * 4], qwts[7][MAXQP];
static int qnp[7] = {0, 0, 0, 0, 0, 0, 0};

int
pho_quad_rule(int order, const double **pts, const double **wts)
/* phgQuadGetQuad3D (quad.c:2914): order 0 uses the order-1 rule. */
{
    static const ORBIT *rules[7] = {rule_p1, rule_p1, rule_p2, rule_p3,
				    rule_p4, rule_p5, rule_p6};
    static const int nrules[7] = {1, 1, 1, 2, 3, 3, 4};
    if (order < 0 || order > 6)
	return -1;
    if (qnp[order] == 0)
	qnp[order] = expand(rules[order], nrules[order], qpts[order],
			    qwts[order]);
    *pts = qpts[order];
    *wts = qwts[order];
    return qnp[order];
}

/*------------------------------- bases ----------------------------------*/

int
pho_nbas(int p)
{
    return p == 1 ? 4 : p == 2 ? 10 : p == 3 ? 20 : -1;
}

void
pho_bas(int p, const double *lambda, double *v)
/* P1_bas lagrange.c:80-105, P2_bas :160-200 (all-bases path),
 * P3_bas :392-440 (all-bases path). */
{
    double L0 = lambda[0], L1 = lambda[1], L2 = lambda[2], L3 = lambda[3];
    if (p == 1) {
	v[0] = L0; v[1] = L1; v[2] = L2; v[3] = L3;
    }
    else if (p == 2) {
	v[0] = L0 * (L0 + L0 - 1.);
	v[1] = L1 * (L1 + L1 - 1.);
	v[2] = L2 * (L2 + L2 - 1.);
	v[3] = L3 * (L3 + L3 - 1.);
	v[4] = 4. * L0 * L1;
	v[5] = 4. * L0 * L2;
	v[6] = 4. * L0 * L3;
	v[7] = 4. * L1 * L2;
	v[8] = 4. * L1 * L3;
	v[9] = 4. * L2 * L3;
    }
    else {
	double L03 = 3. * L0, L13 = 3. * L1, L23 = 3. * L2, L33 = 3. * L3, d;
	v[0] = .5 * (L03 - 1.) * (L03 - 2.) * L0;
	v[1] = .5 * (L13 - 1.) * (L13 - 2.) * L1;
	v[2] = .5 * (L23 - 1.) * (L23 - 2.) * L2;
	v[3] = .5 * (L33 - 1.) * (L33 - 2.) * L3;
	d = L0 * L1;
	v[4] = 4.5 * (L03 - 1.) * d;
	v[5] = 4.5 * (L13 - 1.) * d;
	d = L0 * L2;
	v[6] = 4.5 * (L03 - 1.) * d;
	v[7] = 4.5 * (L23 - 1.) * d;
	d = L0 * L3;
	v[8] = 4.5 * (L03 - 1.) * d;
	v[9] = 4.5 * (L33 - 1.) * d;
	d = L1 * L2;
	v[10] = 4.5 * (L13 - 1.) * d;
	v[11] = 4.5 * (L23 - 1.) * d;
	d = L1 * L3;
	v[12] = 4.5 * (L13 - 1.) * d;
	v[13] = 4.5 * (L33 - 1.) * d;
	d = L2 * L3;
	v[14] = 4.5 * (L23 - 1.) * d;
	v[15] = 4.5 * (L33 - 1.) * d;
	v[16] = 27. * L1 * L2 * L3;
	v[17] = 27. * L0 * L2 * L3;
	v[18] = 27. * L0 * L1 * L3;
	v[19] = 27. * L0 * L1 * L2;
    }
}

/* local edge -> (first, second) local vertex */
static const int edge_v[6][2] = {{0,1},{0,2},{0,3},{1,2},{1,3},{2,3}};

void
pho_grad_lambda(int p, const double *l, double *G)
/* d phi / d lambda: P1_grad lagrange.c:111-140, P2_grad :248-355,
 * P3_grad :538-727.  G is N x 4. */
{
    int n = pho_nbas(p), k, e;
    memset(G, 0, (size_t)n * 4 * sizeof(double));
    if (p == 1) {
	for (k = 0; k < 4; k++)
	    G[4 * k + k] = 1.0;
	return;
    }
    if (p == 2) {
	for (k = 0; k < 4; k++)
	    G[4 * k + k] = 4. * l[k] - 1.;
	for (e = 0; e < 6; e++) {
	    int a = edge_v[e][0], b = edge_v[e][1];
	    G[4 * (4 + e) + a] = 4. * l[b];
	    G[4 * (4 + e) + b] = 4. * l[a];
	}
	return;
    }
    for (k = 0; k < 4; k++)
	G[4 * k + k] = (13.5 * l[k] - 9.) * l[k] + 1.;
    for (e = 0; e < 6; e++) {
	int a = edge_v[e][0], b = edge_v[e][1];
	/* node nearest vertex a, then node nearest vertex b */
	G[4 * (4 + 2 * e) + a] = (27. * l[a] - 4.5) * l[b];
	G[4 * (4 + 2 * e) + b] = 4.5 * l[a] * (3. * l[a] - 1.);
	G[4 * (5 + 2 * e) + a] = 4.5 * l[b] * (3. * l[b] - 1.);
	G[4 * (5 + 2 * e) + b] = (27. * l[b] - 4.5) * l[a];
    }
    for (k = 0; k < 4; k++) {
	/* face k is opposite vertex k: phi = 27 * product of the others */
	int o[3], m = 0, i;
	for (i = 0; i < 4; i++)
	    if (i != k)
		o[m++] = i;
	G[4 * (16 + k) + o[0]] = 27. * l[o[1]] * l[o[2]];
	G[4 * (16 + k) + o[1]] = 27. * l[o[0]] * l[o[2]];
	G[4 * (16 + k) + o[2]] = 27. * l[o[0]] * l[o[1]];
    }
}

static void
basis_gradients(int p, const double *J, int np, const double *pts,
		double *grad /* [N][np][3] */)
/* phgQuadGetBasisGradient (quad.c:3314-3421): vertex bases use the diagonal
 * shortcut (P1: copy of J's row; P2/P3: d * J[k][c]), the others the full
 * 4-term sum G[0]*J[0][c] + ... + G[3]*J[3][c]. */
{
    int n = pho_nbas(p), k, q, c;
    double G[20 * 4];
    for (q = 0; q < np; q++) {
	pho_grad_lambda(p, pts + 4 * q, G);
	for (k = 0; k < n; k++) {
	    double *o = grad + 3 * (k * np + q);
	    const double *g = G + 4 * k;
	    if (k < 4) {
		if (p == 1) {
		    for (c = 0; c < 3; c++)
			o[c] = J[4 * k + c];
		}
		else {
		    double d = g[k];
		    for (c = 0; c < 3; c++)
			o[c] = d * J[4 * k + c];
		}
	    }
	    else {
		for (c = 0; c < 3; c++)
		    o[c] = g[0] * J[0 * 4 + c] + g[1] * J[1 * 4 + c] +
			   g[2] * J[2 * 4 + c] + g[3] * J[3 * 4 + c];
	    }
	}
    }
}

/* The element integrals from the element's geometry (J, volume): PHG
 * computes them from the coordinates (compute_jacobian, geom.c:103-169) on
 * elements it imported and interpolates them from the parent on elements
 * bisection made (geom.c:460-565); either way phgQuad* read the stored
 * values (phgGeomGetJacobian_, geom.c:855-884). */
static void
elem_stiffness_geo(int p, const double *J, double vol, double kappa, double *A)
{
    int n = pho_nbas(p), np, a, b, q, order = 2 * (p - 1);
    const double *pts, *w;
    double grad[20 * MAXQP * 3];

    np = pho_quad_rule(order, &pts, &w);
    basis_gradients(p, J, np, pts, grad);
    for (a = 0; a < n; a++)
	for (b = 0; b <= a; b++) {
	    double d = 0.;
	    for (q = 0; q < np; q++) {
		const double *g1 = grad + 3 * (b * np + q);
		const double *g2 = grad + 3 * (a * np + q);
		double d0 = 0.;
		d0 += g1[0] * g2[0] + g1[1] * g2[1] + g1[2] * g2[2];
		if (kappa < 0.)
		    d += d0 * w[q];
		else
		    d += d0 * w[q] * kappa;
	    }
	    A[a * n + b] = A[b * n + a] = d * vol;
	}
}

void
pho_elem_stiffness(int p, const double *x, double kappa, double *A)
/* The reference user loop (examples/poisson.c:126-139) calls
 * phgQuadGradBasAGradBas(e, u, j, A, u, i, QUAD_DEFAULT) for j <= i
 * (quad.c:5260-5344): order (p-1)+(p-1) (+0 for a P0 coefficient),
 * d = sum_q (0 + g_j.g_i) * w_q [* kappa], times the volume. */
{
    double J[16];
    pho_jacobian(x, J);
    elem_stiffness_geo(p, J, pho_volume(x), kappa, A);
}

static void
elem_mass_vol(int p, double vol, double *M)
{
    int n = pho_nbas(p), np, a, b, q;
    const double *pts, *w;
    double bas[MAXQP][20];

    np = pho_quad_rule(2 * p, &pts, &w);
    for (q = 0; q < np; q++)
	pho_bas(p, pts + 4 * q, bas[q]);
    for (a = 0; a < n; a++)
	for (b = 0; b <= a; b++) {
	    double d = 0.;
	    for (q = 0; q < np; q++) {
		double d0 = 0.;
		d0 += bas[q][b] * bas[q][a];
		d += d0 * w[q];
	    }
	    M[a * n + b] = M[b * n + a] = d * vol;
	}
}

void
pho_elem_mass(int p, const double *x, double *M)
/* phgQuadBasABas with A = NULL (quad.c:5582-5625): order p+p,
 * d = sum_q (0 + phi_j phi_i) * w_q, times the volume. */
{
    elem_mass_vol(p, pho_volume(x), M);
}

static void
elem_rhs_vol(int p, double vol, const double *f_local, double *res)
{
    int n = pho_nbas(p), np, a, q, k;
    const double *pts, *w;
    double bas[MAXQP][20], fq[MAXQP];

    np = pho_quad_rule(2 * p, &pts, &w);
    for (q = 0; q < np; q++) {
	double v = 0.0;
	pho_bas(p, pts + 4 * q, bas[q]);
	for (k = 0; k < n; k++)
	    v += bas[q][k] * f_local[k];
	fq[q] = v;
    }
    for (a = 0; a < n; a++) {
	double d = 0.0;
	for (q = 0; q < np; q++)
	    d += bas[q][a] * w[q] * fq[q];
	res[a] = d * vol;
    }
}

void
pho_elem_rhs(int p, const double *x, const double *f_local, double *res)
/* phgQuadDofTimesBas(e, f_h, u_h, i, QUAD_DEFAULT) (quad.c:5481-5530):
 * order p+p; f at the points by phgDofEval_ (dof-utils.c:100-300), i.e.
 * 0 + phi_0 f_0 + phi_1 f_1 + ... in basis order; then
 * d = sum_q phi_i * w_q * f_q, times the volume. */
{
    elem_rhs_vol(p, pho_volume(x), f_local, res);
}

/*------------------------------ assembly ---------------------------------*/

typedef struct { int32_t *cols; double *vals; int64_t n, alloc; } ROW;

static void
row_add(ROW *r, int32_t col, double val)
/* add_columns_to_row, SORT_COLUMNS == 0 branch (matvec.c:3286-3321):
 * linear search, add to an existing column, else append. */
{
    int64_t i;
    for (i = 0; i < r->n; i++)
	if (r->cols[i] == col) {
	    r->vals[i] += val;
	    return;
	}
    if (r->n >= r->alloc) {
	r->alloc = r->alloc ? 2 * r->alloc : 16;
	r->cols = realloc(r->cols, r->alloc * sizeof(*r->cols));
	r->vals = realloc(r->vals, r->alloc * sizeof(*r->vals));
    }
    r->cols[r->n] = col;
    r->vals[r->n++] = val;
}

static void
pack(const ROW *rows, int64_t n, int64_t **ptr, int32_t **cols, double **vals)
{
    int64_t i, k = 0, nnz = 0;
    for (i = 0; i < n; i++)
	nnz += rows[i].n;
    *ptr = malloc((n + 1) * sizeof(**ptr));
    *cols = malloc((nnz + 1) * sizeof(**cols));
    *vals = malloc((nnz + 1) * sizeof(**vals));
    (*ptr)[0] = 0;
    for (i = 0; i < n; i++) {
	memcpy(*cols + k, rows[i].cols, rows[i].n * sizeof(int32_t));
	memcpy(*vals + k, rows[i].vals, rows[i].n * sizeof(double));
	k += rows[i].n;
	(*ptr)[i + 1] = k;
    }
}

int
pho_assemble(int p, int64_t nvert, const double *verts, int64_t nelem,
	     const int32_t *elems, const int32_t *e2l, int64_t ndof,
	     const uint8_t *bdry, const double *f, const double *g,
	     const double *kappa, double mass_coef, const double *geom,
	     pho_system *S)
{
    int N = pho_nbas(p), a, b;
    int64_t e, i, j;
    ROW *rows;
    double A[400], M[400], B[20], R[20], x[12], fl[20];

    if (N < 0)
	return -1;
    memset(S, 0, sizeof(*S));
    S->n = ndof;
    rows = calloc(ndof, sizeof(*rows));
    S->rhs_raw = calloc(ndof, sizeof(double));

    /* the user element loop (examples/poisson.c:101-170) */
    for (e = 0; e < nelem; e++) {
	const int32_t *I = e2l + e * N;
	for (a = 0; a < 4; a++) {
	    int32_t v = elems[4 * e + a];
	    if (v < 0 || v >= nvert)
		return -2;
	    memcpy(x + 3 * a, verts + 3 * (int64_t)v, 3 * sizeof(double));
	}
	for (a = 0; a < N; a++) {
	    if (I[a] < 0 || I[a] >= ndof)
		return -3;
	    fl[a] = f != NULL ? f[I[a]] : 0.0;
	}
	{   /* the element's geometry: PHG's stored values when given */
	    double J[16], vol;
	    if (geom != NULL) {
		memcpy(J, geom + 17 * e, 16 * sizeof(double));
		vol = geom[17 * e + 16];
	    }
	    else {
		pho_jacobian(x, J);
		vol = pho_volume(x);
	    }
	    elem_stiffness_geo(p, J, vol, kappa != NULL ? kappa[e] : -1.0, A);
	    /* stiffness + c * mass (examples/simplest.c:68-72) */
	    if (mass_coef != 0.0) {
		elem_mass_vol(p, vol, M);
		for (a = 0; a < N * N; a++)
		    A[a] = A[a] + mass_coef * M[a];
	    }
	    elem_rhs_vol(p, vol, fl, R);
	}
	for (a = 0; a < N; a++) {
	    if (bdry[I[a]]) {
		/* phgDofDirichletBC nodal path (dof-utils.c:1369-1392):
		 * unit row, rhs = g at the node; zeros are dropped by
		 * phgMatAddEntries (matvec.c:5459-5461) */
		B[a] = g != NULL ? g[I[a]] : 0.0;
		row_add(&rows[I[a]], I[a], 1.0);
	    }
	    else {
		B[a] = R[a];
		for (b = 0; b < N; b++)
		    if (A[a * N + b] != 0.0)
			row_add(&rows[I[a]], I[b], A[a * N + b]);
	    }
	}
	/* phgVecAddEntries_ (matvec.c:5661-5730): zeros skipped */
	for (a = 0; a < N; a++)
	    if (B[a] != 0.0)
		S->rhs_raw[I[a]] += B[a];
    }
    pack(rows, ndof, &S->raw_ptr, &S->raw_cols, &S->raw_vals);

    /* phgMatAssemble, serial path: boundary rows are already diagonal and
     * stay (save_local_bdry_equations skips them, matvec.c:4364-4366);
     * save_bdry_columns(mat, TRUE) (matvec.c:4430-4488) moves every boundary
     * column to bdry_rows, keeping the diagonal in both. */
    {
	ROW *brows = calloc(ndof, sizeof(*brows));
	for (i = 0; i < ndof; i++) {
	    ROW *r = &rows[i];
	    int64_t l = 0;
	    for (j = 0; j < r->n; j++) {
		int32_t c = r->cols[j];
		if (c == i || !bdry[c]) {
		    r->cols[l] = c;
		    r->vals[l++] = r->vals[j];
		}
		if (bdry[c])
		    row_add(&brows[i], c, r->vals[j]);
	    }
	    r->n = l;
	}
	pack(rows, ndof, &S->ptr, &S->cols, &S->vals);
	pack(brows, ndof, &S->bptr, &S->bcols, &S->bvals);
	for (i = 0; i < ndof; i++) {
	    free(brows[i].cols);
	    free(brows[i].vals);
	}
	free(brows);
    }
    for (i = 0; i < ndof; i++) {
	free(rows[i].cols);
	free(rows[i].vals);
    }
    free(rows);

    /* update_rhs(A, rhs, A, rhs, 1.0, TRUE) (solver.c:707-725):
     * rhs_i -= 1.0 * rhs_k * a_ik / D_kk over the saved boundary columns,
     * D_kk = the diagonal kept in bdry_rows[k] */
    S->rhs = malloc(ndof * sizeof(double));
    memcpy(S->rhs, S->rhs_raw, ndof * sizeof(double));
    for (i = 0; i < ndof; i++)
	for (j = S->bptr[i]; j < S->bptr[i + 1]; j++) {
	    int32_t k = S->bcols[j];
	    if (k == i)
		continue;
	    S->rhs[i] -= 1.0 * S->rhs[k] * S->bvals[j] / S->bvals[S->bptr[k]];
	}

    /* phgMatSetupDiagonal (matvec.c:500-549): first entry with col == i */
    S->diag = malloc(ndof * sizeof(double));
    for (i = 0; i < ndof; i++) {
	S->diag[i] = 0.0;
	for (j = S->ptr[i]; j < S->ptr[i + 1]; j++)
	    if (S->cols[j] == i) {
		S->diag[i] = S->vals[j];
		break;
	    }
    }
    return 0;
}

void
pho_system_free(pho_system *S)
{
    free(S->raw_ptr); free(S->raw_cols); free(S->raw_vals);
    free(S->ptr); free(S->cols); free(S->vals);
    free(S->bptr); free(S->bcols); free(S->bvals);
    free(S->rhs_raw); free(S->rhs); free(S->diag);
    memset(S, 0, sizeof(*S));
}

/*----------------------------- solver -----------------------------------*/

void
pho_spmv(int64_t n, const int64_t *ptr, const int32_t *cols,
	 const double *vals, const double *x, double *y)
/* phgMatVec CSR loop (matvec.c:891-928): beta = a_0 x_c0 + a_1 x_c1 + ... */
{
    int64_t i, j;
    for (i = 0; i < n; i++) {
	double beta;
	if (ptr[i + 1] == ptr[i]) {
	    y[i] = 0.0;
	    continue;
	}
	beta = vals[ptr[i]] * x[cols[ptr[i]]];
	for (j = ptr[i] + 1; j < ptr[i + 1]; j++)
	    beta += vals[j] * x[cols[j]];
	y[i] = 0.0 + beta;
    }
}

static double
norm2(int64_t n, const double *v)
/* phgVecNorm2 (matvec.c:51-90) */
{
    double s = 0.0;
    int64_t i;
    for (i = 0; i < n; i++)
	s += v[i] * v[i];
    return sqrt(s);
}

static double
dot(int64_t n, const double *x, const double *y)
/* phgVecDot (matvec.c:1193-1234) */
{
    double s = 0.0;
    int64_t i;
    for (i = 0; i < n; i++)
	s += x[i] * y[i];
    return s;
}

#define IS_ZERO(a) (fabs(a) < 10.0 * DBL_MIN)	/* utils.h:451 */

int
pho_pcg(int64_t n, const int64_t *ptr, const int32_t *cols,
	const double *vals, const double *diag, const double *b, double *x,
	int maxit, double rtol, double btol, double atol, double *res,
	double *hist)
/* solver_pcg (solver-phg.c:485-604) with jacobi_pc (:207-245). */
{
    double *r = malloc(n * sizeof(double)), *z = malloc(n * sizeof(double));
    double *p = malloc(n * sizeof(double)), *Ap = malloc(n * sizeof(double));
    double rb, r0, residual, tol, rz1 = 0., rz2, alpha, x1 = 0.0;
    int64_t i;
    int nits = 0;

    rb = norm2(n, b);
    if (IS_ZERO(rb)) {
	memset(x, 0, n * sizeof(double));
	free(r); free(z); free(p); free(Ap);
	if (res != NULL)
	    *res = 0.0;
	return 0;
    }
    for (i = 0; i < n; i++)
	x1 += fabs(x[i]);
    if (!IS_ZERO(x1 / n)) {
	/* r = b - A x: phgVecAXPBY(1.0, b, -1.0, &r) negates, then adds b */
	pho_spmv(n, ptr, cols, vals, x, r);
	for (i = 0; i < n; i++)
	    r[i] = -r[i];
	for (i = 0; i < n; i++)
	    r[i] += b[i];
    }
    else
	memcpy(r, b, n * sizeof(double));
    r0 = residual = norm2(n, r);
    /* get_tol (solver-phg.c:104-115) */
    tol = r0 * rtol;
    if (tol < rb * btol)
	tol = rb * btol;
    if (tol < atol)
	tol = atol;
    if (hist != NULL)
	hist[0] = residual;

    while (residual > tol && nits < maxit) {
	for (i = 0; i < n; i++)
	    z[i] = r[i] / diag[i];
	nits++;
	if (nits == 1) {
	    memcpy(p, z, n * sizeof(double));
	    rz1 = dot(n, r, z);
	}
	else {
	    double beta;
	    rz2 = rz1;
	    rz1 = dot(n, r, z);
	    if (rz2 == 0.0)
		break;
	    /* phgVecAXPBY(1.0, z, rz1 / rz2, &p): p = beta p, then p += z */
	    beta = rz1 / rz2;
	    if (beta != 1.0)
		for (i = 0; i < n; i++)
		    p[i] = beta * p[i];
	    for (i = 0; i < n; i++)
		p[i] += z[i];
	}
	pho_spmv(n, ptr, cols, vals, p, Ap);
	if ((alpha = dot(n, p, Ap)) == 0.0)
	    break;
	alpha = rz1 / alpha;
	for (i = 0; i < n; i++)
	    x[i] += alpha * p[i];
	alpha = -1.0 * alpha;
	for (i = 0; i < n; i++)
	    r[i] += alpha * Ap[i];
	residual = norm2(n, r);
	if (hist != NULL)
	    hist[nits] = residual;
    }
    free(r); free(z); free(p); free(Ap);
    if (res != NULL)
	*res = residual;
    return nits;
}

/* y = b y + a x with the rounding of phgVecAXPBY (matvec.c:1237-1295): the
 * special cases a, b = +-1 there give the same values as the general form. */
static void
axpby(int64_t n, double a, const double *x, double b, double *y)
{
    int64_t i;
    if (b != 1.0)
	for (i = 0; i < n; i++)
	    y[i] = b * y[i];
    if (a == 0.0)
	return;
    for (i = 0; i < n; i++)
	y[i] += a * x[i];
}

int
pho_bicgstab(int64_t n, const int64_t *ptr, const int32_t *cols,
	     const double *vals, const double *diag, const double *b,
	     double *x, int maxit, double rtol, double btol, double atol,
	     double *res, double *hist, int *status)
/* solver_BiCGstab (solver-phg.c:606-781) with jacobi_pc (:207-245).
 * *status: 0 normal end, 1 rho == 0 ("method failed"), 2 ||s|| <= 1e-60
 * (x corrected and the residual recomputed from b - A x). */
{
    double *r1 = malloc(n * sizeof(double)), *rg = malloc(n * sizeof(double));
    double *rh = malloc(n * sizeof(double)), *pg = malloc(n * sizeof(double));
    double *ph = calloc(n, sizeof(double)), *sg = malloc(n * sizeof(double));
    double *sh = calloc(n, sizeof(double)), *tg = malloc(n * sizeof(double));
    double *vg = malloc(n * sizeof(double));
    double rb, r0, residual, tol, rho0 = 0., rho1, alpha = 0., beta, omega = 0.;
    double x1 = 0.0;
    int64_t i;
    int nits = 0;

    if (status != NULL)
	*status = 0;
    rb = norm2(n, b);
    if (IS_ZERO(rb)) {
	memset(x, 0, n * sizeof(double));
	residual = 0.0;
	goto done;
    }
    for (i = 0; i < n; i++)
	x1 += fabs(x[i]);
    if (!IS_ZERO(x1 / n)) {
	pho_spmv(n, ptr, cols, vals, x, r1);
	memcpy(rg, r1, n * sizeof(double));
	axpby(n, 1.0, b, -1.0, rg);
    }
    else
	memcpy(rg, b, n * sizeof(double));
    r0 = residual = norm2(n, rg);
    tol = r0 * rtol;
    if (tol < rb * btol)
	tol = rb * btol;
    if (tol < atol)
	tol = atol;
    if (hist != NULL)
	hist[0] = residual;
    memcpy(rh, rg, n * sizeof(double));

    while (residual > tol && nits < maxit) {
	nits++;
	rho1 = dot(n, rg, rh);
	if (rho1 == 0.0) {
	    if (status != NULL)
		*status = 1;
	    break;
	}
	if (nits == 1)
	    memcpy(pg, rg, n * sizeof(double));
	else {
	    beta = (rho1 * alpha) / (rho0 * omega);
	    memcpy(sg, pg, n * sizeof(double));
	    axpby(n, -omega, vg, 1., sg);
	    memcpy(pg, rg, n * sizeof(double));
	    axpby(n, beta, sg, 1., pg);
	}
	rho0 = rho1;
	for (i = 0; i < n; i++)
	    ph[i] = pg[i] / diag[i];
	pho_spmv(n, ptr, cols, vals, ph, vg);
	alpha = rho1 / dot(n, rh, vg);
	memcpy(sg, rg, n * sizeof(double));
	axpby(n, -alpha, vg, 1., sg);
	omega = norm2(n, sg);
	if (omega <= 1e-60) {
	    axpby(n, alpha, ph, 1., x);
	    pho_spmv(n, ptr, cols, vals, x, r1);
	    memcpy(rg, b, n * sizeof(double));
	    axpby(n, -1, r1, 1., rg);
	    residual = norm2(n, rg);
	    if (hist != NULL)
		hist[nits] = residual;
	    if (status != NULL)
		*status = 2;
	    break;
	}
	for (i = 0; i < n; i++)
	    sh[i] = sg[i] / diag[i];
	pho_spmv(n, ptr, cols, vals, sh, tg);
	omega = dot(n, tg, sg) / dot(n, tg, tg);
	axpby(n, omega, sh, alpha, ph);
	axpby(n, 1, ph, 1, x);
	memcpy(rg, sg, n * sizeof(double));
	axpby(n, -omega, tg, 1, rg);
	residual = norm2(n, rg);
	if (hist != NULL)
	    hist[nits] = residual;
	if (residual <= tol)
	    break;
    }
done:
    free(r1); free(rg); free(rh); free(pg); free(ph);
    free(sg); free(sh); free(tg); free(vg);
    if (res != NULL)
	*res = residual;
    return nits;
}

/* y = alpha x (+ y when accumulate): phgMatVec with A = NULL
 * (matvec.c:606-760); the special cases alpha = +-1 give the same values. */
static void
scale_add(int64_t n, double alpha, const double *x, int accumulate, double *y)
{
    int64_t i;
    if (accumulate)
	for (i = 0; i < n; i++)
	    y[i] += alpha * x[i];
    else
	for (i = 0; i < n; i++)
	    y[i] = alpha * x[i];
}

/* z = b - A x as phgVecCopy(b, &z) + phgMatVec(MAT_OP_N, -1.0, A, x, 1.0,
 * &z) (matvec.c:840-928): each row adds sum_j a_ij (-x_j), which equals
 * b_i - sum_j a_ij x_j exactly. */
static void
residual_vec(int64_t n, const int64_t *ptr, const int32_t *cols,
	     const double *vals, const double *b, const double *x, double *z)
{
    int64_t i, j;
    for (i = 0; i < n; i++) {
	double s;
	z[i] = b[i];
	if (ptr[i + 1] == ptr[i])
	    continue;
	s = vals[ptr[i]] * -x[cols[ptr[i]]];
	for (j = ptr[i] + 1; j < ptr[i + 1]; j++)
	    s += vals[j] * -x[cols[j]];
	z[i] += s;
    }
}

int
pho_gmres(int64_t n, const int64_t *ptr, const int32_t *cols,
	  const double *vals, const double *diag, const double *b, double *x,
	  int restart, int maxit, double rtol, double btol, double atol,
	  double *res)
/* solver_GMRES_r (solver-phg.c:1050-1260): right-preconditioned restarted
 * GMRES with modified Gram-Schmidt and Givens rotations, Jacobi PC.  The
 * residual reported is the rotated estimate |s[i+1]| at convergence and
 * ||r0|| when maxit ends the run, as in the reference. */
{
    int R, nits = 0, i, j, k;
    double b_norm, r0_norm, r_norm, residual, tol, tmp, h1, h2, x1 = 0.0;
    double **V, *H, *y, *s, *c1, *c2, *z, *r;
    int64_t l;

    if (restart <= 0)
	restart = maxit + 1;
    R = restart + 2;
    b_norm = norm2(n, b);
    if (IS_ZERO(b_norm)) {
	memset(x, 0, n * sizeof(double));
	if (res != NULL)
	    *res = 0.0;
	return 0;
    }
    V = malloc(R * sizeof(*V));
    for (i = 0; i < R; i++)
	V[i] = malloc(n * sizeof(double));
    H = malloc((size_t)R * R * sizeof(double));
    y = malloc(4 * R * sizeof(double));
    s = y + R;
    c1 = y + 2 * R;
    c2 = y + 3 * R;
    z = malloc(n * sizeof(double));
    r = V[0];
#define Hij(a, b) H[(size_t)(a) * R + (b)]

    for (l = 0; l < n; l++)
	x1 += fabs(x[l]);
    if (x1 != 0.)
	residual_vec(n, ptr, cols, vals, b, x, z);
    else
	memcpy(z, b, n * sizeof(double));
    r0_norm = r_norm = residual = norm2(n, z);
    tol = r0_norm * rtol;
    if (tol < b_norm * btol)
	tol = b_norm * btol;
    if (tol < atol)
	tol = atol;

    s[0] = 1.;
    while (nits < maxit) {
	s[1] = r_norm = norm2(n, z);
	scale_add(n, 1.0 / r_norm, z, 0, V[1]);
	i = 0;
	memset(H, 0, (size_t)R * R * sizeof(double));
	while (i < restart && r_norm > tol && nits < maxit) {
	    double *v1;
	    i++, nits++;
	    v1 = V[i + 1];
	    for (l = 0; l < n; l++)
		r[l] = V[i][l] / diag[l];
	    pho_spmv(n, ptr, cols, vals, r, v1);
	    for (k = 1; k <= i; k++) {
		Hij(i, k) = dot(n, v1, V[k]);
		scale_add(n, -Hij(i, k), V[k], 1, v1);
	    }
	    Hij(i, i + 1) = norm2(n, v1);
	    if (IS_ZERO(Hij(i, i + 1))) {
		i--;
		break;
	    }
	    tmp = 1.0 / Hij(i, i + 1);
	    for (l = 0; l < n; l++)
		v1[l] *= tmp;
	    for (j = 1; j < i; j++) {
		h1 = c1[j] * Hij(i, j) + c2[j] * Hij(i, j + 1);
		h2 = -c2[j] * Hij(i, j) + c1[j] * Hij(i, j + 1);
		Hij(i, j) = h1;
		Hij(i, j + 1) = h2;
	    }
	    tmp = sqrt(Hij(i, i) * Hij(i, i) + Hij(i, i + 1) * Hij(i, i + 1));
	    if (IS_ZERO(tmp))
		tmp = 1.e-16;
	    c1[i] = Hij(i, i) / tmp;
	    c2[i] = Hij(i, i + 1) / tmp;
	    s[i + 1] = -c2[i] * s[i];
	    s[i] = c1[i] * s[i];
	    Hij(i, i) = c1[i] * Hij(i, i) + c2[i] * Hij(i, i + 1);
	    r_norm = fabs(s[i + 1]);
	    if (r_norm <= tol)
		break;
	}
	for (j = i; j > 0; j--) {
	    y[j] = s[j] / Hij(j, j);
	    for (k = j - 1; k > 0; k--)
		s[k] -= Hij(j, k) * y[j];
	}
	if (i > 0) {
	    scale_add(n, y[1], V[1], 0, z);
	    for (j = 2; j <= i; j++)
		scale_add(n, y[j], V[j], 1, z);
	}
	for (l = 0; l < n; l++)
	    r[l] = z[l] / diag[l];
	for (l = 0; l < n; l++)
	    x[l] += r[l];
	if (r_norm <= tol) {
	    residual = r_norm;
	    break;
	}
	residual_vec(n, ptr, cols, vals, b, x, z);
    }
#undef Hij
    for (i = 0; i < R; i++)
	free(V[i]);
    free(V); free(H); free(y); free(z);
    if (res != NULL)
	*res = residual;
    return nits;
}

int
pho_flgmres(int64_t n, const int64_t *ptr, const int32_t *cols,
	    const double *vals, const double *diag, const double *b, double *x,
	    int restart, int augk, int maxit, double rtol, double btol,
	    double atol, double *res)
/* solver_FLGMRES_r (solver-phg.c:2063-2340), PHG's default GMRES: flexible
 * right-preconditioned GMRES whose basis is augmented with the corrections z
 * of the last augk cycles (preconditioned like the basis vectors).  Cycle k
 * (k = 0, 1, ...) runs up to mk + min(k, augk) steps, mk the restart; steps
 * past mk precondition the stored corrections.  x += sum_j y_j M^-1 v_j with
 * the preconditioned vectors kept (flv); the stored correction is sum_j y_j
 * v_j over the unpreconditioned vectors (and the augmenting corrections).
 * When a cycle ends without a step (happy breakdown at its first step) the
 * reference adds the cycle's starting residual z to x, and so does this. */
{
    int R, mk, nits = 0, i, j, k, itr_out = 0, zi;
    double b_norm, r0_norm, r_norm, residual, tol, tmp, h1, h2, x1 = 0.0;
    double **V, **Z, **F, *H, *y, *s, *c1, *c2, *z, *r;
    int64_t l;

    if (restart <= 0)
	restart = maxit + 1;
    if (augk <= 0)
	augk = 2;
    b_norm = norm2(n, b);
    if (IS_ZERO(b_norm)) {
	memset(x, 0, n * sizeof(double));
	if (res != NULL)
	    *res = 0.0;
	return 0;
    }
    mk = restart;
    restart += augk;
    R = restart + 2;
    V = malloc(R * sizeof(*V));
    F = malloc(R * sizeof(*F));
    for (i = 0; i < R; i++) {
	V[i] = malloc(n * sizeof(double));
	F[i] = malloc(n * sizeof(double));
    }
    Z = malloc(augk * sizeof(*Z));
    for (i = 0; i < augk; i++)
	Z[i] = calloc(n, sizeof(double));
    H = malloc((size_t)R * R * sizeof(double));
    y = malloc(4 * R * sizeof(double));
    s = y + R;
    c1 = y + 2 * R;
    c2 = y + 3 * R;
    z = malloc(n * sizeof(double));
    r = V[0];
#define Hij(a, b) H[(size_t)(a) * R + (b)]

    for (l = 0; l < n; l++)
	x1 += fabs(x[l]);
    if (x1 != 0.)
	residual_vec(n, ptr, cols, vals, b, x, z);
    else
	memcpy(z, b, n * sizeof(double));
    r0_norm = r_norm = residual = norm2(n, z);
    tol = r0_norm * rtol;
    if (tol < b_norm * btol)
	tol = b_norm * btol;
    if (tol < atol)
	tol = atol;

    s[0] = 1.;
    while (nits < maxit) {
	restart = itr_out <= augk ? mk + itr_out : mk + augk;
	s[1] = r_norm = norm2(n, z);
	scale_add(n, 1.0 / r_norm, z, 0, V[1]);
	i = 0;
	memset(H, 0, (size_t)R * R * sizeof(double));
	while (i < restart && r_norm > tol && nits < maxit) {
	    double *v1;
	    const double *src;
	    i++, nits++;
	    v1 = V[i + 1];
	    src = i <= mk ? V[i] : Z[i - mk - 1];
	    for (l = 0; l < n; l++)
		r[l] = src[l] / diag[l];
	    pho_spmv(n, ptr, cols, vals, r, v1);
	    memcpy(F[i], r, n * sizeof(double));
	    for (k = 1; k <= i; k++) {
		Hij(i, k) = dot(n, v1, V[k]);
		scale_add(n, -Hij(i, k), V[k], 1, v1);
	    }
	    Hij(i, i + 1) = norm2(n, v1);
	    if (IS_ZERO(Hij(i, i + 1))) {
		i--;
		break;
	    }
	    tmp = 1.0 / Hij(i, i + 1);
	    for (l = 0; l < n; l++)
		v1[l] *= tmp;
	    for (j = 1; j < i; j++) {
		h1 = c1[j] * Hij(i, j) + c2[j] * Hij(i, j + 1);
		h2 = -c2[j] * Hij(i, j) + c1[j] * Hij(i, j + 1);
		Hij(i, j) = h1;
		Hij(i, j + 1) = h2;
	    }
	    tmp = sqrt(Hij(i, i) * Hij(i, i) + Hij(i, i + 1) * Hij(i, i + 1));
	    if (IS_ZERO(tmp))
		tmp = 1.e-16;
	    c1[i] = Hij(i, i) / tmp;
	    c2[i] = Hij(i, i + 1) / tmp;
	    s[i + 1] = -c2[i] * s[i];
	    s[i] = c1[i] * s[i];
	    Hij(i, i) = c1[i] * Hij(i, i) + c2[i] * Hij(i, i + 1);
	    r_norm = fabs(s[i + 1]);
	    if (r_norm <= tol)
		break;
	}
	for (j = i; j > 0; j--) {
	    y[j] = s[j] / Hij(j, j);
	    for (k = j - 1; k > 0; k--)
		s[k] -= Hij(j, k) * y[j];
	}
	if (i > 0) {
	    scale_add(n, y[1], F[1], 0, z);
	    for (j = 2; j <= i; j++)
		scale_add(n, y[j], F[j], 1, z);
	}
	for (l = 0; l < n; l++)
	    x[l] = z[l] + x[l];
	if (i > 0) {
	    int top = i <= mk ? i : mk;
	    scale_add(n, y[1], V[1], 0, z);
	    for (j = 2; j <= top; j++)
		scale_add(n, y[j], V[j], 1, z);
	    if (i > mk) {
		int ak = itr_out < augk ? itr_out : augk;
		for (j = 1; j <= ak; j++)
		    scale_add(n, y[j + mk], Z[j - 1], 1, z);
	    }
	}
	zi = itr_out % augk;
	memcpy(Z[zi], z, n * sizeof(double));
	if (r_norm <= tol) {
	    residual = r_norm;
	    break;
	}
	residual_vec(n, ptr, cols, vals, b, x, z);
	itr_out++;
    }
#undef Hij
    for (i = 0; i < R; i++) {
	free(V[i]);
	free(F[i]);
    }
    for (i = 0; i < augk; i++)
	free(Z[i]);
    free(V); free(F); free(Z); free(H); free(y); free(z);
    if (res != NULL)
	*res = residual;
    return nits;
}
