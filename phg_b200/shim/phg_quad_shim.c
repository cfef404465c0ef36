/*
 * Per-call drop-in for PHG's element integrals, answered from a table the
 * GPU computes for the whole mesh at once.
 *
 * Loaded ahead of a shared PHG library (LD_PRELOAD, or linked before
 * libphg), this library defines
 *
 *   FLOAT  phgQuadGradBasAGradBas(ELEMENT *e, DOF *u, int n, DOF *A,
 *                                 DOF *v, int m, int order)
 *   FLOAT  phgQuadBasABas(ELEMENT *e, DOF *u, int n, DOF *A, DOF *v,
 *                         int m, int order)
 *   FLOAT *phgQuadDofTimesBas(ELEMENT *e, DOF *u, DOF *v, int n, int order,
 *                             FLOAT *res)
 *
 * with the reference's signatures (include/phg/quad.h:136-146).  For the
 * cases the GPU element kernel covers -- u == v a scalar Lagrange P1/P2/P3
 * DOF, A NULL or a scalar P0 coefficient (NULL only, for the mass matrix
 * phgQuadBasDotBas), the default quadrature order -- the first call for a
 * mesh computes every element's matrix (or right-hand side) with
 * phgGpuElementMatrices and later calls read the table: the values are bit
 * for bit those of src/quad.c:5260-5344, 5582-5674 and 5481-5530.
 * Every other call goes to PHG's own function (dlsym RTLD_NEXT), so an
 * unmodified user program (examples/poisson.c) runs unchanged.
 *
 * A table is rebuilt when the grid changes (GRID pointer, serial_no, element
 * count), when another DOF type or coefficient DOF is used, and -- checked
 * when the element loop starts again (the table's first call repeats) -- when
 * the coefficient's or source's values changed.  Calls are serialised by a
 * mutex (the build is lazy), so OpenMP element loops may call in.  Set
 * PHG_QUAD_SHIM_STATS to print how many calls were answered at exit.
 */
#define _GNU_SOURCE
#include "phg.h"
#include "phg_gpu.h"

#include <dlfcn.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef FLOAT (*gbag_fn)(ELEMENT *, DOF *, int, DOF *, DOF *, int, int);
typedef FLOAT *(*dtb_fn)(ELEMENT *, DOF *, DOF *, int, int, FLOAT *);
typedef FLOAT (*baab_fn)(ELEMENT *, DOF *, int, DOF *, DOF *, int, int);

typedef struct {
    FLOAT *val;              /* nelem x N x N (matrices) or nelem x N (rhs) */
    DOF *coef;               /* the coefficient (A) or source (u) DOF */
    uint64_t sum;            /* checksum of coef's values when built */
    INT first_e;             /* the first call after the build ... */
    int first_n, first_m;    /* ... marks the start of an element loop */
    int valid;
} Table;

static struct {
    pthread_mutex_t lock;
    phgGpuSystem *sys;
    GRID *g;
    int serial;
    INT nelem;
    DOF_TYPE *type;
    int N, p;
    Table K, R, M;
    long served_k, served_r, served_m, forwarded;
    int stats_registered;
} S = {PTHREAD_MUTEX_INITIALIZER};

static gbag_fn orig_gbag(void) {
    static gbag_fn f = NULL;
    if (f == NULL) f = (gbag_fn)dlsym(RTLD_NEXT, "phgQuadGradBasAGradBas");
    return f;
}

static dtb_fn orig_dtb(void) {
    static dtb_fn f = NULL;
    if (f == NULL) f = (dtb_fn)dlsym(RTLD_NEXT, "phgQuadDofTimesBas");
    return f;
}

static baab_fn orig_baab(void) {
    static baab_fn f = NULL;
    if (f == NULL) f = (baab_fn)dlsym(RTLD_NEXT, "phgQuadBasABas");
    return f;
}

static int lagrange_order(DOF *u) {
    if (u == NULL || u->dim != 1) return 0;
    if (u->type == DOF_P1) return 1;
    if (u->type == DOF_P2) return 2;
    if (u->type == DOF_P3) return 3;
    return 0;
}

static uint64_t checksum(DOF *d) {
    uint64_t h = 1469598103934665603ull;
    INT i, n;
    if (d == NULL) return 0;
    n = DofDataCount(d);
    for (i = 0; i < n; i++) {
        uint64_t b;
        memcpy(&b, d->data + i, sizeof(b));
        h = (h ^ b) * 1099511628211ull;
    }
    return h;
}

static void print_stats(void) {
    fprintf(stderr, "phg_quad_shim: stiffness %ld from the GPU table, rhs %ld, mass %ld, forwarded %ld\n",
            S.served_k, S.served_r, S.served_m, S.forwarded);
}

static void fail(const char *what) {
    fprintf(stderr, "phg_quad_shim: %s: %s\n", what, phgGpuLastError());
    abort();
}

/* Uploads the grid and u's element -> data map (called with the lock held). */
static void prepare(GRID *g, DOF *u) {
    ELEMENT *e;
    INT *elems, *e2l;
    double *geo;
    unsigned char *bdry;
    INT ndof, it;
    int k;
    if (S.g == g && S.serial == g->serial_no && S.nelem == g->nelem && S.type == u->type) return;
    if (S.sys == NULL && phgGpuCreate(0, NULL, &S.sys) != PHG_GPU_OK) fail("phgGpuCreate");
    S.p = lagrange_order(u);
    S.N = u->type->nbas;
    elems = (INT *)malloc(sizeof(INT) * 4 * (size_t)g->nelem);
    e2l = (INT *)malloc(sizeof(INT) * (size_t)S.N * g->nelem);
    ndof = DofDataCount(u);
    bdry = (unsigned char *)calloc((size_t)ndof, 1);
    /* the user's element loop is running (ForAllElements keeps its index in
     * the grid): loop with an index of our own */
    ForAllElements2(g, e, it) {
        for (k = 0; k < 4; k++) elems[4 * (size_t)e->index + k] = e->verts[k];
        for (k = 0; k < S.N; k++) e2l[(size_t)S.N * e->index + k] = phgDofMapE2D_(u, e, k, FALSE);
    }
    if (phgGpuSetMesh(S.sys, g->nvert, &g->verts[0][0], g->nelem, elems) != PHG_GPU_OK) fail("phgGpuSetMesh");
    /* PHG's own Jacobians and volumes (interpolated from the parent on
     * elements made by bisection, geom.c:460-565), which its phgQuad* use */
    geo = (double *)malloc(sizeof(double) * 17 * (size_t)g->nelem);
    ForAllElements2(g, e, it) {
        const FLOAT *J = phgGeomGetJacobian(g, e);
        for (k = 0; k < 16; k++) geo[17 * (size_t)e->index + k] = J[k];
        geo[17 * (size_t)e->index + 16] = phgGeomGetVolume(g, e);
    }
    if (phgGpuSetGeometry(S.sys, g->nelem, geo) != PHG_GPU_OK) fail("phgGpuSetGeometry");
    free(geo);
    if (phgGpuSetDofMap(S.sys, S.p, ndof, e2l, bdry) != PHG_GPU_OK) fail("phgGpuSetDofMap");
    free(elems);
    free(e2l);
    free(bdry);
    S.g = g;
    S.serial = g->serial_no;
    S.nelem = g->nelem;
    S.type = u->type;
    S.K.valid = S.R.valid = S.M.valid = 0;
    if (!S.stats_registered && getenv("PHG_QUAD_SHIM_STATS") != NULL) {
        atexit(print_stats);
        S.stats_registered = 1;
    }
}

static void build_K(DOF *A, ELEMENT *e, int n, int m) {
    FLOAT *kappa = NULL;
    ELEMENT *el;
    INT it;
    if (A != NULL) {
        kappa = (FLOAT *)malloc(sizeof(FLOAT) * (size_t)S.nelem);
        ForAllElements2(S.g, el, it) kappa[el->index] = A->data[phgDofMapE2D_(A, el, 0, FALSE)];
    }
    S.K.val = (FLOAT *)realloc(S.K.val, sizeof(FLOAT) * (size_t)S.nelem * S.N * S.N);
    if (phgGpuElementMatrices(S.sys, kappa, 0.0, NULL, S.K.val, NULL) != PHG_GPU_OK) fail("phgGpuElementMatrices");
    free(kappa);
    S.K.coef = A;
    S.K.sum = checksum(A);
    S.K.first_e = e->index;
    S.K.first_n = n;
    S.K.first_m = m;
    S.K.valid = 1;
}

/* The mass matrices: with kappa = 0 the element kernel's entry is
 * 0 + 1 * (vol * sum_q w_q phi_n phi_m), the reference's phgQuadBasABas
 * value (A = NULL, order 2p). */
static void build_M(void) {
    FLOAT *zero = (FLOAT *)calloc((size_t)S.nelem, sizeof(FLOAT));
    S.M.val = (FLOAT *)realloc(S.M.val, sizeof(FLOAT) * (size_t)S.nelem * S.N * S.N);
    if (phgGpuElementMatrices(S.sys, zero, 1.0, NULL, S.M.val, NULL) != PHG_GPU_OK) fail("phgGpuElementMatrices");
    free(zero);
    S.M.coef = NULL;
    S.M.valid = 1;
}

static void build_R(DOF *f, ELEMENT *e, int n) {
    S.R.val = (FLOAT *)realloc(S.R.val, sizeof(FLOAT) * (size_t)S.nelem * S.N);
    if (phgGpuElementMatrices(S.sys, NULL, 0.0, f->data, NULL, S.R.val) != PHG_GPU_OK)
        fail("phgGpuElementMatrices");
    S.R.coef = f;
    S.R.sum = checksum(f);
    S.R.first_e = e->index;
    S.R.first_n = n;
    S.R.first_m = 0;
    S.R.valid = 1;
}

FLOAT phgQuadGradBasAGradBas(ELEMENT *e, DOF *u, int n, DOF *A, DOF *v, int m, int order) {
    const int p = lagrange_order(u);
    FLOAT r;
    if (p == 0 || v != u || (A != NULL && (A->type != DOF_P0 || A->dim != 1)) ||
        (order >= 0 && order != 2 * (p - 1))) {
        __atomic_add_fetch(&S.forwarded, 1, __ATOMIC_RELAXED);
        return orig_gbag()(e, u, n, A, v, m, order);
    }
    pthread_mutex_lock(&S.lock);
    prepare(u->g, u);
    if (!S.K.valid || S.K.coef != A)
        build_K(A, e, n, m);
    else if (e->index == S.K.first_e && n == S.K.first_n && m == S.K.first_m && checksum(A) != S.K.sum)
        build_K(A, e, n, m);
    r = S.K.val[((size_t)e->index * S.N + m) * S.N + n];
    S.served_k++;
    pthread_mutex_unlock(&S.lock);
    return r;
}

FLOAT *phgQuadDofTimesBas(ELEMENT *e, DOF *u, DOF *v, int n, int order, FLOAT *res) {
    const int p = lagrange_order(v);
    if (p == 0 || u == NULL || u->type != v->type || u->dim != 1 || u->g != v->g ||
        (order >= 0 && order != 2 * p)) {
        __atomic_add_fetch(&S.forwarded, 1, __ATOMIC_RELAXED);
        return orig_dtb()(e, u, v, n, order, res);
    }
    pthread_mutex_lock(&S.lock);
    prepare(v->g, v);
    if (!S.R.valid || S.R.coef != u)
        build_R(u, e, n);
    else if (e->index == S.R.first_e && n == S.R.first_n && checksum(u) != S.R.sum)
        build_R(u, e, n);
    res[0] = S.R.val[(size_t)e->index * S.N + n];
    S.served_r++;
    pthread_mutex_unlock(&S.lock);
    return res;
}

FLOAT phgQuadBasABas(ELEMENT *e, DOF *u, int n, DOF *A, DOF *v, int m, int order) {
    const int p = lagrange_order(u);
    FLOAT r;
    /* A != NULL, another order, or a type with mass lumping go to PHG */
    if (p == 0 || v != u || A != NULL || (order >= 0 && order != 2 * p) ||
        (u->type->mass_lumping != NULL && u->type->mass_lumping->weights != NULL)) {
        __atomic_add_fetch(&S.forwarded, 1, __ATOMIC_RELAXED);
        return orig_baab()(e, u, n, A, v, m, order);
    }
    pthread_mutex_lock(&S.lock);
    prepare(u->g, u);
    if (!S.M.valid)
        build_M();
    r = S.M.val[((size_t)e->index * S.N + m) * S.N + n];
    S.served_m++;
    pthread_mutex_unlock(&S.lock);
    return r;
}
