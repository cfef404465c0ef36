/*
 * phg_oracle -- CPU restatement of the reference (PHG 0.9.7) arithmetic for
 * the element-assembly + Jacobi-PCG path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle that tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg compare with.  The product
 * (phg_b200/) never links, loads or calls it.
 *
 * Every routine follows one reference routine operation by operation (same
 * operand order, no fused multiply-add: compiled with -ffp-contract=off) so
 * that its doubles match the reference's bit for bit; each one cites the
 * reference file:line it restates.
 *
 * Conventions (as in the reference's serial build, FLOAT = double,
 * INT = int): a tetrahedron has local vertices 0..3, local edges
 * 0:(0,1) 1:(0,2) 2:(0,3) 3:(1,2) 4:(1,3) 5:(2,3), local face k opposite
 * vertex k.  Lagrange P1/P2/P3 local bases are ordered vertices, edges
 * (two per edge for P3, first one nearest the edge's first local vertex),
 * faces.  Element->DOF maps (`e2l`) already include the edge orientation
 * that phgDofMapE2D applies, so DOF values are read as v[e2l[e*N + k]].
 */
#ifndef PHG_ORACLE_H
#define PHG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 4x4 barycentric Jacobian, J[i*4+k] = d lambda_i / d x_k (k < 3),
 * J[i*4+3] = c_i (geom.c:103-169).  x = 4 vertices x 3 coordinates. */
void pho_jacobian(const double *x, double *J);
/* |det| / 6 (geom.c:46-78) */
double pho_volume(const double *x);

/* Quadrature rule of the given order (quad.c:2914 + rules :1799-1988):
 * returns the number of points, and pointers to barycentric points
 * (npoints x 4) and weights (sum 1).  Orders 0..6.  Returns -1 otherwise. */
int pho_quad_rule(int order, const double **pts, const double **wts);

/* Number of P-order Lagrange basis functions (4, 10, 20). */
int pho_nbas(int p);
/* Basis values at barycentric point lambda (lagrange.c:80,160,392). */
void pho_bas(int p, const double *lambda, double *values);
/* d phi / d lambda, N x 4 (lagrange.c:111,248,538). */
void pho_grad_lambda(int p, const double *lambda, double *grads);

/* Element matrices.  `kappa` < 0 means "no coefficient" (A = NULL in the
 * reference), otherwise a piecewise-constant coefficient.  A is N x N
 * row-major: A[a*N+b] = integral of grad phi_b . kappa grad phi_a, computed
 * as the reference's user loop calls it for b <= a and mirrored.
 * quad.c:5260-5344 (stiffness), quad.c:3314-3421 (basis gradients),
 * quad.c:5582-5674 (mass). */
void pho_elem_stiffness(int p, const double *x, double kappa, double *A);
void pho_elem_mass(int p, const double *x, double *M);
/* b[a] = integral of f_h phi_a where f_h has local DOF values f_local
 * (quad.c:5481-5530 with phgQuadGetDofValues quad.c:3552 / phgDofEval_
 * dof-utils.c:59-300). */
void pho_elem_rhs(int p, const double *x, const double *f_local, double *b);

/* Result of assembling the linear system the way the reference's user loop
 * (examples/poisson.c:101-170) + phgSolverAssemble + phgSolverUpdateRHS do.
 * All arrays are allocated by the oracle; free with pho_system_free. */
typedef struct {
    int64_t n;			/* rows = DOFs */
    /* rows before phgMatAssemble (first-touch order, zeros dropped) */
    int64_t *raw_ptr; int32_t *raw_cols; double *raw_vals;
    /* rows after boundary-column removal (matvec.c:4430-4488) */
    int64_t *ptr; int32_t *cols; double *vals;
    /* saved boundary columns (bdry_rows) */
    int64_t *bptr; int32_t *bcols; double *bvals;
    double *rhs_raw;		/* after phgSolverAddRHSEntries */
    double *rhs;		/* after update_rhs (solver.c:508-731) */
    double *diag;		/* phgMatSetupDiagonal (matvec.c:500-549) */
} pho_system;

/* kappa may be NULL (no coefficient), g may be NULL (zero BC). */
int pho_assemble(int p, int64_t nvert, const double *verts, int64_t nelem,
		 const int32_t *elems, const int32_t *e2l, int64_t ndof,
		 const uint8_t *bdry, const double *f, const double *g,
		 const double *kappa, double mass_coef, const double *geom,
		 pho_system *sys);
void pho_system_free(pho_system *sys);

/* y = A x for the CSR (ptr int64) (matvec.c:891-928). */
void pho_spmv(int64_t n, const int64_t *ptr, const int32_t *cols,
	      const double *vals, const double *x, double *y);

/* Jacobi-PCG (solver-phg.c:485-604, jacobi_pc :207-245, get_tol :104).
 * x holds the initial guess on entry and the solution on exit.  Returns
 * the number of iterations; *residual gets the final residual 2-norm.
 * hist (optional, length maxit+1) gets the residual after each iteration,
 * hist[0] = initial residual. */
int pho_pcg(int64_t n, const int64_t *ptr, const int32_t *cols,
	    const double *vals, const double *diag, const double *b,
	    double *x, int maxit, double rtol, double btol, double atol,
	    double *residual, double *hist);

/* Jacobi-preconditioned BiCGstab (solver_BiCGstab, solver-phg.c:606-781):
 * arguments as pho_pcg; hist[k] = ||r|| after iteration k.  *status (may be
 * NULL): 0 normal end, 1 rho = 0 (the reference's "method failed" break),
 * 2 ||s|| <= 1e-60 (x corrected, residual recomputed from b - A x). */
int pho_bicgstab(int64_t n, const int64_t *ptr, const int32_t *cols,
		 const double *vals, const double *diag, const double *b,
		 double *x, int maxit, double rtol, double btol, double atol,
		 double *residual, double *hist, int *status);

/* Restarted right-preconditioned GMRES with the Jacobi PC (solver_GMRES_r,
 * solver-phg.c:1050-1260; -solver gmres -gmres_type gmres_r).  restart <= 0
 * means no restart.  *residual: the rotated residual estimate at
 * convergence, ||r0|| when maxit ends the run (as the reference). */
int pho_gmres(int64_t n, const int64_t *ptr, const int32_t *cols,
	      const double *vals, const double *diag, const double *b,
	      double *x, int restart, int maxit, double rtol, double btol,
	      double atol, double *residual);

/* PHG's default GMRES, flexible augmented FLGMRES_r (solver_FLGMRES_r,
 * solver-phg.c:2063-2340; -solver gmres, -gmres_type flgmres_r the default):
 * restart steps plus up to augk (<= 0: 2) steps on the corrections of the
 * previous cycles, Jacobi PC.  *residual as pho_gmres. */
int pho_flgmres(int64_t n, const int64_t *ptr, const int32_t *cols,
		const double *vals, const double *diag, const double *b,
		double *x, int restart, int augk, int maxit, double rtol,
		double btol, double atol, double *residual);

#ifdef __cplusplus
}
#endif
#endif
