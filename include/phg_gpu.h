/*
 * phg_gpu.h -- C ABI of the B200 (sm_100a) element-assembly + Jacobi-PCG
 * path for PHG (Parallel Hierarchical Grid) tetrahedral Lagrange P1/P2/P3
 * finite elements.
 *
 * The library stands in for the reference's element loop and linear-solver
 * calls.  PHG keeps the mesh, refinement and DOF numbering on the host; the
 * host hands the arrays PHG already holds to this ABI:
 *
 *   GRID  g->verts (FLOAT[nvert][3]), e->verts (INT[4] per element)
 *   DOF   the vector index of every element basis function
 *         (phgSolverMapE2L, include/phg/solver.h:297), the Dirichlet flag of
 *         every DOF (what phgDofDirichletBC returns), f_h->data, and the
 *         per-element coefficient (DOF_P0 data)
 *
 * and gets back the same CSR matrix, right-hand side and PCG solution the
 * reference computes.  Types follow the reference's default build:
 * FLOAT = double, INT = int (include/phg.h:88,97).
 *
 * Pointer arguments may be host or device memory (the library asks the CUDA
 * runtime which); device pointers must be on the system's device.  All
 * functions return PHG_GPU_OK (0) or a negative PHG_GPU_ERR_* code, and
 * phgGpuLastError() describes the last failure of the calling thread.  One
 * system is used from one host thread at a time; its work is issued in
 * order on its stream.
 */
#ifndef PHG_GPU_H
#define PHG_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHG_GPU_OK		0
#define PHG_GPU_ERR_ARG		(-1)	/* invalid argument / index */
#define PHG_GPU_ERR_CUDA	(-2)	/* CUDA runtime error */
#define PHG_GPU_ERR_STATE	(-3)	/* call out of order */
#define PHG_GPU_ERR_LIMIT	(-4)	/* size beyond a documented limit */
#define PHG_GPU_ERR_BREAKDOWN	(-5)	/* breakdown the reference cannot continue
					   from (BiCGstab, the adjoint solve) */
#define PHG_GPU_ERR_NAN		(-6)	/* non-finite value in the iteration */

typedef struct phgGpuSystem_ phgGpuSystem;

/* Text of the calling thread's last error ("" if none). */
const char *phgGpuLastError(void);
/* Text of the warning the calling thread's last solver call raised ("" if
 * none; every solver call clears it).  A PCG breakdown -- r.z or p.Ap of 0,
 * where the reference prints "Warning! the matrix may not be SPD" and returns
 * its iteration count (src/solver-phg.c:547-571) -- returns the iteration
 * count with x as it is and sets this text. */
const char *phgGpuLastWarning(void);
/* Library version, major * 10000 + minor * 100 + patch. */
int phgGpuVersion(void);

/* Creates a system on CUDA device `device`.  `stream` is a cudaStream_t
 * (NULL: the library creates its own non-blocking stream). */
int phgGpuCreate(int device, void *stream, phgGpuSystem **sys);
int phgGpuDestroy(phgGpuSystem *sys);
/* Re-targets later work to `stream` (cudaStream_t). */
int phgGpuSetStream(phgGpuSystem *sys, void *stream);

/* The mesh: replaces the reference's per-element reads of g->verts and
 * e->verts (phgGeomGetJacobian_, src/geom.c:855-884, computed by
 * compute_jacobian, src/geom.c:103-169, and phgGeomGetVolume, :809). */
int phgGpuSetMesh(phgGpuSystem *sys, int64_t nvert, const double *verts,
		  int64_t nelem, const int32_t *elem_verts);

/* PHG's stored element geometry, used instead of the one computed from the
 * coordinates until the next phgGpuSetMesh: geo[17 * e + 0..15] is the
 * element's Jacobian (phgGeomGetJacobian, src/geom.c:855-884; row c holds
 * the gradient of barycentric c, then its constant term) and geo[17 * e + 16]
 * its volume (phgGeomGetVolume, src/geom.c:809).  On elements PHG made by
 * bisection these are interpolated from the parent (src/geom.c:460-565) and
 * differ from the coordinates' in the last bits; the assembled rows follow
 * PHG's values.  Non-finite values are PHG_GPU_ERR_ARG. */
int phgGpuSetGeometry(phgGpuSystem *sys, int64_t nelem, const double *geo);

/* The DOF layout of a scalar Lagrange P`order` space (order 1, 2 or 3):
 * e2l[e * nbas + k] = vector index of element basis k (phgSolverMapE2L,
 * include/phg/solver.h:297 -> phgDofMapE2D_, src/dof.c:4821-4881), and
 * bdry[i] != 0 for Dirichlet DOFs (phgDofDirichletBC__,
 * src/dof-utils.c:1269-1392).  nbas = 4, 10, 20. */
int phgGpuSetDofMap(phgGpuSystem *sys, int order, int64_t ndof,
		    const int32_t *e2l, const uint8_t *bdry);

/* The batched element loop of a reference user program plus assembly:
 * for every element and basis pair phgQuadGradBasAGradBas (src/quad.c:
 * 5260-5344; kappa == NULL is phgQuadGradBasDotGradBas), per basis
 * phgDofDirichletBC (unit row, rhs = g) or phgQuadDofTimesBas (src/quad.c:
 * 5481-5530), phgMatAddEntries_ (src/matvec.c:5348-5493, exact zeros
 * dropped, rows in first-touch order), phgVecAddEntries_, then
 * phgMatAssemble (src/matvec.c:4602-4671: boundary columns removed from the
 * rows and saved) and phgSolverUpdateRHS (src/solver.c:508-754).
 *   kappa  per-element coefficient (nelem) or NULL
 *   f      f_h DOF values (ndof) or NULL (zero)
 *   g      Dirichlet values at the DOFs (ndof) or NULL (zero)
 * The matrix and RHS stay on the device for the solver calls below. */
int phgGpuBuildLinearSystem(phgGpuSystem *sys, const double *kappa,
			    const double *f, const double *g);

/* The same with a mass term, for -div(kappa grad u) + c u = f: each element
 * matrix is phgQuadGradBasAGradBas + mass_coef * phgQuadBasDotBas
 * (phgQuadBasABas with A = NULL, src/quad.c:5582-5625, order 2p rule), the
 * element loop of examples/simplest.c:66-73 (reaction-diffusion, also the
 * implicit time step of examples/heat.c:155-162 with the roles of the two
 * coefficients exchanged).  mass_coef = 0 is phgGpuBuildLinearSystem.
 * phgGpuAdjointGradient refuses a system with a mass term. */
int phgGpuBuildLinearSystemMass(phgGpuSystem *sys, const double *kappa,
				double mass_coef, const double *f,
				const double *g);

/* The element loop's integrals alone: Ke[e][a][b] (nelem x N x N) is what
 * phgQuadGradBasAGradBas(e, u, b, kappa, u, a, QUAD_DEFAULT) returns (plus
 * mass_coef * phgQuadBasDotBas when mass_coef != 0; src/quad.c:5260-5344,
 * 5582-5625) and Re[e][a] (nelem x N) what phgQuadDofTimesBas(e, f_h, u, a,
 * QUAD_DEFAULT, &r) returns (src/quad.c:5481-5530), bit for bit, for every
 * element at once.  Needs phgGpuSetMesh and phgGpuSetDofMap (the map locates
 * f's values); Ke or Re may be NULL.  Serves per-element shims of those
 * calls (phg_b200/shim). */
int phgGpuElementMatrices(phgGpuSystem *sys, const double *kappa,
			  double mass_coef, const double *f, double *Ke,
			  double *Re);

/* Installs an already-assembled matrix instead (the rows PHG hands an OEM
 * solver, src/solver.c:223-285): CSR with int64 row pointers (PHG's
 * size_t packed_ind), int32 columns, and the right-hand side. */
int phgGpuSetMatrix(phgGpuSystem *sys, int64_t n, const int64_t *ptr,
		    const int32_t *cols, const double *vals, const double *rhs);

/* Rows from recorded row segments, the way phgMatAddEntries_ builds them
 * (src/matvec.c:5348-5493 -> add_columns_to_row :3045-3332): segment r adds
 * the values rec_vals[rec_ptr[r] .. rec_ptr[r + 1]) at columns rec_cols[..]
 * to row rec_row[r] (0 <= row < n), segments applied in their order; exact
 * zeros and negative columns are skipped, a column's first appearance fixes
 * its place in the row, later ones add to it.  The result -- PHG's rows
 * before phgMatAssemble -- becomes the system's matrix (phgGpuGetMatrix
 * returns it; the right-hand side is zero).  rec_ptr is int64 (nrec + 1,
 * rec_ptr[0] = 0).  A row whose first non-empty segment names a column twice
 * (which the reference would keep twice) is PHG_GPU_ERR_ARG; rows longer
 * than 1024 entries are PHG_GPU_ERR_LIMIT.  Serves the per-call shim of
 * phgMatAddEntries_ (phg_b200/shim). */
int phgGpuAssembleRows(phgGpuSystem *sys, int64_t n, int64_t nrec,
		       const int32_t *rec_row, const int64_t *rec_ptr,
		       const int32_t *rec_cols, const double *rec_vals);

/* Replaces the right-hand side the solvers use (n values, boundary
 * elimination already applied) and keeps the matrix: a new phgSolverVecSolve
 * on the same matrix (src/solver.c:1131-1150) or a change of
 * solver->rhs->data before phgSolverSolve.  Non-finite values:
 * PHG_GPU_ERR_NAN. */
int phgGpuSetRHS(phgGpuSystem *sys, const double *rhs);

/* Sizes of the assembled system: rows, matrix entries, saved boundary
 * column entries. */
int phgGpuGetSizes(phgGpuSystem *sys, int64_t *n, int64_t *nnz,
		   int64_t *nnz_bdry);
/* Copies out the matrix rows (phgMatPack layout, src/matvec.c:279-416:
 * row order and in-row order kept), any argument may be NULL. */
int phgGpuGetMatrix(phgGpuSystem *sys, int64_t *ptr, int32_t *cols,
		    double *vals);
/* Copies out the saved boundary columns (MAT.bdry_rows). */
int phgGpuGetBdryColumns(phgGpuSystem *sys, int64_t *ptr, int32_t *cols,
			 double *vals);
/* Copies out the updated right-hand side / the Jacobi diagonal
 * (phgMatSetupDiagonal, src/matvec.c:500-549). */
int phgGpuGetRHS(phgGpuSystem *sys, double *rhs);
int phgGpuGetDiagonal(phgGpuSystem *sys, double *diag);

/* y = A x  (phgMatVec(MAT_OP_N, 1.0, A, x, 0.0, &y), src/matvec.c:552).
 * When x and y are both device pointers the call is asynchronous on the
 * system's stream; otherwise it returns with y written. */
int phgGpuMatVec(phgGpuSystem *sys, const double *x, double *y);

/* Jacobi-preconditioned CG on the assembled system, FP64 throughout
 * (solver_pcg, src/solver-phg.c:485-604; jacobi_pc :207-245; stopping rule
 * ||r|| <= max(rtol ||r0||, btol ||b||, atol), get_tol :104).
 * x: initial guess in, solution out (n).  Returns the iteration count
 * (>= 0) or a negative error code; *residual gets the final ||r||_2.
 * hist (optional, maxit + 1 doubles) receives ||r|| after each
 * iteration, hist[0] = ||r0||.  On a breakdown (the matrix may not be SPD)
 * the iteration stops and the count is returned, as in the reference, with
 * the warning in phgGpuLastWarning(). */
int phgGpuSolverPCG(phgGpuSystem *sys, double rtol, double btol,
		    double atol, int maxit, double *x, double *residual,
		    double *hist);

/* Jacobi-preconditioned BiCGstab, FP64 (solver_BiCGstab,
 * src/solver-phg.c:606-781, what phgSolverSolve runs with -solver bicgstab;
 * same stopping rule and arguments as phgGpuSolverPCG).  For matrices that
 * are not symmetric positive definite (the reference flags it M_UNSYM,
 * :2542-2547), e.g. installed with phgGpuSetMatrix.  Where the reference
 * stops because rho = r.rh is 0 ("method failed", :676-680) the call
 * returns the iteration count as the reference does; a zero rh.v or t.t,
 * where the reference would divide by zero, is PHG_GPU_ERR_BREAKDOWN. */
int phgGpuSolverBiCGstab(phgGpuSystem *sys, double rtol, double btol,
			 double atol, int maxit, double *x, double *residual,
			 double *hist);

/* Restarted right-preconditioned GMRES with the Jacobi preconditioner,
 * FP64 (solver_GMRES_r, src/solver-phg.c:1050-1260: what phgSolverSolve
 * runs with -solver gmres -gmres_type gmres_r -gmres_pc_type jacobi
 * -gmres_restart `restart`; modified Gram-Schmidt, Givens rotations, same
 * stopping rule as phgGpuSolverPCG).  restart in 1..64 (the reference's
 * restart <= 0, "never restart", has no counterpart here).  *residual is
 * the reference's: the rotated residual estimate on convergence, ||r0||
 * when maxit ends the solve.  Returns the iteration count. */
int phgGpuSolverGMRES(phgGpuSystem *sys, int restart, double rtol,
		      double btol, double atol, int maxit, double *x,
		      double *residual);

/* PHG's default GMRES: the flexible, augmented FLGMRES_r
 * (solver_FLGMRES_r, src/solver-phg.c:2063-2340; what phgSolverSolve runs
 * with -solver gmres and the default -gmres_type flgmres_r), Jacobi
 * preconditioner, FP64.  Cycle k takes restart + min(k, augk) steps, the
 * steps past `restart` preconditioning the corrections of the last augk
 * cycles (augk <= 0: 2, the reference's -lgmres_augk default); restart +
 * augk <= 64.  Stopping rule, *residual and return value as
 * phgGpuSolverGMRES. */
int phgGpuSolverFLGMRES(phgGpuSystem *sys, int restart, int augk, double rtol,
			double btol, double atol, int maxit, double *x,
			double *residual);

/* Jacobi-PCG for many right-hand sides at once: column k of B (n x nrhs,
 * row major: B[i * nrhs + k]) is solved by its own PCG recurrence and
 * stopping rule (rtol relative to ||b_k||, from x = 0), and the columns share
 * one SpMM per iteration, so the matrix is read once per tile of columns.
 * mixed = 0: FP64; mixed = 1: FP32 matrix values, vectors and SpMM with FP64
 * reliable updates (as phgGpuSolverPCGMixed).  X (n x nrhs, row major) gets
 * the solutions, nits[k] (optional) the iterations, res[k] (optional)
 * ||b_k - A x_k||_2 in FP64.  At most 64 columns per call.  The SpMM tile
 * width (8/16/32/64 columns, which fixes the rows per warp) is autotuned at
 * the first call for a shape.  Extends the reference (its PCG takes one
 * vector, solver-phg.c:495). */
int phgGpuSolverBlockPCG(phgGpuSystem *sys, int nrhs, const double *B,
			 double *X, double rtol, int maxit, int mixed,
			 int *nits, double *res);
/* The SpMM tile chosen for the last block solve and the measured time of
 * each candidate (8, 16, 32, 64 columns; 0 when not tried). */
int phgGpuGetBlockTile(phgGpuSystem *sys, int *tile, double *times_ms);

/* Adjoint gradient of J = 1/2 ||u - u_obs||_2^2 (sum over all DOFs) with
 * respect to log kappa_e for every element, for the system last built by
 * phgGpuBuildLinearSystem (its kappa): solves A lambda = u - u_obs on the
 * free DOFs (lambda = 0 on Dirichlet DOFs) with the FP64 PCG to relative
 * residual rtol, then grad[e] = -kappa_e lambda_e^T K_e^0 u_e.  u is the
 * solution of that system (n), u_obs the data (n); grad gets nelem values;
 * *J (optional) the functional, *nits (optional) the adjoint iterations.
 * No counterpart in the reference (it has no derivatives). */
int phgGpuAdjointGradient(phgGpuSystem *sys, const double *u,
			  const double *u_obs, double rtol, int maxit,
			  double *grad, double *J, int *nits);

/* Mixed-precision Jacobi-PCG on the assembled system: FP32 matrix values,
 * Krylov vectors and SpMV (products and sums rounded one by one) with
 * FP64-accumulated dot products, in the single-reduction (Chronopoulos-Gear)
 * form of PCG, inside FP64 refinement -- the FP64 solution x is brought up
 * to date and the explicit FP64 residual b - A x recomputed ("reliable
 * updates") whenever the FP32 residual has fallen tenfold, and the search
 * direction is kept across updates, so the iteration converges like the
 * FP64 one.  The stopping rule is the reference's (get_tol,
 * src/solver-phg.c:104, on the initial residual) applied to the FP64
 * residual; on return *residual is ||b - A x||_2 computed in FP64.  Extends
 * the reference (its FLOAT is fixed at build time, configure.in:627-671).
 * Returns the number of FP32 iterations or a negative error code;
 * *nupdates gets the number of reliable updates.  A breakdown stops the
 * iteration as in phgGpuSolverPCG (count returned, phgGpuLastWarning()). */
int phgGpuSolverPCGMixed(phgGpuSystem *sys, double rtol, double btol,
			 double atol, int maxit, double *x, double *residual,
			 int *nupdates);

/* The SpMV layout the autotuner chose for the current matrix (no
 * counterpart in the reference): at the first solve or product for a matrix
 * shape it times CSR with 4/8/16/32 lanes per row and SELL-C-sigma (32-row
 * slices, rows sorted by length in 256-row windows) with 2/4/8-fold
 * unrolling, and keeps the fastest.  kind: 0 = CSR (param = lanes per row),
 * 1 = SELL (param = unroll), 2 = q16 (param = 1; the 16-bit-column layout
 * with FP64 values, a candidate only when every row fits two 65536-column
 * windows); times_ms (optional, 18 doubles) gets the
 * measured time of each candidate in that order, then the times of the FP32
 * products of the mixed solver (SELL unrolled 4/8/16, pair-SELL -- two
 * consecutive entries per lane -- unrolled 2/4/8, q16 -- four entries per
 * lane with 16-bit column offsets from two per-row bases -- unrolled 1/2;
 * 0 for a layout the matrix does not fit), the unroll chosen for it and its
 * layout (0 SELL, 1 pair SELL, 2 q16); 0 before a mixed solve.  Returns the
 * number of FP64 candidates. */
int phgGpuGetSpMVPlan(phgGpuSystem *sys, int *kind, int *param,
		      double *times_ms);

/* Forces the FP32 product layout of the mixed solver for the current matrix
 * instead of the autotuner's choice (no counterpart in the reference):
 * layout 0 = SELL (unroll 4/8/16), 1 = pair SELL (unroll 2/4/8), 2 = q16
 * (unroll 1/2; PHG_GPU_ERR_ARG when a row of the matrix spans more than two
 * 65536-column windows).  A matrix of another shape is tuned again. */
int phgGpuSetSpMVPlan32(phgGpuSystem *sys, int layout, int unroll);

/* Average device time of one SpMV with the chosen layout, FP64 values
 * (fp32 = 0) or the FP32 values of the mixed solver (fp32 = 1), over `reps`
 * back-to-back launches on the system's stream (no counterpart in the
 * reference; used to report the SpMV roofline). */
int phgGpuTimeSpMV(phgGpuSystem *sys, int fp32, int reps, double *ms_per_launch);

/* Bytes one product moves in the layout the solvers use for the current
 * matrix, FP64 (fp32 = 0) or the mixed solver's FP32 product (fp32 = 1):
 * values, column indices, per-row metadata and slice offsets as stored
 * (padding included), x read once and y written once (no counterpart in the
 * reference; the denominator of the layout's bandwidth). */
int phgGpuSpMVBytes(phgGpuSystem *sys, int fp32, int64_t *bytes);

/* Overrides the autotuner for the current matrix shape: kind 0 = CSR with
 * param = 4/8/16/32 lanes per row, kind 1 = SELL with param = 2/4/8, kind 2
 * = q16 with param = 1 (PHG_GPU_ERR_ARG when a row spans more than two
 * 65536-column windows) (no counterpart in the reference). */
int phgGpuSetSpMVPlan(phgGpuSystem *sys, int kind, int param);

/* Number of kernels this system has launched so far (the nodes of captured
 * PCG graphs included): no counterpart in the reference, an aid for
 * profiling. */
int phgGpuGetLaunchCount(phgGpuSystem *sys, int64_t *count);

/* Jacobi-PCG on a CSR matrix in device memory, allocating no memory (no
 * counterpart in the reference; the same iteration as phgGpuSolverPCG).
 * For callers that cannot allocate device memory -- an application whose
 * own pool has reserved the GPU, or a plugin in a process whose device
 * memory another runtime owns.  The working vectors live in a fixed array
 * that is part of the library (about 9 MB held on every GPU that loads the
 * library, until the process exits), which limits n to
 * PHG_GPU_NOALLOC_MAX_ROWS (larger n: PHG_GPU_ERR_LIMIT).  ptr (int64,
 * n + 1), cols, vals, rhs and x (initial guess in, solution out) must be
 * device memory of the current device; work runs on `stream`
 * (cudaStream_t, NULL = default stream) and the call returns when it is
 * done.  Every call looks up the array's address in the current device's
 * context (so a context created again after cudaDeviceReset is served
 * correctly); the first call on a device also loads the library's device
 * code, so make that first call before any stream capture.  All calls share
 * the one array, so calls that overlap on the GPU (other host threads, other
 * streams) race: serialise them.  Returns the iteration count or a negative
 * error code; a breakdown is reported as in phgGpuSolverPCG. */
#define PHG_GPU_NOALLOC_MAX_ROWS 262144
int phgGpuSolverPCGNoAlloc(int64_t n, const int64_t *ptr, const int32_t *cols,
			   const double *vals, const double *rhs, double *x,
			   double rtol, double btol, double atol, int maxit,
			   void *stream, double *residual);

#ifdef __cplusplus
}
#endif
#endif /* PHG_GPU_H */
