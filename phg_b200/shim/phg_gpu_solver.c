/*
 * PHG linear solvers on the GPU, as OEM_SOLVER instances
 * (include/phg/solver.h:60-90) that a PHG program passes to
 * phgSolverCreate:
 *
 *   solver = phgSolverCreate(&phgSolverGpuPCG_, u_h, NULL);
 *
 * PHG accepts any OEM_SOLVER pointer (src/solver.c:847-895), so its own
 * solver list needs no edit.  Like PHG's built-in Krylov solvers
 * (src/solver-phg.c:2535-2560) these keep PHG's assembled matrix instead of
 * taking rows one by one (AddMatrixEntries NULL): Solve packs it
 * (phgMatPack, src/matvec.c:279-416), hands the CSR and the updated
 * right-hand side to the GPU once, and solves there.  A later Solve on the
 * same solver (a new right-hand side, src/solver.c:1131-1150) sends only the
 * right-hand side.
 *
 *   phgSolverGpuPCG_       Jacobi-PCG, FP64       (-solver pcg: solver_pcg)
 *   phgSolverGpuPCGMixed_  Jacobi-PCG, FP32 inner iteration with FP64
 *                          reliable updates, the same FP64 stopping rule
 *   phgSolverGpuBiCGstab_  Jacobi-BiCGstab, FP64  (-solver bicgstab)
 *   phgSolverGpuGMRES_     restarted Jacobi-GMRES, FP64: PHG's -gmres_type
 *                          (its default flgmres_r, or gmres_r), restart from
 *                          -gmres_restart, augmentation from -lgmres_augk
 *
 * Tolerances, maxit and the initial guess are PHG's (solver->rtol, btol,
 * atol, maxit, x).  A PCG breakdown prints the reference's warning once and
 * returns the iteration count (solver-phg.c:547-571); other failures print
 * the library's message and return -1, which phgSolverVecSolve turns into
 * phgError as it does for every OEM solver.  Serial PHG only (one process,
 * one GPU: device 0, or $PHG_GPU_DEVICE).
 */
#include "phg.h"
#include "phg_gpu.h"

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { GPU_PCG = 0, GPU_PCG_MIXED = 1, GPU_BICGSTAB = 2, GPU_GMRES = 3 };

typedef struct {
    phgGpuSystem *sys;
    int kind;
    int matrix_sent;	/* the GPU holds this solver's matrix */
    BOOLEAN warned;	/* the breakdown warning was printed */
} GPU_DATA;

#define _g ((GPU_DATA *)solver->oem_data)

static INT gmres_restart = 10;	/* PHG's default (-gmres_restart) */
static INT lgmres_augk = 2;	/* PHG's default (-lgmres_augk) */
static int gmres_flexible = 1;	/* PHG's default -gmres_type is flgmres_r */

static int
Init(SOLVER *solver)
{
    GPU_DATA *d = phgCalloc(1, sizeof(*d));
    const char *dev = getenv("PHG_GPU_DEVICE");

    solver->oem_data = d;
    if (phgGpuCreate(dev == NULL ? 0 : atoi(dev), NULL, &d->sys) != PHG_GPU_OK)
	phgError(1, "%s: %s\n", solver->oem_solver->name, phgGpuLastError());
    return 0;
}

static int
Destroy(SOLVER *solver)
{
    if (solver->oem_data == NULL)
	return 0;
    phgGpuDestroy(_g->sys);
    phgFree(solver->oem_data);
    solver->oem_data = NULL;
    return 0;
}

/* Sends the packed matrix (first call) or the right-hand side (later
 * calls) to the GPU. */
static int
send(SOLVER *solver)
{
    MAT *A = solver->mat;
    int rc;

    if (!_g->matrix_sent) {
	assert(A != NULL && A->type != PHG_DESTROYED);
	phgMatPack(A);
	rc = phgGpuSetMatrix(_g->sys, A->rmap->nlocal,
			     (const int64_t *)A->packed_ind, A->packed_cols,
			     A->packed_data, solver->rhs->data);
	_g->matrix_sent = (rc == PHG_GPU_OK);
    }
    else {
	rc = phgGpuSetRHS(_g->sys, solver->rhs->data);
    }
    if (rc != PHG_GPU_OK)
	phgWarning("%s: %s\n", solver->oem_solver->name, phgGpuLastError());
    return rc;
}

static int
Solve(SOLVER *solver, VEC *x, BOOLEAN destroy)
{
    double res = 0.0;
    int nits, nupd = 0;
    const char *w;

    assert(solver->rhs->assembled && x->map->nlocal == solver->rhs->map->nlocal);
    if (send(solver) != PHG_GPU_OK)
	return -1;

    switch (_g->kind) {
	case GPU_PCG:
	    nits = phgGpuSolverPCG(_g->sys, solver->rtol, solver->btol,
				   solver->atol, solver->maxit, x->data, &res,
				   NULL);
	    break;
	case GPU_PCG_MIXED:
	    nits = phgGpuSolverPCGMixed(_g->sys, solver->rtol, solver->btol,
					solver->atol, solver->maxit, x->data,
					&res, &nupd);
	    break;
	case GPU_BICGSTAB:
	    nits = phgGpuSolverBiCGstab(_g->sys, solver->rtol, solver->btol,
					solver->atol, solver->maxit, x->data,
					&res, NULL);
	    break;
	default:
	    if (gmres_flexible)
		nits = phgGpuSolverFLGMRES(_g->sys, gmres_restart, lgmres_augk,
					   solver->rtol, solver->btol,
					   solver->atol, solver->maxit, x->data,
					   &res);
	    else
		nits = phgGpuSolverGMRES(_g->sys, gmres_restart, solver->rtol,
					 solver->btol, solver->atol,
					 solver->maxit, x->data, &res);
	    break;
    }
    if (nits < 0) {
	phgWarning("%s: %s\n", solver->oem_solver->name, phgGpuLastError());
	return -1;
    }
    w = phgGpuLastWarning();
    if (w[0] != '\0' && !_g->warned) {
	/* the reference's wording (solver-phg.c:551-553) */
	phgPrintf("%s: Warning! the matrix may not be SPD. (%s)\n",
		  solver->oem_solver->name, w);
	_g->warned = TRUE;
    }
    if (solver->monitor)
	phgPrintf("%s: %d iterations, residual %le%s\n",
		  solver->oem_solver->name, nits, res,
		  _g->kind == GPU_PCG_MIXED ? " (FP64)" : "");
    if (destroy) {
	/* the GPU keeps its copy; PHG's may go (as PCG_Solve does) */
	phgMatDestroy(&solver->mat);
	solver->sent_to_oem = TRUE;
    }
    solver->residual = (FLOAT)res;
    return solver->nits = nits;
}

#define DEFINE_INIT(name, k) \
    static int name(SOLVER *solver) { Init(solver); _g->kind = k; return 0; }
DEFINE_INIT(InitPCG, GPU_PCG)
DEFINE_INIT(InitPCGMixed, GPU_PCG_MIXED)
DEFINE_INIT(InitBiCGstab, GPU_BICGSTAB)

static int
InitGMRES(SOLVER *solver)
{
    INT r;
    const char *type;

    Init(solver);
    _g->kind = GPU_GMRES;
    /* PHG's own GMRES options (registered by its GMRES, solver-phg.c:454-470) */
    r = phgOptionsGetInt("-gmres_restart");
    if (r > 0)
	gmres_restart = r;
    r = phgOptionsGetInt("-lgmres_augk");
    lgmres_augk = r > 0 ? r : 2;
    type = phgOptionsGetKeyword("-gmres_type");
    if (type != NULL && strcmp(type, "flgmres_r") != 0 && strcmp(type, "gmres_r") != 0)
	phgError(1, "%s: -gmres_type %s has no GPU counterpart (flgmres_r, gmres_r)\n",
		 solver->oem_solver->name, type);
    gmres_flexible = (type == NULL || strcmp(type, "flgmres_r") == 0);
    return 0;
}

/* called once before the first Solve (send_matrix_to_oem_solver,
 * src/solver.c:236): nothing to set up, the matrix goes over in Solve */
static int
Create(SOLVER *solver)
{
    Unused(solver);
    return 0;
}

/* Fields in the order of include/phg/solver.h:60-90. */
#define GPU_OEM(label, init, sym) { \
    label, NULL /* RegisterOptions */, NULL /* Initialize */, \
    NULL /* Finalize */, init, Create, Destroy, \
    NULL /* AddMatrixEntries: PHG keeps its rows */, \
    NULL /* AddRHSEntries */, NULL /* Assemble */, NULL /* SetPC */, Solve, \
    NULL, NULL, NULL /* GetSolver, GetMatrix, GetPC */, \
    sym, TRUE /* iterative */, FALSE /* parallel */, \
    FALSE /* allow_matrix_free */, FALSE /* allow_extern_pc */ }

OEM_SOLVER phgSolverGpuPCG_ = GPU_OEM("GPU-PCG", InitPCG, M_SPD);
OEM_SOLVER phgSolverGpuPCGMixed_ = GPU_OEM("GPU-PCG-mixed", InitPCGMixed, M_SPD);
OEM_SOLVER phgSolverGpuBiCGstab_ = GPU_OEM("GPU-BiCGstab", InitBiCGstab, M_UNSYM);
OEM_SOLVER phgSolverGpuGMRES_ = GPU_OEM("GPU-GMRES", InitGMRES, M_UNSYM);
