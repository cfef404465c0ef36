/*
 * Test-infrastructure driver around the UNMODIFIED reference library (PHG),
 * compiled from its own sources into oracle/_ref by oracle/Makefile.
 *
 * It runs the reference's element-assembly + Jacobi-PCG path on a Medit mesh
 * exactly the way PHG user programs do it (examples/poisson.c:101-170 shows
 * the pattern: per element, phgQuadGradBasDotGradBas / phgQuadGradBasAGradBas
 * for every basis pair, phgDofDirichletBC or phgQuadDofTimesBas per basis,
 * phgSolverAddMatrixEntries / phgSolverAddRHSEntries per element), then
 * phgSolverAssemble, phgSolverUpdateRHS and phgSolverSolve with "-solver pcg".
 *
 * Two uses:
 *   1. parity fixtures: with -dump_dir it writes the reference's own inputs
 *      (coordinates, element->vertex and element->DOF maps as PHG numbered
 *      them, f and g at the DOF nodes, Dirichlet flags) and outputs (matrix rows
 *      before and after boundary elimination, RHS, Jacobi diagonal, solution)
 *      as raw little-endian binaries;
 *   2. the CPU baseline: it prints one JSON line with the stage timings
 *      (element loop, phgSolverAssemble, phgSolverSolve) measured with
 *      phgGetTime, as examples/poisson.c:436-550 does.
 *
 * It is never linked into, loaded by, or executed from the product library.
 */
#include "phg.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <sys/stat.h>

static char *mesh_file = NULL;
static char *dump_dir = NULL;
static char *kappa_file = NULL;
static INT rhs_case = 0;		/* 0: sine (g = 0), 1: linear u=x+y+z */
static INT repeat = 1;			/* repeat the whole pipeline (timing) */
static INT sample_maxit = 0;		/* > 0: cap PCG iterations after rep 0 */
static FLOAT mass_coef = 0.;		/* != 0: add mass_coef * mass matrix */
static INT refine = 0;			/* uniform bisection levels after import */
static INT refine_corner = 0;		/* local refinement rounds at (0,0,0) */
static const char *rhs_case_names[] = {"sine", "linear", NULL};

#if PHG_GPU_PLUGIN
/* the GPU OEM solvers (phg_b200/shim/phg_gpu_solver.c), chosen with
 * -gpu_solver and passed to phgSolverCreate instead of SOLVER_DEFAULT */
extern OEM_SOLVER phgSolverGpuPCG_, phgSolverGpuPCGMixed_,
		  phgSolverGpuBiCGstab_, phgSolverGpuGMRES_;
static INT gpu_solver = 0;
static const char *gpu_solver_names[] =
	{"none", "pcg", "pcg_mixed", "bicgstab", "gmres", NULL};
static OEM_SOLVER *gpu_solvers[] = {NULL, &phgSolverGpuPCG_,
	&phgSolverGpuPCGMixed_, &phgSolverGpuBiCGstab_, &phgSolverGpuGMRES_};
#define OEM_CHOICE	gpu_solvers[gpu_solver]
#else
#define OEM_CHOICE	SOLVER_DEFAULT
#endif

static void
func_f(FLOAT x, FLOAT y, FLOAT z, FLOAT *value)
{
    if (rhs_case == 0)
	*value = 3. * M_PI * M_PI * sin(M_PI * x) * sin(M_PI * y) *
		 sin(M_PI * z);
    else
	*value = 0.;
}

static void
func_g(FLOAT x, FLOAT y, FLOAT z, FLOAT *value)
{
    if (rhs_case == 0)
	*value = 0.;
    else
	*value = x + y + z;
}

static void
write_bin(const char *name, const void *data, size_t size, size_t count)
{
    char path[4096];
    FILE *fp;

    snprintf(path, sizeof(path), "%s/%s", dump_dir, name);
    if ((fp = fopen(path, "wb")) == NULL)
	phgError(1, "cannot write %s\n", path);
    if (count > 0 && fwrite(data, size, count, fp) != count)
	phgError(1, "short write on %s\n", path);
    fclose(fp);
}

/* writes a row list (MAT_ROW[n]) as ptr (int64[n+1]), cols, vals */
static void
dump_rows(const char *prefix, const MAT_ROW *rows, INT n)
{
    char name[256];
    long long *ptr = malloc((n + 1) * sizeof(*ptr));
    size_t nnz = 0, k = 0;
    INT i, *cols;
    FLOAT *vals;

    for (i = 0; i < n; i++)
	nnz += rows[i].ncols;
    cols = malloc((nnz + 1) * sizeof(*cols));
    vals = malloc((nnz + 1) * sizeof(*vals));
    ptr[0] = 0;
    for (i = 0; i < n; i++) {
	memcpy(cols + k, rows[i].cols, rows[i].ncols * sizeof(*cols));
	memcpy(vals + k, rows[i].data, rows[i].ncols * sizeof(*vals));
	k += rows[i].ncols;
	ptr[i + 1] = (long long)k;
    }
    snprintf(name, sizeof(name), "%s_ptr.i64", prefix);
    write_bin(name, ptr, sizeof(*ptr), n + 1);
    snprintf(name, sizeof(name), "%s_cols.i32", prefix);
    write_bin(name, cols, sizeof(*cols), nnz);
    snprintf(name, sizeof(name), "%s_vals.f64", prefix);
    write_bin(name, vals, sizeof(*vals), nnz);
    free(ptr);
    free(cols);
    free(vals);
}

int
main(int argc, char *argv[])
{
    GRID *g;
    ELEMENT *e;
    DOF *u_h, *f_h, *kappa = NULL;
    SOLVER *solver;
    INT ndof, nbas, i, rep;
    double t0, t_build = 0., t_asm = 0., t_solve = 0.;
    BOOLEAN dump;
    INT *e2l = NULL, *elems = NULL, *order = NULL;
    FLOAT *gvals = NULL;
    unsigned char *bdry = NULL;

    phgOptionsRegisterFilename("-mesh_file", "Mesh file", &mesh_file);
    phgOptionsRegisterFilename("-dump_dir", "Dump directory", &dump_dir);
    phgOptionsRegisterFilename("-kappa_file",
		"Per-element coefficient (float64, by element index)",
		&kappa_file);
    phgOptionsRegisterKeyword("-rhs_case", "Right-hand side / BC case",
		rhs_case_names, &rhs_case);
    phgOptionsRegisterInt("-repeat", "Repeat the pipeline (timing)", &repeat);
    phgOptionsRegisterFloat("-mass_coef",
		"Coefficient c of the mass term (-div kappa grad u + c u = f)",
		&mass_coef);
    phgOptionsRegisterInt("-refine", "Uniform refinement levels (phgRefineAllElements)",
		&refine);
    phgOptionsRegisterInt("-refine_corner",
		"Rounds of local refinement of the elements near (0,0,0)",
		&refine_corner);
    phgOptionsRegisterInt("-sample_maxit",
		"PCG iteration cap for repetitions after the first (timing samples)",
		&sample_maxit);

#if PHG_GPU_PLUGIN
    phgOptionsRegisterKeyword("-gpu_solver", "GPU OEM solver (none: PHG's own)",
		gpu_solver_names, &gpu_solver);
#endif

    phgInit(&argc, &argv);
    if (mesh_file == NULL)
	phgError(1, "-mesh_file is required\n");
    dump = (dump_dir != NULL && dump_dir[0] != '\0');

    g = phgNewGrid(-1);
    if (!phgImport(g, mesh_file, FALSE))
	phgError(1, "can't read file \"%s\".\n", mesh_file);
    /* meshes PHG refines itself: uniform bisection, then local bisection of
     * the elements whose centroid lies within 0.25 of the corner (0,0,0)
     * (the marking pattern of examples/eigen.c:398-411) */
    if (refine > 0)
	phgRefineAllElements(g, refine);
    for (i = 0; i < refine_corner; i++) {
	ForAllElements(g, e) {
	    FLOAT c[3] = {0., 0., 0.};
	    int k;
	    for (k = 0; k < NVert; k++) {
		c[0] += g->verts[e->verts[k]][0] * 0.25;
		c[1] += g->verts[e->verts[k]][1] * 0.25;
		c[2] += g->verts[e->verts[k]][2] * 0.25;
	    }
	    e->mark = (c[0] * c[0] + c[1] * c[1] + c[2] * c[2] < 0.0625) ? 1 : 0;
	}
	phgRefineMarkedElements(g);
    }

    u_h = phgDofNew(g, DOF_DEFAULT, 1, "u_h", DofNoAction);
    phgDofSetDataByValue(u_h, 0.0);
    u_h->DB_mask = BDRY_MASK;
    f_h = phgDofNew(g, DOF_DEFAULT, 1, "f_h", func_f);
    if (kappa_file != NULL && kappa_file[0] != '\0') {
	FILE *fp = fopen(kappa_file, "rb");
	if (fp == NULL)
	    phgError(1, "can't open \"%s\"\n", kappa_file);
	kappa = phgDofNew(g, DOF_P0, 1, "kappa", DofNoAction);
	if (fread(kappa->data, sizeof(FLOAT), g->nelem, fp) != (size_t)g->nelem)
	    phgError(1, "short kappa file \"%s\"\n", kappa_file);
	fclose(fp);
    }

    ndof = DofDataCount(u_h);
    nbas = u_h->type->nbas;

    for (rep = 0; rep < repeat; rep++) {
	BOOLEAN last = (rep == repeat - 1);
	phgDofSetDataByValue(u_h, 0.0);
	solver = phgSolverCreate(OEM_CHOICE, u_h, NULL);
	if (rep > 0 && sample_maxit > 0) {
	    solver->maxit = sample_maxit;
	    solver->warn_maxit = FALSE;
	}

	if (dump && last) {
	    e2l = phgAlloc(g->nelem * nbas * sizeof(*e2l));
	    elems = phgAlloc(g->nelem * NVert * sizeof(*elems));
	    order = phgAlloc(g->nelem * sizeof(*order));
	    gvals = phgCalloc(ndof, sizeof(*gvals));
	    bdry = phgCalloc(ndof, sizeof(*bdry));
	}

	t0 = phgGetTime(NULL);
	i = 0;
	/* the OpenMP build runs the element loop on all threads, as
	 * examples/poisson.c:116-119 does (serial when dumping fixtures, so
	 * the element order of the dumps is the grid's) */
#if USE_OMP
#pragma omp parallel for private(e) if (!(dump && last))
#endif
	ForAllElementsBegin(g, e) {
	    int a, b, N = DofNBas(u_h, e);
	    FLOAT A[N][N], B[N], buffer[N], *row;
	    INT I[N];

	    for (a = 0; a < N; a++) {
		I[a] = phgSolverMapE2L(solver, 0, e, a);
		for (b = 0; b <= a; b++) {
		    if (kappa == NULL)
			A[a][b] = phgQuadGradBasDotGradBas(e, u_h, b, u_h, a,
							   QUAD_DEFAULT);
		    else
			A[a][b] = phgQuadGradBasAGradBas(e, u_h, b, kappa,
							 u_h, a, QUAD_DEFAULT);
		    /* stiffness + c * mass, as examples/simplest.c:68-72 */
		    if (mass_coef != 0.)
			A[a][b] = A[a][b] + mass_coef *
			    phgQuadBasDotBas(e, u_h, b, u_h, a, QUAD_DEFAULT);
		    A[b][a] = A[a][b];
		}
	    }
	    for (a = 0; a < N; a++) {
		if (phgDofDirichletBC(u_h, e, a, func_g, buffer, B + a,
				      DOF_PROJ_NONE)) {
		    row = buffer;
		    if (bdry != NULL) {
			bdry[I[a]] = 1;
			gvals[I[a]] = B[a];
		    }
		}
		else {
		    phgQuadDofTimesBas(e, f_h, u_h, a, QUAD_DEFAULT, B + a);
		    row = A[a];
		}
		phgSolverAddMatrixEntries(solver, 1, I + a, N, I, row);
	    }
	    phgSolverAddRHSEntries(solver, N, I, B);

	    if (e2l != NULL) {
		for (a = 0; a < N; a++)
		    e2l[e->index * nbas + a] = I[a];
		for (a = 0; a < NVert; a++)
		    elems[e->index * NVert + a] = e->verts[a];
		order[i] = e->index;
		i++;
	    }
	} ForAllElementsEnd
	t_build = phgGetTime(NULL) - t0;

	if (dump && last) {
	    dump_rows("rows_raw", solver->mat->rows, solver->mat->rmap->nlocal);
	    write_bin("rhs_raw.f64", solver->rhs->data, sizeof(FLOAT), ndof);
	}

	t0 = phgGetTime(NULL);
	phgSolverAssemble(solver);
	phgSolverUpdateRHS(solver);
	t_asm = phgGetTime(NULL) - t0;

	if (dump && last) {
	    dump_rows("rows", solver->mat->rows, solver->mat->rmap->nlocal);
	    dump_rows("bdry_rows", solver->mat->bdry_rows,
		      solver->mat->rmap->nlocal);
	    write_bin("rhs.f64", solver->rhs->data, sizeof(FLOAT), ndof);
	}

	t0 = phgGetTime(NULL);
	phgSolverSolve(solver, FALSE, u_h, NULL);
	t_solve = phgGetTime(NULL) - t0;

	if (dump && last) {
	    FILE *fp;
	    char path[4096];
	    write_bin("x.f64", u_h->data, sizeof(FLOAT), ndof);
	    if (solver->mat->diag == NULL)	/* a solver without Jacobi setup */
		phgMatSetupDiagonal(solver->mat);
	    write_bin("diag.f64", solver->mat->diag, sizeof(FLOAT), ndof);
	    write_bin("verts.f64", g->verts, sizeof(FLOAT), 3 * g->nvert);
	    write_bin("elems.i32", elems, sizeof(INT), NVert * g->nelem);
	    {	/* PHG's element geometry (J, 16 values, then the volume):
		 * on refined meshes it is interpolated from the parents
		 * (geom.c:460-565), not computed from the coordinates */
		FLOAT *geo = phgAlloc(17 * (size_t)g->nelem * sizeof(*geo));
		ForAllElements(g, e) {
		    memcpy(geo + 17 * (size_t)e->index, phgGeomGetJacobian(g, e),
			   16 * sizeof(FLOAT));
		    geo[17 * (size_t)e->index + 16] = phgGeomGetVolume(g, e);
		}
		write_bin("geom.f64", geo, sizeof(FLOAT), 17 * (size_t)g->nelem);
		phgFree(geo);
	    }
	    write_bin("e2l.i32", e2l, sizeof(INT), nbas * g->nelem);
	    write_bin("order.i32", order, sizeof(INT), g->nelem);
	    write_bin("f.f64", f_h->data, sizeof(FLOAT), ndof);
	    write_bin("g.f64", gvals, sizeof(FLOAT), ndof);
	    write_bin("bdry.u8", bdry, 1, ndof);
	    if (kappa != NULL)
		write_bin("kappa.f64", kappa->data, sizeof(FLOAT), g->nelem);
	    snprintf(path, sizeof(path), "%s/meta.txt", dump_dir);
	    fp = fopen(path, "w");
	    fprintf(fp, "nvert %d\nnelem %d\nndof %d\nnbas %d\norder %d\n"
			"nits %d\nresidual %.17g\nrtol %.17g\nbtol %.17g\n"
			"atol %.17g\nnedge %d\nnface %d\nmass_coef %.17g\n",
		    (int)g->nvert, (int)g->nelem, (int)ndof, (int)nbas,
		    (int)u_h->type->order, solver->nits,
		    (double)solver->residual, (double)solver->rtol,
		    (double)solver->btol, (double)solver->atol,
		    (int)g->nedge, (int)g->nface, (double)mass_coef);
	    fclose(fp);
	    phgFree(e2l);
	    phgFree(elems);
	    phgFree(order);
	    phgFree(gvals);
	    phgFree(bdry);
	    e2l = elems = order = NULL;
	    gvals = NULL;
	    bdry = NULL;
	}

	printf("{\"rep\": %d, \"nelem\": %d, \"ndof\": %d, \"nbas\": %d, "
	       "\"nits\": %d, \"residual\": %.6e, \"t_build\": %.6f, "
	       "\"t_assemble\": %.6f, \"t_solve\": %.6f, \"threads\": %d}\n",
	       (int)rep, (int)g->nelem, (int)ndof, (int)nbas, solver->nits,
	       (double)solver->residual, t_build, t_asm, t_solve,
	       phgMaxThreads);
	fflush(stdout);
	phgSolverDestroy(&solver);
    }

    phgDofFree(&u_h);
    phgDofFree(&f_h);
    if (kappa != NULL)
	phgDofFree(&kappa);
    phgFreeGrid(&g);
    phgFinalize();
    return 0;
}
