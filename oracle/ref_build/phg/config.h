/* Build-configuration header for compiling the unmodified PHG sources of the
 * element-assembly + PCG path into a serial, MPI-free test oracle.
 *
 * PHG normally generates this header with its autoconf script; here the
 * values are written by hand for one fixed configuration: serial (no MPI),
 * FLOAT = double, INT = int, no external solvers or graphics, no debug
 * checks.  An OpenMP flavour of the same build is selected with -DORACLE_OMP=1.
 * Test infrastructure only: nothing in the product links against it. */
#ifndef PHG_CONFIG_H
#define PHG_CONFIG_H

#define HAVE_FCLOSEALL		0
#define HAVE_REGEX_H		0
#define HAVE_EXECINFO_H		0
#define USE_ANONYMOUS_UNION	1
#define USE_QUAD_CUBOID		0
#define USE_HB_FOR_DG		0
#define USE_MPI			0
#define USE_MPIIO		0
#ifdef ORACLE_OMP
#define USE_OMP			ORACLE_OMP
#else
#define USE_OMP			0
#endif
#define USE_PAPI		0
#define USE_TCL			0
#define USE_TK			0
#define USE_METIS		0
#define USE_ZOLTAN		0
#define USE_PARMETIS		0
#define USE_VTK			0
#define DEBUG			0
#define ALLOW_CURVED_BOUNDARY	1
#define PHG_BIGENDIAN		0
#define GRID_TYPE_TET		0
#define GRID_TYPE_HEX		1
#define GRID_TYPE_MIX		2
#define PHG_GRID_TYPE		GRID_TYPE_TET

#define USE_HYPRE		0
#define HYPRE_VERSION_MAJOR	0
#define HYPRE_VERSION_MINOR	0
#define USE_PETSC		0
#define USE_TRILINOS		0
#define HAVE_TRILINOS_VERSION_H	0
#define USE_SUPERLU		0
#define USE_SUPERLU_PARSYMBFACT	0
#define SUPERLU_VERSION_MAJOR	3
#define USE_PASTIX		0
#define USE_HIPS		0
#define USE_MUMPS		0
#define USE_SPOOLES		0
#define USE_PARDISO		0
#define USE_SSPARSE		0
#define USE_LASPACK		0
#define USE_HSPARSE		0
#define USE_MINRES		0
#define USE_X9AMG		0
#define USE_OSKI		0

#define USE_ARPACK		0
#define USE_JDBSYM		0
#define USE_JDBSYM_PARALLEL	0
#define USE_BLOPEX		0
#define USE_SLEPC		0
#define USE_PRIMME		0
#define USE_GWLOBPCG		0
#define USE_TRILINOS_ANASAZI	0

#define F77_FUNC(s,S)	s ## _
#define F77_FUNC_(s,S)	s ## __
#define FC_FUNC(s,S)	s ## _
#define FC_FUNC_(s,S)	s ## __
#define USE_BLAS		0
#define USE_LAPACK		0
#define BLAS_INT		int
#define SIZEOF_BLAS_INT		4
#define LAPACK_INT		BLAS_INT
#define SIZEOF_LAPACK_INT	SIZEOF_BLAS_INT
#define USE_SCALAPACK		0

/* INT = int */
#define dFMT			"d"
#define IT_PHG			IT_INT
#define SIZEOF_SHORT		2
#define SIZEOF_INT		4
#define SIZEOF_LONG		8
#define SIZEOF_LONG_LONG	8
#define TYPEOF_PHG_INT		int
#define SIZEOF_PHG_INT		4

/* FLOAT = double */
#define FT_PHG			FT_DOUBLE
#define SIZEOF_DOUBLE		8
#define SIZEOF_FLOAT		4
#define SIZEOF_LONG_DOUBLE	16
#define SIZEOF___FLOAT128	16
#define HAVE_LIBQUADMATH	0
#define HAVE_QUADMATH_H		0
#define HAVE_Q_SUFFIX		0
#define TYPEOF_PHG_FLOAT	double
#define SIZEOF_PHG_FLOAT	8
#define HAVE_FEENABLEEXCEPT	1
#define HAVE_LIBMATHEVAL	0
#define HAVE_LIBGMP		0
#define HAVE_LIBMPFR		0
#define HAVE_PSAPI		0
#define HAVE_P4EST		0

#define NO_NEW_COMMUNICATOR	0
#define SENDRECV_TEST		0
#define ALLTOALLV_HACK		0
#define REALLOC_HACK		0
#define OMP_ALLOC_HACK		0

#if !defined(assert) && !defined(NDEBUG)
#include <assert.h>
#define NDEBUG
#endif

#define NO_DIST			1
#endif  /* !defined(PHG_CONFIG_H) */
