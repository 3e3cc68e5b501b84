/*
 * Single-rank stand-in for the subset of PETSc 3.7.3 that the reference
 * (PIGFEM 4.6.1) calls.  It exists only so the reference's own sources can be
 * compiled here and run serially as the CPU oracle that pins this project's
 * restatement.  Test infrastructure: nothing in the product links it.
 *
 * What it models:
 *   - Vec: a dense double array (sequential; "MPI" vectors are the same).
 *   - Mat (AIJ): per-row sorted (column, value) arrays with insertion, i.e.
 *     the same per-entry binary search MatSetValue does in PETSc's SeqAIJ.
 *   - Mat (dense): column-major array.
 *   - KSP: every solve is a direct sparse Cholesky (LDL^T) of the operator in
 *     reverse Cuthill-McKee order, standing in for PCCHOLESKY + MUMPS; the
 *     preconditioner/Krylov choice is recorded and ignored.
 *   - SNES: Newton with a backtracking (quadratic/cubic) line search and the
 *     PETSc default tests atol=1e-50, rtol=1e-8, stol=1e-8, maxit=50,
 *     standing in for SNESNEWTONLS.
 */
#ifndef PG_REF_SHIM_PETSC_H
#define PG_REF_SHIM_PETSC_H

#include <stddef.h>
#include <stdio.h>
#include "mpi.h"

typedef int PetscErrorCode;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef enum { PETSC_COPY_VALUES, PETSC_OWN_POINTER, PETSC_USE_POINTER } PetscCopyMode;

#define PETSC_NULL NULL
#define PETSC_DEFAULT (-2)
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE (-1)
#define PETSC_COMM_WORLD MPI_COMM_WORLD
#define PETSC_COMM_SELF MPI_COMM_SELF

#define CHKERRQ(ierr) do { if (ierr) return (ierr); } while (0)
#define CHKERRV(ierr) do { if (ierr) return; } while (0)
#define CHKERRABORT(comm, ierr) do { if (ierr) { fprintf(stderr, "shim error %d\n", (int)(ierr)); abort(); } } while (0)

typedef enum { NOT_SET_VALUES, INSERT_VALUES, ADD_VALUES, MAX_VALUES } InsertMode;
typedef enum { SCATTER_FORWARD = 0, SCATTER_REVERSE = 1 } ScatterMode;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_FROBENIUS = 2, NORM_INFINITY = 3 } NormType;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum {
    MAT_NEW_NONZERO_LOCATIONS, MAT_NEW_NONZERO_LOCATION_ERR, MAT_NEW_NONZERO_ALLOCATION_ERR,
    MAT_SYMMETRIC, MAT_SPD, MAT_STRUCTURALLY_SYMMETRIC, MAT_IGNORE_OFF_PROC_ENTRIES,
    MAT_KEEP_NONZERO_PATTERN, MAT_HERMITIAN, MAT_SYMMETRY_ETERNAL
} MatOption;
typedef enum { MAT_FACTOR_NONE, MAT_FACTOR_LU, MAT_FACTOR_CHOLESKY, MAT_FACTOR_ILU, MAT_FACTOR_ICC } MatFactorType;
typedef enum { KSP_CG_SYMMETRIC = 0, KSP_CG_HERMITIAN = 1 } KSPCGType;
typedef enum {
    SNES_CONVERGED_FNORM_ABS = 2, SNES_CONVERGED_FNORM_RELATIVE = 3, SNES_CONVERGED_SNORM_RELATIVE = 4,
    SNES_CONVERGED_ITS = 5, SNES_CONVERGED_TR_DELTA = 7,
    SNES_DIVERGED_FUNCTION_DOMAIN = -1, SNES_DIVERGED_FUNCTION_COUNT = -2, SNES_DIVERGED_LINEAR_SOLVE = -3,
    SNES_DIVERGED_FNORM_NAN = -4, SNES_DIVERGED_MAX_IT = -5, SNES_DIVERGED_LINE_SEARCH = -6,
    SNES_DIVERGED_INNER = -7, SNES_DIVERGED_LOCAL_MIN = -8, SNES_CONVERGED_ITERATING = 0
} SNESConvergedReason;

typedef const char* MatType;
typedef const char* KSPType;
typedef const char* PCType;
typedef const char* SNESType;
typedef const char* MatSolverPackage;
typedef const char* MatOrderingType;

#define MATAIJ "aij"
#define MATSEQAIJ "seqaij"
#define MATMPIAIJ "mpiaij"
#define MATDENSE "dense"
#define MATSEQDENSE "seqdense"
#define KSPPREONLY "preonly"
#define KSPCG "cg"
#define KSPGMRES "gmres"
#define PCCHOLESKY "cholesky"
#define PCLU "lu"
#define PCJACOBI "jacobi"
#define PCSOR "sor"
#define PCGAMG "gamg"
#define PCHYPRE "hypre"
#define PCNONE "none"
#define SNESNEWTONLS "newtonls"
#define SNESNEWTONTR "newtontr"
#define MATSOLVERMUMPS "mumps"
#define MATSOLVERSUPERLU_DIST "superlu_dist"
#define MATSOLVERPETSC "petsc"
#define MATORDERINGND "nd"
#define MATORDERINGNATURAL "natural"
#define MATORDERINGRCM "rcm"

typedef struct _p_Vec* Vec;
typedef struct _p_Mat* Mat;
typedef struct _p_KSP* KSP;
typedef struct _p_PC* PC;
typedef struct _p_SNES* SNES;
typedef struct _p_IS* IS;
typedef struct _p_VecScatter* VecScatter;
typedef struct { double fill; double levels; double shiftamount; } MatFactorInfo;

#ifdef __cplusplus
extern "C" {
#endif

PetscErrorCode PetscInitialize(int* argc, char*** argv, const char file[], const char help[]);
PetscErrorCode PetscFinalize(void);
PetscErrorCode MatFactorInfoInitialize(MatFactorInfo* info);

/* Vec */
PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec* v);
PetscErrorCode VecCreateMPI(MPI_Comm comm, PetscInt n, PetscInt N, Vec* v);
PetscErrorCode VecDestroy(Vec* v);
PetscErrorCode VecDuplicate(Vec v, Vec* out);
PetscErrorCode VecZeroEntries(Vec v);
PetscErrorCode VecSet(Vec v, PetscScalar a);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecAYPX(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y);
PetscErrorCode VecScale(Vec v, PetscScalar a);
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar* val);
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal* val);
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar a, InsertMode mode);
PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt ix[], const PetscScalar y[], InsertMode mode);
PetscErrorCode VecGetValues(Vec v, PetscInt n, const PetscInt ix[], PetscScalar y[]);
PetscErrorCode VecAssemblyBegin(Vec v);
PetscErrorCode VecAssemblyEnd(Vec v);
PetscErrorCode VecGetArray(Vec v, PetscScalar** a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar** a);
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar** a);
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar** a);
PetscErrorCode VecGetSize(Vec v, PetscInt* n);
PetscErrorCode VecGetLocalSize(Vec v, PetscInt* n);
PetscErrorCode VecGetOwnershipRange(Vec v, PetscInt* lo, PetscInt* hi);
PetscErrorCode VecScatterCreate(Vec x, IS ix, Vec y, IS iy, VecScatter* sc);
PetscErrorCode VecScatterCreateToAll(Vec x, VecScatter* sc, Vec* out);
PetscErrorCode VecScatterBegin(VecScatter sc, Vec x, Vec y, InsertMode mode, ScatterMode smode);
PetscErrorCode VecScatterEnd(VecScatter sc, Vec x, Vec y, InsertMode mode, ScatterMode smode);
PetscErrorCode VecScatterDestroy(VecScatter* sc);

/* IS */
PetscErrorCode ISCreateGeneral(MPI_Comm comm, PetscInt n, const PetscInt idx[], PetscCopyMode mode, IS* is);
PetscErrorCode ISDestroy(IS* is);

/* Mat */
PetscErrorCode MatCreate(MPI_Comm comm, Mat* A);
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt M, PetscInt N);
PetscErrorCode MatSetType(Mat A, MatType t);
PetscErrorCode MatSetFromOptions(Mat A);
PetscErrorCode MatMPIAIJSetPreallocation(Mat A, PetscInt d_nz, const PetscInt d_nnz[], PetscInt o_nz, const PetscInt o_nnz[]);
PetscErrorCode MatSeqAIJSetPreallocation(Mat A, PetscInt nz, const PetscInt nnz[]);
PetscErrorCode MatCreateSeqAIJ(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt nz, const PetscInt nnz[], Mat* A);
PetscErrorCode MatCreateSeqDense(MPI_Comm comm, PetscInt m, PetscInt n, PetscScalar* data, Mat* A);
PetscErrorCode MatCreateDense(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N, PetscScalar* data, Mat* A);
PetscErrorCode MatSetUp(Mat A);
PetscErrorCode MatSetOption(Mat A, MatOption op, PetscBool flg);
PetscErrorCode MatSetBlockSize(Mat A, PetscInt bs);
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode);
PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt im[], PetscInt n, const PetscInt in[], const PetscScalar v[], InsertMode mode);
PetscErrorCode MatGetValues(Mat A, PetscInt m, const PetscInt im[], PetscInt n, const PetscInt in[], PetscScalar v[]);
PetscErrorCode MatAssemblyBegin(Mat A, MatAssemblyType t);
PetscErrorCode MatAssemblyEnd(Mat A, MatAssemblyType t);
PetscErrorCode MatZeroEntries(Mat A);
PetscErrorCode MatDestroy(Mat* A);
PetscErrorCode MatMult(Mat A, Vec x, Vec y);
PetscErrorCode MatMultAdd(Mat A, Vec x, Vec y, Vec z);
PetscErrorCode MatMultTranspose(Mat A, Vec x, Vec y);
PetscErrorCode MatGetSize(Mat A, PetscInt* m, PetscInt* n);
PetscErrorCode MatGetLocalSize(Mat A, PetscInt* m, PetscInt* n);
PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt* lo, PetscInt* hi);
PetscErrorCode MatGetOwnershipRangeColumn(Mat A, PetscInt* lo, PetscInt* hi);
PetscErrorCode MatGetColumnVector(Mat A, Vec v, PetscInt col);
PetscErrorCode MatGetOrdering(Mat A, MatOrderingType t, IS* rperm, IS* cperm);
PetscErrorCode MatGetFactor(Mat A, MatSolverPackage pkg, MatFactorType t, Mat* F);
PetscErrorCode MatCholeskyFactorSymbolic(Mat F, Mat A, IS perm, const MatFactorInfo* info);
PetscErrorCode MatCholeskyFactorNumeric(Mat F, Mat A, const MatFactorInfo* info);
PetscErrorCode MatMatSolve(Mat F, Mat B, Mat X);
PetscErrorCode MatTranspose(Mat A, int reuse, Mat* B);

/* KSP / PC */
PetscErrorCode KSPCreate(MPI_Comm comm, KSP* ksp);
PetscErrorCode KSPDestroy(KSP* ksp);
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat P);
PetscErrorCode KSPGetPC(KSP ksp, PC* pc);
PetscErrorCode KSPSetType(KSP ksp, KSPType t);
PetscErrorCode KSPCGSetType(KSP ksp, KSPCGType t);
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal abstol, PetscReal dtol, PetscInt maxits);
PetscErrorCode KSPSetFromOptions(KSP ksp);
PetscErrorCode KSPSetUp(KSP ksp);
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPSolveTranspose(KSP ksp, Vec b, Vec x);
PetscErrorCode PCSetType(PC pc, PCType t);
PetscErrorCode PCFactorSetMatSolverPackage(PC pc, MatSolverPackage pkg);
PetscErrorCode PCHYPRESetType(PC pc, const char* t);
PetscErrorCode PCSetCoordinates(PC pc, PetscInt dim, PetscInt n, PetscReal* coords);

/* SNES */
typedef PetscErrorCode (*SNESFunctionFn)(SNES, Vec, Vec, void*);
typedef PetscErrorCode (*SNESJacobianFn)(SNES, Vec, Mat, Mat, void*);
typedef PetscErrorCode (*SNESMonitorFn)(SNES, PetscInt, PetscReal, void*);
PetscErrorCode SNESCreate(MPI_Comm comm, SNES* snes);
PetscErrorCode SNESDestroy(SNES* snes);
PetscErrorCode SNESGetKSP(SNES snes, KSP* ksp);
PetscErrorCode SNESSetType(SNES snes, SNESType t);
PetscErrorCode SNESSetTolerances(SNES snes, PetscReal abstol, PetscReal rtol, PetscReal stol, PetscInt maxit, PetscInt maxf);
PetscErrorCode SNESSetFunction(SNES snes, Vec r, SNESFunctionFn f, void* ctx);
PetscErrorCode SNESSetJacobian(SNES snes, Mat A, Mat P, SNESJacobianFn f, void* ctx);
PetscErrorCode SNESMonitorSet(SNES snes, SNESMonitorFn f, void* ctx, void* destroy);
PetscErrorCode SNESSolve(SNES snes, Vec b, Vec x);
PetscErrorCode SNESGetFunctionNorm(SNES snes, PetscReal* norm);
PetscErrorCode SNESGetConvergedReason(SNES snes, SNESConvergedReason* reason);
PetscErrorCode SNESGetIterationNumber(SNES snes, PetscInt* its);

/* Shim-only introspection used by the oracle driver (not PETSc API). */
PetscInt pgshim_mat_rows(Mat A);
PetscInt pgshim_mat_cols(Mat A);
PetscInt pgshim_mat_row_nnz(Mat A, PetscInt row);
void pgshim_mat_row(Mat A, PetscInt row, PetscInt* cols, PetscScalar* vals);
PetscInt pgshim_vec_size(Vec v);
PetscScalar* pgshim_vec_data(Vec v);
double pgshim_ksp_seconds(void);
long pgshim_ksp_solves(void);
long pgshim_snes_iterations(void);
void pgshim_set_snes_verbose(int v);

#ifdef __cplusplus
}
#endif

#endif
