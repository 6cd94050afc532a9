/* Minimal PETSc KSP/MatShell stand-in used ONLY to compile the reference
 * solver as a CPU oracle (test infrastructure).  It provides sequential
 * vectors, a shell matrix with a user MatMult callback, and a restarted
 * GMRES(30) Krylov solver written from Saad & Schultz (1986), "GMRES: a
 * generalized minimal residual algorithm for solving nonsymmetric linear
 * systems", SIAM J. Sci. Stat. Comput. 7(3), with modified Gram-Schmidt
 * and Givens rotations.  No preconditioner (the reference selects PCNONE).
 * Convergence follows PETSc's documented default test:
 *   ||r_k||_2 <= max(rtol * ||b||_2, atol). */
#ifndef ORACLE_SHIM_PETSCKSP_H
#define ORACLE_SHIM_PETSCKSP_H
#include <mpi.h>
#include <cstdio>
#include <cstdlib>

typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscErrorCode;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef MPI_Comm PetscComm;
typedef struct oracle_vec *Vec;
typedef struct oracle_mat *Mat;
typedef struct oracle_ksp *KSP;
typedef struct oracle_pc *PC;
typedef const char *KSPType;
typedef const char *PCType;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_INFINITY = 3 } NormType;
typedef enum { MATOP_MULT = 3 } MatOperation;
typedef enum {
  KSP_CONVERGED_ITERATING = 0,
  KSP_CONVERGED_RTOL = 2,
  KSP_CONVERGED_ATOL = 3,
  KSP_DIVERGED_ITS = -3,
  KSP_DIVERGED_DTOL = -4,
  KSP_DIVERGED_BREAKDOWN = -5
} KSPConvergedReason;

#define PETSC_COMM_WORLD MPI_COMM_WORLD
#define PETSC_DEFAULT (-2)
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE PETSC_DECIDE
#define MPIU_INT MPI_INT
#define MPIU_SCALAR MPI_DOUBLE
#define MPIU_REAL MPI_DOUBLE
#define KSPGMRES "gmres"
#define PCNONE "none"
#define PETSC_ERR_LIB 76
#define PETSC_ERR_ARG_NULL 85
#define PETSC_ERR_ARG_WRONG 62

#define PetscCallAbort(comm, expr)                                                  \
  do {                                                                              \
    PetscErrorCode oracle_ierr_ = (expr);                                           \
    if (oracle_ierr_) {                                                             \
      std::fprintf(stderr, "oracle petsc shim: error %d in %s\n", oracle_ierr_, #expr); \
      std::abort();                                                                 \
    }                                                                               \
  } while (0)
#define PetscCall(expr)                              \
  do {                                               \
    PetscErrorCode oracle_ierr_ = (expr);            \
    if (oracle_ierr_) return oracle_ierr_;           \
  } while (0)
#define PetscCheck(cond, comm, code, ...)            \
  do {                                               \
    if (!(cond)) {                                   \
      std::fprintf(stderr, __VA_ARGS__);             \
      std::fprintf(stderr, "\n");                    \
      return code;                                   \
    }                                                \
  } while (0)
#define SETERRQ(comm, code, ...)                     \
  do {                                               \
    std::fprintf(stderr, __VA_ARGS__);               \
    std::fprintf(stderr, "\n");                      \
    return code;                                     \
  } while (0)
#define PetscFunctionBeginUser
#define PetscFunctionReturn(x) return (x)

PetscErrorCode PetscInitialize(int *argc, char ***argv, const char *file, const char *help);
PetscErrorCode PetscFinalize(void);
PetscErrorCode PetscInitialized(PetscBool *flag);

PetscErrorCode VecCreateMPI(MPI_Comm comm, PetscInt n, PetscInt N, Vec *v);
PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec *v);
PetscErrorCode VecDuplicate(Vec v, Vec *out);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecSet(Vec v, PetscScalar a);
PetscErrorCode VecNorm(Vec v, NormType t, PetscReal *out);
PetscErrorCode VecGetArray(Vec v, PetscScalar **a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a);
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a);
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a);
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n);

PetscErrorCode MatCreateShell(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N, void *ctx, Mat *A);
PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*fn)(void));
PetscErrorCode MatShellGetContext(Mat A, void *ctx_out);
PetscErrorCode MatMult(Mat A, Vec x, Vec y);
PetscErrorCode MatDestroy(Mat *A);

PetscErrorCode KSPCreate(MPI_Comm comm, KSP *ksp);
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat P);
PetscErrorCode KSPSetType(KSP ksp, KSPType t);
PetscErrorCode KSPGetPC(KSP ksp, PC *pc);
PetscErrorCode PCSetType(PC pc, PCType t);
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal atol, PetscReal dtol, PetscInt maxit);
PetscErrorCode KSPSetFromOptions(KSP ksp);
PetscErrorCode KSPSetInitialGuessNonzero(KSP ksp, PetscBool flag);
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason *reason);
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt *its);
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal *rnorm);
PetscErrorCode KSPDestroy(KSP *ksp);

/* Oracle-only hooks: override the tolerances the solver asked for (parity
 * runs need a tight solve), and read the last solve's statistics. */
void oracle_ksp_force_tolerances(double rtol, double atol, int maxit);
int oracle_ksp_last_iterations(void);
#endif
