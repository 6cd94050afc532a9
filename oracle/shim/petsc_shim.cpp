// Minimal PETSc stand-in (oracle build only; see petscksp.h).
#include "petscksp.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

struct oracle_vec {
  std::vector<double> a;
};
typedef PetscErrorCode (*oracle_mult_fn)(Mat, Vec, Vec);
struct oracle_mat {
  PetscInt n = 0;
  void *ctx = nullptr;
  oracle_mult_fn mult = nullptr;
};
struct oracle_pc {
  int none = 1;
};
struct oracle_ksp {
  Mat A = nullptr;
  oracle_pc pc;
  double rtol = 1e-5, atol = 1e-50, dtol = 1e4;
  int maxit = 10000;
  bool guess_nonzero = false;
  int its = 0;
  double rnorm = 0.0;
  KSPConvergedReason reason = KSP_CONVERGED_ITERATING;
};

namespace {
bool g_force = false;
double g_rtol = 0.0, g_atol = 0.0;
int g_maxit = 0;
int g_last_its = 0;
constexpr int kRestart = 30;

double dot(const std::vector<double> &x, const std::vector<double> &y) {
  double s = 0.0;
  for (size_t i = 0; i < x.size(); ++i) s += x[i] * y[i];
  return s;
}
double nrm2(const std::vector<double> &x) { return std::sqrt(dot(x, x)); }
}  // namespace

void oracle_ksp_force_tolerances(double rtol, double atol, int maxit) {
  g_force = true;
  g_rtol = rtol;
  g_atol = atol;
  g_maxit = maxit;
}
int oracle_ksp_last_iterations(void) { return g_last_its; }

PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *) { return 0; }
PetscErrorCode PetscFinalize(void) { return 0; }
PetscErrorCode PetscInitialized(PetscBool *flag) {
  *flag = PETSC_TRUE;
  return 0;
}

PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt n, PetscInt, Vec *v) {
  *v = new oracle_vec();
  (*v)->a.assign((size_t)std::max(n, 0), 0.0);
  return 0;
}
PetscErrorCode VecCreateSeq(MPI_Comm c, PetscInt n, Vec *v) { return VecCreateMPI(c, n, n, v); }
PetscErrorCode VecDuplicate(Vec v, Vec *out) {
  *out = new oracle_vec();
  (*out)->a.assign(v->a.size(), 0.0);
  return 0;
}
PetscErrorCode VecDestroy(Vec *v) {
  delete *v;
  *v = nullptr;
  return 0;
}
PetscErrorCode VecSet(Vec v, PetscScalar a) {
  std::fill(v->a.begin(), v->a.end(), a);
  return 0;
}
PetscErrorCode VecNorm(Vec v, NormType t, PetscReal *out) {
  if (t == NORM_2) {
    *out = nrm2(v->a);
  } else if (t == NORM_1) {
    double s = 0.0;
    for (double x : v->a) s += std::fabs(x);
    *out = s;
  } else {
    double s = 0.0;
    for (double x : v->a) s = std::max(s, std::fabs(x));
    *out = s;
  }
  return 0;
}
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) {
  *a = v->a.data();
  return 0;
}
PetscErrorCode VecRestoreArray(Vec, PetscScalar **a) {
  *a = nullptr;
  return 0;
}
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a) {
  *a = v->a.data();
  return 0;
}
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **a) {
  *a = nullptr;
  return 0;
}
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n) {
  *n = (PetscInt)v->a.size();
  return 0;
}

PetscErrorCode MatCreateShell(MPI_Comm, PetscInt m, PetscInt, PetscInt, PetscInt, void *ctx, Mat *A) {
  *A = new oracle_mat();
  (*A)->n = m;
  (*A)->ctx = ctx;
  return 0;
}
PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*fn)(void)) {
  if (op != MATOP_MULT) return PETSC_ERR_ARG_WRONG;
  A->mult = reinterpret_cast<oracle_mult_fn>(fn);
  return 0;
}
PetscErrorCode MatShellGetContext(Mat A, void *ctx_out) {
  std::memcpy(ctx_out, &A->ctx, sizeof(void *));
  return 0;
}
PetscErrorCode MatMult(Mat A, Vec x, Vec y) { return A->mult(A, x, y); }
PetscErrorCode MatDestroy(Mat *A) {
  delete *A;
  *A = nullptr;
  return 0;
}

PetscErrorCode KSPCreate(MPI_Comm, KSP *ksp) {
  *ksp = new oracle_ksp();
  return 0;
}
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat) {
  ksp->A = A;
  return 0;
}
PetscErrorCode KSPSetType(KSP, KSPType t) { return std::strcmp(t, KSPGMRES) ? PETSC_ERR_ARG_WRONG : 0; }
PetscErrorCode KSPGetPC(KSP ksp, PC *pc) {
  *pc = &ksp->pc;
  return 0;
}
PetscErrorCode PCSetType(PC, PCType t) { return std::strcmp(t, PCNONE) ? PETSC_ERR_ARG_WRONG : 0; }
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal atol, PetscReal dtol, PetscInt maxit) {
  if (rtol != PETSC_DEFAULT) ksp->rtol = rtol;
  if (atol != PETSC_DEFAULT) ksp->atol = atol;
  if (dtol != PETSC_DEFAULT) ksp->dtol = dtol;
  if (maxit != PETSC_DEFAULT) ksp->maxit = maxit;
  return 0;
}
PetscErrorCode KSPSetFromOptions(KSP) { return 0; }
PetscErrorCode KSPSetInitialGuessNonzero(KSP ksp, PetscBool flag) {
  ksp->guess_nonzero = (flag == PETSC_TRUE);
  return 0;
}
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason *r) {
  *r = ksp->reason;
  return 0;
}
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt *its) {
  *its = ksp->its;
  return 0;
}
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal *rnorm) {
  *rnorm = ksp->rnorm;
  return 0;
}
PetscErrorCode KSPDestroy(KSP *ksp) {
  delete *ksp;
  *ksp = nullptr;
  return 0;
}

// Restarted GMRES(m), Saad & Schultz (1986) Algorithm 4 with modified
// Gram-Schmidt orthogonalisation and Givens rotations for the small
// least-squares problem.
PetscErrorCode KSPSolve(KSP ksp, Vec bv, Vec xv) {
  const double rtol = g_force ? g_rtol : ksp->rtol;
  const double atol = g_force ? g_atol : ksp->atol;
  const int maxit = g_force ? g_maxit : ksp->maxit;
  const size_t n = bv->a.size();
  std::vector<double> &x = xv->a;
  const std::vector<double> &b = bv->a;
  if (!ksp->guess_nonzero) std::fill(x.begin(), x.end(), 0.0);

  oracle_vec tmp_in, tmp_out;
  tmp_in.a.assign(n, 0.0);
  tmp_out.a.assign(n, 0.0);
  auto apply = [&](const std::vector<double> &v, std::vector<double> &out) -> PetscErrorCode {
    tmp_in.a = v;
    PetscErrorCode e = MatMult(ksp->A, &tmp_in, &tmp_out);
    out = tmp_out.a;
    return e;
  };

  const double bnorm = nrm2(b);
  const double ttol = std::max(rtol * bnorm, atol);
  std::vector<double> r(n), Ax(n);
  ksp->its = 0;
  ksp->reason = KSP_CONVERGED_ITERATING;

  while (true) {
    PetscCall(apply(x, Ax));
    for (size_t i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    double beta = nrm2(r);
    ksp->rnorm = beta;
    if (beta <= ttol) {
      ksp->reason = (beta <= atol) ? KSP_CONVERGED_ATOL : KSP_CONVERGED_RTOL;
      break;
    }
    if (ksp->its >= maxit) {
      ksp->reason = KSP_DIVERGED_ITS;
      break;
    }
    if (beta > ksp->dtol * std::max(bnorm, 1e-300)) {
      ksp->reason = KSP_DIVERGED_DTOL;
      break;
    }
    std::vector<std::vector<double>> V(kRestart + 1, std::vector<double>(n, 0.0));
    std::vector<std::vector<double>> H(kRestart + 1, std::vector<double>(kRestart, 0.0));
    std::vector<double> cs(kRestart, 0.0), sn(kRestart, 0.0), g(kRestart + 1, 0.0);
    for (size_t i = 0; i < n; ++i) V[0][i] = r[i] / beta;
    g[0] = beta;
    int k = 0;
    bool stop = false;
    for (; k < kRestart && ksp->its < maxit; ++k) {
      std::vector<double> w(n);
      PetscCall(apply(V[k], w));
      for (int j = 0; j <= k; ++j) {
        H[j][k] = dot(w, V[j]);
        for (size_t i = 0; i < n; ++i) w[i] -= H[j][k] * V[j][i];
      }
      H[k + 1][k] = nrm2(w);
      if (H[k + 1][k] > 0.0)
        for (size_t i = 0; i < n; ++i) V[k + 1][i] = w[i] / H[k + 1][k];
      for (int j = 0; j < k; ++j) {
        const double t = cs[j] * H[j][k] + sn[j] * H[j + 1][k];
        H[j + 1][k] = -sn[j] * H[j][k] + cs[j] * H[j + 1][k];
        H[j][k] = t;
      }
      const double den = std::hypot(H[k][k], H[k + 1][k]);
      cs[k] = den > 0.0 ? H[k][k] / den : 1.0;
      sn[k] = den > 0.0 ? H[k + 1][k] / den : 0.0;
      H[k][k] = den;
      H[k + 1][k] = 0.0;
      g[k + 1] = -sn[k] * g[k];
      g[k] = cs[k] * g[k];
      ksp->its++;
      ksp->rnorm = std::fabs(g[k + 1]);
      if (ksp->rnorm <= ttol || den == 0.0) {
        ++k;
        stop = true;
        break;
      }
    }
    // Back-substitute y = H^{-1} g and update x += V y.
    std::vector<double> y(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
      double s = g[i];
      for (int j = i + 1; j < k; ++j) s -= H[i][j] * y[j];
      y[i] = H[i][i] != 0.0 ? s / H[i][i] : 0.0;
    }
    for (int j = 0; j < k; ++j)
      for (size_t i = 0; i < n; ++i) x[i] += y[j] * V[j][i];
    (void)stop;
  }
  g_last_its = ksp->its;
  return 0;
}
