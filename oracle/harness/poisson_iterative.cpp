/*
 * poisson_iterative.cpp -- ORACLE TEST INFRASTRUCTURE.  Implements the
 * reference's PoissonSolver classes (include/PoissonSolver.h:1-51) for the
 * single-rank oracle build, in place of src/PoissonSolver.cpp:48-78, which
 * factorises with Amesos-KLU (Trilinos, third-party, absent here).
 *
 * The matrix is the reference's own (MeshQuantities::init_matrix,
 * src/mcmodel.cpp:4695-4869, collected by the shim Epetra_CrsMatrix).
 * KLU is a direct solve; here a Jacobi-preconditioned BiCGSTAB iterates to a
 * relative residual of 1e-14 (the Aztec path of the same file asks
 * Iterate(320, 1e-14), src/PoissonSolver.cpp:41), which is what "the same
 * potential" means for a direct solve in double precision.
 */
#include "mcmodel.h"
#include "PoissonSolver.h"

namespace {

void crs_apply(const Epetra_CrsMatrix &A, const std::vector<double> &x, std::vector<double> &y) {
  const Epetra_Map &m = A.RowMap();
  for (int r = 0; r < A.NumMyRows(); ++r) {
    double s = 0;
    for (const auto &e : A.Row(r)) s += e.second * x[m.LID(e.first)];
    y[r] = s;
  }
}

double dot(const std::vector<double> &a, const std::vector<double> &b) {
  double s = 0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}

/* Jacobi-preconditioned BiCGSTAB (van der Vorst 1992). */
void bicgstab(const Epetra_CrsMatrix &A, const std::vector<double> &b, std::vector<double> &x) {
  const int n = A.NumMyRows();
  const Epetra_Map &m = A.RowMap();
  std::vector<double> dinv(n, 1.0);
  for (int r = 0; r < n; ++r)
    for (const auto &e : A.Row(r))
      if (m.LID(e.first) == r && e.second != 0) dinv[r] = 1.0 / e.second;
  std::vector<double> r(n), rh(n), p(n, 0), v(n, 0), s(n), t(n), ph(n), sh(n), ax(n);
  crs_apply(A, x, ax);
  for (int i = 0; i < n; ++i) r[i] = b[i] - ax[i];
  rh = r;
  const double bn = std::sqrt(dot(b, b)) > 0 ? std::sqrt(dot(b, b)) : 1.0;
  double rho = 1, alpha = 1, omega = 1;
  for (int it = 0; it < 20000; ++it) {
    if (std::sqrt(dot(r, r)) / bn < 1e-14) break;
    double rho1 = dot(rh, r);
    if (rho1 == 0) break;
    double beta = (rho1 / rho) * (alpha / omega);
    for (int i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    for (int i = 0; i < n; ++i) ph[i] = dinv[i] * p[i];
    crs_apply(A, ph, v);
    alpha = rho1 / dot(rh, v);
    for (int i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
    for (int i = 0; i < n; ++i) sh[i] = dinv[i] * s[i];
    crs_apply(A, sh, t);
    double tt = dot(t, t);
    omega = tt > 0 ? dot(t, s) / tt : 0;
    for (int i = 0; i < n; ++i) x[i] += alpha * ph[i] + omega * sh[i];
    for (int i = 0; i < n; ++i) r[i] = s[i] - omega * t[i];
    rho = rho1;
    if (omega == 0) break;
  }
}

}  // namespace

PoissonSolver::PoissonSolver(MeshQuantities *mq) { A = mq->init_matrix(); }

Amesos_PoissonSolver::Amesos_PoissonSolver(MeshQuantities *mq) : PoissonSolver(mq) {
  Amesos_Problem = new Epetra_LinearProblem;
  Amesos_Problem->SetOperator(A);
  DSolver = nullptr;
}

void Amesos_PoissonSolver::solve_poisson(Epetra_Vector *rhs, Epetra_Vector *sol) {
  std::vector<double> b(rhs->MyLength()), x(sol->MyLength());
  for (int i = 0; i < rhs->MyLength(); ++i) b[i] = (*rhs)[i];
  for (int i = 0; i < sol->MyLength(); ++i) x[i] = (*sol)[i];
  bicgstab(*A, b, x);
  for (int i = 0; i < sol->MyLength(); ++i) (*sol)[i] = x[i];
}

Amesos_PoissonSolver::~Amesos_PoissonSolver() { delete Amesos_Problem; }

Aztec_PoissonSolver::Aztec_PoissonSolver(MeshQuantities *mq) : PoissonSolver(mq) {
  Aztec_Problem = new Epetra_LinearProblem;
  Aztec_Problem->SetOperator(A);
}

void Aztec_PoissonSolver::solve_poisson(Epetra_Vector *rhs, Epetra_Vector *sol) {
  std::vector<double> b(rhs->MyLength()), x(sol->MyLength());
  for (int i = 0; i < rhs->MyLength(); ++i) b[i] = (*rhs)[i];
  for (int i = 0; i < sol->MyLength(); ++i) x[i] = (*sol)[i];
  bicgstab(*A, b, x);
  for (int i = 0; i < sol->MyLength(); ++i) (*sol)[i] = x[i];
}

Aztec_PoissonSolver::~Aztec_PoissonSolver() { delete Aztec_Problem; }
