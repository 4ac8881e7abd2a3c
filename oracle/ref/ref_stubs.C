// Link stubs for third-party libraries that the reference links in binary
// form (EXT_LIB: UMFPACK, AMG driver, LAPACK).  None of them is on the path
// the oracle driver runs, except the dense LU pair dgetrf_/dgetrs_ reached
// through the coarse smoother "17" (TMGLevel3D::SolveExact -> SolveLinearSystem,
// src/FE/LinAlg.C:106-130); those two are written here from the textbook
// algorithm (Doolittle LU with partial pivoting, column-major like LAPACK).
// Everything else aborts loudly if ever reached.
#include <SquareMatrix.h>
#include <DirectSolver.h>
#include <cstdio>
#include <cstdlib>
#include <cmath>

static void unavailable(const char *what)
{
  fprintf(stderr, "oracle driver: %s is not available in this build\n", what);
  abort();
}

void DirectSolver(TSquareMatrix *, double *, double *) { unavailable("DirectSolver (UMFPACK)"); }
void DirectSolver(TSquareMatrix *, double *, double *, double *&, int *&, int *&, void *&, void *&, int)
{
  unavailable("DirectSolver (UMFPACK)");
}

extern "C" {
int AMG(...) { unavailable("AMG"); return 0; }
int AMG_Build(...) { unavailable("AMG_Build"); return 0; }
int AMG_Solve(...) { unavailable("AMG_Solve"); return 0; }
int AMG_Delete(...) { unavailable("AMG_Delete"); return 0; }
void dsteqr_(...) { unavailable("dsteqr_"); }
void dsptrd_(...) { unavailable("dsptrd_"); }
void dopgtr_(...) { unavailable("dopgtr_"); }
void dgetri_(...) { unavailable("dgetri_"); }
void dgemm_(...) { unavailable("dgemm_"); }

// LU factorisation with partial pivoting of an m x n column-major matrix.
void dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info)
{
  int M = *m, N = *n, ld = *lda, K = M < N ? M : N;
  *info = 0;
  for (int k = 0; k < K; k++)
  {
    int p = k;
    double best = fabs(a[k + (long)k * ld]);
    for (int i = k + 1; i < M; i++)
      if (fabs(a[i + (long)k * ld]) > best) { best = fabs(a[i + (long)k * ld]); p = i; }
    ipiv[k] = p + 1;
    if (best == 0.0) { if (!*info) *info = k + 1; continue; }
    if (p != k)
      for (int j = 0; j < N; j++)
      {
        double t = a[k + (long)j * ld];
        a[k + (long)j * ld] = a[p + (long)j * ld];
        a[p + (long)j * ld] = t;
      }
    double inv = 1.0 / a[k + (long)k * ld];
    for (int i = k + 1; i < M; i++) a[i + (long)k * ld] *= inv;
    for (int j = k + 1; j < N; j++)
    {
      double akj = a[k + (long)j * ld];
      if (akj != 0.0)
        for (int i = k + 1; i < M; i++) a[i + (long)j * ld] -= a[i + (long)k * ld] * akj;
    }
  }
}

// Solve with the factors of dgetrf_ (trans = 'N' or 'T').
void dgetrs_(char *trans, int *n, int *nrhs, double *a, int *lda, int *ipiv, double *b, int *ldb, int *info)
{
  int N = *n, ld = *lda, ldB = *ldb;
  *info = 0;
  bool t = (*trans == 'T' || *trans == 't');
  for (int r = 0; r < *nrhs; r++)
  {
    double *x = b + (long)r * ldB;
    if (!t)
    {
      for (int k = 0; k < N; k++)
        if (ipiv[k] - 1 != k) { double s = x[k]; x[k] = x[ipiv[k] - 1]; x[ipiv[k] - 1] = s; }
      for (int j = 0; j < N; j++)
        for (int i = j + 1; i < N; i++) x[i] -= a[i + (long)j * ld] * x[j];
      for (int j = N - 1; j >= 0; j--)
      {
        x[j] /= a[j + (long)j * ld];
        for (int i = 0; i < j; i++) x[i] -= a[i + (long)j * ld] * x[j];
      }
    }
    else
    {
      for (int j = 0; j < N; j++)
      {
        double s = x[j];
        for (int i = 0; i < j; i++) s -= a[i + (long)j * ld] * x[i];
        x[j] = s / a[j + (long)j * ld];
      }
      for (int j = N - 1; j >= 0; j--)
      {
        double s = x[j];
        for (int i = j + 1; i < N; i++) s -= a[i + (long)j * ld] * x[i];
        x[j] = s;
      }
      for (int k = N - 1; k >= 0; k--)
        if (ipiv[k] - 1 != k) { double s = x[k]; x[k] = x[ipiv[k] - 1]; x[ipiv[k] - 1] = s; }
    }
  }
}
}

// Tecplot binary writer (TOutput3D::WriteBinaryPlt): report failure, as the
// writer does when the library cannot open its file
int TECINI112(...) { return -1; }
int TECZNE112(...) { return -1; }
int TECDAT112(...) { return -1; }
int TECNOD112(...) { return -1; }
int TECEND112(...) { return -1; }
int TECEND(...) { return -1; }
