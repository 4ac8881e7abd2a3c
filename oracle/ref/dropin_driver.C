// Drop-in check of TPmgSystemCD3D (parmoon_b200/shim) against the reference's
// own TSystemCD3D, both driven the way 3DPrograms/CD3D_ParMooN.C:385-450
// drives the system class: same domain, same FE spaces, same callbacks.
// This file is test infrastructure: the reference arm is the checker.
//
//   pmg_dropin <outdir> key=value ...
// Keys: order(1) levels(3) coarse_steps(1) problem(laplace|cd)
//   geo(Wuerfel|SixTetras) device_coeffs(0) red(1e-10)
// order is ANSATZ_ORDER: 1 and 2 give Q1 and Q2 on Wuerfel, P1 and P2 on
// SixTetras.  Prints one line "dropin k=v ..." for the tests.
#include <Domain.h>
#include <Database.h>
#include <FEDatabase3D.h>
#include <FESpace3D.h>
#include <SquareMatrix3D.h>
#include <SystemCD3D.h>
#include <LinAlg.h>
#include <MooNMD_Io.h>
#include <FEFunction3D.h>
#include <Output3D.h>
#include <Collection.h>
#include <BaseCell.h>
#include "../../parmoon_b200/shim/pmg_parmoon.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include <sys/stat.h>

static std::map<std::string, std::string> g_opt;
static double optd(const char *k, double d) { return g_opt.count(k) ? atof(g_opt[k].c_str()) : d; }
static std::string opts(const char *k, const char *d) { return g_opt.count(k) ? g_opt[k] : std::string(d); }
static double wall() {
  return 1e-9 * std::chrono::duration_cast<std::chrono::nanoseconds>(
                    std::chrono::steady_clock::now().time_since_epoch()).count();
}

// problem 0: Laplace.h of Examples/CD_3D (u = sin sin sin); problem 1: convection-
// diffusion-reaction with a non-constant field and non-zero boundary values
static int g_problem = 0;
void BoundCondFn(int, double, double, double, BoundCond &cond) { cond = DIRICHLET; }
void BoundValueFn(int, double x, double y, double z, double &value) {
  value = g_problem == 0 ? sin(Pi * x) * sin(Pi * y) * sin(Pi * z) : 1.0 + x - 0.5 * y * z;
}
void CoeffsFn(int n_points, double *X, double *Y, double *Z, double **, double **coeffs) {
  for (int i = 0; i < n_points; i++) {
    double *c = coeffs[i];
    if (g_problem == 0) {
      c[0] = 1; c[1] = c[2] = c[3] = c[4] = 0;
      c[5] = 3 * Pi * Pi * sin(Pi * X[i]) * sin(Pi * Y[i]) * sin(Pi * Z[i]);
    } else {
      c[0] = 0.05 * (1.0 + 0.5 * sin(2 * Pi * X[i]) * cos(Pi * Y[i]));
      c[1] = 1.0; c[2] = 0.5 * Z[i]; c[3] = -0.25;
      c[4] = 0.5;
      c[5] = 1.0 + X[i] * Y[i];
    }
    c[6] = sqrt(c[1] * c[1] + c[2] * c[2] + c[3] * c[3]);
  }
}

// the reference system class, with its level matrices readable for the comparison
struct RefSystem : public TSystemCD3D {
  using TSystemCD3D::TSystemCD3D;
  TSquareMatrix3D *A(int i) { return sqmatrixA[i]; }
};

int main(int argc, char **argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s <outdir> key=value...\n", argv[0]);
    return 1;
  }
  std::string out = argv[1];
  mkdir(out.c_str(), 0777);
  for (int i = 2; i < argc; i++) {
    std::string a = argv[i];
    size_t p = a.find('=');
    if (p != std::string::npos) g_opt[a.substr(0, p)] = a.substr(p + 1);
  }
  std::string self = argv[0];
  size_t sl = self.rfind('/');
  std::string data = opts("data", ((sl == std::string::npos ? std::string(".") : self.substr(0, sl)) + "/data").c_str());
  const int order = (int)optd("order", 1), levels = (int)optd("levels", 3), coarse = (int)optd("coarse_steps", 1);
  g_problem = opts("problem", "laplace") == "laplace" ? 0 : 1;
  const std::string geo = opts("geo", "Wuerfel");

  std::string dat = out + "/run.dat";
  FILE *f = fopen(dat.c_str(), "w");
  fprintf(f, "VERSION: 1\nGEOFILE: %s/%s.GEO\nBNDFILE: %s/Wuerfel.PRM\n", data.c_str(), geo.c_str(), data.c_str());
  fprintf(f, "OUTFILE: %s/dropin.out\nLOGFILE: %s/dropin.log\nMESH_TYPE: 0\nUSE_PRM: 1\n", out.c_str(), out.c_str());
  fprintf(f, "ANSATZ_ORDER: %d\nLEVELS: %d\nUNIFORM_STEPS: %d\nSOLVER_TYPE: 1\nSC_VERBOSE: 0\n", order, levels, coarse);
  fclose(f);
  TDatabase *Database = new TDatabase();
  TFEDatabase3D *FEDatabase = new TFEDatabase3D();
  TDomain *Domain = new TDomain((char *)dat.c_str());
  OpenFiles();
  TParamDB *db = TDatabase::ParamDB;
  db->ANSATZ_ORDER = order;
  db->INTERNAL_POLYNOMIAL_DEGREE = order;
  db->INTERNAL_PROBLEM_LINEAR = 1;
  db->DISCTYPE = GALERKIN;
  db->SC_SOLVER_SCALAR = 16;
  db->SC_PRECONDITIONER_SCALAR = 5;
  db->SC_SMOOTHER_SCALAR = 3;
  db->SC_PRE_SMOOTH_SCALAR = db->SC_POST_SMOOTH_SCALAR = 2;
  db->SC_COARSE_SMOOTHER_SCALAR = 3;
  db->SC_COARSE_MAXIT_SCALAR = 10;
  db->SC_COARSE_RED_FACTOR_SCALAR = 0.1;
  db->SC_LIN_RED_FACTOR_SCALAR = optd("red", 1e-10);
  db->SC_LIN_RES_NORM_MIN_SCALAR = 0.0;
  db->SC_LIN_MAXIT_SCALAR = 1000;
  db->SC_GMRES_RESTART = 20;
  db->SC_FLEXIBLE_KRYLOV_SPACE_SOLVER = 1;
  db->SC_MG_CYCLE_SCALAR = 1;
  db->SC_SMOOTH_DAMP_FACTOR_SCALAR = db->SC_SMOOTH_DAMP_FACTOR_FINE_SCALAR = 1.0;
  db->SC_GMG_DAMP_FACTOR_SCALAR = 1.0;
  db->SC_STEP_LENGTH_CONTROL_ALL_SCALAR = db->SC_STEP_LENGTH_CONTROL_FINE_SCALAR = 0;
  db->SC_MG_TYPE_SCALAR = 0;
  db->SC_VERBOSE = 0;
  Domain->Init(db->BNDFILE, db->GEOFILE);
  for (int i = 0; i < coarse; i++) Domain->RegRefineAll();

  // FE spaces and one set of arrays per arm (CD3D_ParMooN.C:278-351)
  char Name[] = "c", Desc[] = "c";
  std::vector<TFESpace3D *> sp(levels);
  std::vector<std::vector<double>> sr(levels), rr(levels), sp_(levels), rp_(levels);
  std::vector<double *> Sol_ref(levels), Rhs_ref(levels), Sol_pmg(levels), Rhs_pmg(levels);
  for (int i = 0; i < levels; i++) {
    if (i) Domain->RegRefineAll();
    sp[i] = new TFESpace3D(Domain->GetCollection(It_Finest, 0), Name, Desc, BoundCondFn, order);
    const int N = sp[i]->GetN_DegreesOfFreedom();
    sr[i].assign(N, 0.0); rr[i].assign(N, 0.0); sp_[i].assign(N, 0.0); rp_[i].assign(N, 0.0);
    Sol_ref[i] = sr[i].data(); Rhs_ref[i] = rr[i].data(); Sol_pmg[i] = sp_[i].data(); Rhs_pmg[i] = rp_[i].data();
  }
  const int F = levels - 1, N = sp[F]->GetN_DegreesOfFreedom();

  // reference arm
  RefSystem *R = new RefSystem(levels, sp.data(), Sol_ref.data(), Rhs_ref.data(), GALERKIN, GMG);
  R->Init(CoeffsFn, BoundCondFn, BoundValueFn, NULL);
  double t0 = wall();
  R->Assemble();
  const double t_ref_asm = wall() - t0;
  std::vector<double> rhs_ref(Rhs_ref[F], Rhs_ref[F] + N);
  t0 = wall();
  R->Solve(Sol_ref[F], Rhs_ref[F]);
  const double t_ref_solve = wall() - t0;

  // device arm, through the drop-in class
  TPmgSystemCD3D *P = new TPmgSystemCD3D(levels, sp.data(), Sol_pmg.data(), Rhs_pmg.data(), GALERKIN, GMG);
  if (optd("device_coeffs", 0) != 0 && g_problem == 0) {
    pmg_coeff_desc c{};
    c.kind = PMG_COEF_SINE_RHS;
    c.eps = 1.0;
    P->Init(CoeffsFn, BoundCondFn, BoundValueFn, NULL, c);
  } else {
    P->Init(CoeffsFn, BoundCondFn, BoundValueFn, NULL);
  }
  P->Assemble();  // first call: device set-up (patterns, slot maps, tables)
  t0 = wall();
  P->Assemble();
  const double t_pmg_asm = wall() - t0;
  std::vector<double> rhs_pmg(Rhs_pmg[F], Rhs_pmg[F] + N);
  t0 = wall();
  P->Solve(Sol_pmg[F], Rhs_pmg[F]);
  const double t_pmg_solve = wall() - t0;
  P->CopyMatricesToHost();
  if (P->GetLastStatus() != PMG_OK) {
    printf("dropin status=%d\n", P->GetLastStatus());
    return 2;
  }

  // comparison: every level's matrix, the finest rhs, the solution, the true residuals
  double mat = 0, mat_scale = 0;
  for (int i = 0; i < levels; i++) {
    const int nnz = R->A(i)->GetN_Entries();
    const double *a = R->A(i)->GetEntries(), *b = P->GetAMatrix()[i]->GetEntries();
    for (int k = 0; k < nnz; k++) {
      mat = std::fmax(mat, std::fabs(a[k] - b[k]));
      mat_scale = std::fmax(mat_scale, std::fabs(a[k]));
    }
  }
  double rhs = 0, rhs_scale = 0, sol = 0, sol_scale = 0;
  for (int k = 0; k < N; k++) {
    rhs = std::fmax(rhs, std::fabs(rhs_ref[k] - rhs_pmg[k]));
    rhs_scale = std::fmax(rhs_scale, std::fabs(rhs_ref[k]));
    sol = std::fmax(sol, std::fabs(Sol_ref[F][k] - Sol_pmg[F][k]));
    sol_scale = std::fmax(sol_scale, std::fabs(Sol_ref[F][k]));
  }
  std::vector<double> d(N);
  double res_ref, res_pmg;
  ScalarDefect(R->A(F), Sol_ref[F], rhs_ref.data(), d.data(), res_ref);
  ScalarDefect(R->A(F), Sol_pmg[F], rhs_ref.data(), d.data(), res_pmg);
  printf("dropin N=%d levels=%d mat_rel=%.3e rhs_rel=%.3e sol_rel=%.3e res_ref=%.3e res_pmg=%.3e "
         "pmg_iterations=%d t_ref_assemble=%.4f t_pmg_assemble=%.4f t_ref_solve=%.4f t_pmg_solve=%.4f\n",
         N, levels, mat / mat_scale, rhs / rhs_scale, sol / sol_scale, res_ref, res_pmg,
         P->GetSolveStats().iterations, t_ref_asm, t_pmg_asm, t_ref_solve, t_pmg_solve);
  // vtk=1: the finest solution of each arm as a VTK file, the reference's
  // through TOutput3D::WriteVtk (as CD3D_ParMooN.C:477-495), ours through
  // pmg_write_vtk from the device-resident solution
  if (optd("vtk", 0) != 0) {
    TFEFunction3D *fe = new TFEFunction3D(sp[F], Name, Desc, Sol_ref[F], N);
    TOutput3D *out3 = new TOutput3D(2, 2, 1, 1, Domain);
    out3->AddFEFunction(fe);
    out3->WriteVtk((out + "/ref.vtk").c_str());
    TCollection *coll = sp[F]->GetCollection();
    std::vector<int> region(coll->GetN_Cells());
    for (int c = 0; c < coll->GetN_Cells(); c++) region[c] = coll->GetCell(c)->GetRegionID();
    const int rc = pmg_write_vtk(P->GetHandle(), F, NULL, region.data(), (out + "/pmg.vtk").c_str(), Name);
    printf("vtk status=%d\n", rc);
  }
  delete P;
  (void)Database; (void)FEDatabase;
  return 0;
}
