// Oracle driver for the compiled reference (ParMooN) 3D scalar convection-
// diffusion path.  This file is ours; it links against the reference's own
// objects (built by oracle/ref/Makefile from the read-only sources) and
// exercises exactly the classes the GPU path replaces:
//
//   TSquareStructure3D + Sort           src/FE/SquareStructure3D.C:58-527
//   TAssembleMat3D::Init/Reset/Assemble3D src/System/AssembleMat3D.C:261-535
//   BilinearAssemble / _SD               src/FE/ConvDiff3D.C:87-214
//   TMGLevel3D / TMultiGrid3D::Cycle     src/FE/MGLevel3D.C, src/FE/MultiGrid3D.C
//   TMultiGridScaIte / TFgmresIte        src/FE/MultiGridScaIte.C, src/FE/FgmresIte.C
//   Prolongate / DefectRestriction       src/FE/MGComponents3D.C:208, :732
//   TSystemTCD3D (time-dependent pin)    src/System/SystemTCD3D.C
//
// The driver is modelled on 3DPrograms/CD3D_ParMooN.C:72-599 and
// 3DPrograms/TCD3D_ParMooN.C:89-; it writes raw little-endian arrays into a
// dump directory so the Python tests and the C restatement can be compared
// against the reference entry by entry, and it times Assemble()/Solve() with
// a wall clock (the reference's own GetTime() is CPU user time).
//
// Usage:
//   pmg_ref cd3d   <outdir> key=value ...
//   pmg_ref tcd3d  <outdir> key=value ...
// Keys (defaults in parentheses): order(1) levels(3) coarse_steps(2)
//   problem(laplace|cdsupg|cdgal) eps(1) b1 b2 b3 (0) linear_quad(1)
//   disc(1=Galerkin,2=SUPG) restart(20) red(1e-10) maxit(1000) smoother(3)
//   pre(2) post(2) coarse_smoother(3) coarse_maxit(10) dump(1) solve(1)
//   omega(1) slc_all(0) slc_fine(0) dump_solution(0) mg_type(0: one space of
//   `order` per level; 1: N_Q1 / N_P1 on every mesh + `order` on the finest)
//   repeat(0) warmup(0) start_file (timing mode of the benchmark)
//   tau, endtime (tcd3d) geo(Wuerfel|SixTetras) order 12 = P2 on tetrahedra
#include <Domain.h>
#include <Database.h>
#include <FEDatabase3D.h>
#include <FESpace3D.h>
#include <SquareStructure3D.h>
#include <SquareMatrix3D.h>
#include <AssembleMat3D.h>
#include <DiscreteForm3D.h>
#include <AuxParam3D.h>
#include <MultiGrid3D.h>
#include <MGLevel3D.h>
#include <MultiGridScaIte.h>
#include <FgmresIte.h>
#include <ItMethod.h>
#include <LinAlg.h>
// Local-form signatures from src/FE/ConvDiff3D.C (the header that declares
// them also defines global tables, so they are declared here directly).
void BilinearAssemble(double Mult, double *coeff, double hK, double **OrigValues,
                      int *N_BaseFuncts, double ***LocMatrices, double **LocRhs);
void BilinearAssemble_SD(double Mult, double *coeff, double hK, double **OrigValues,
                         int *N_BaseFuncts, double ***LocMatrices, double **LocRhs);
// Term tables of the scalar CD forms: the four derivative values the forms
// read (d/dx, d/dy, d/dz, value), one square matrix, one rhs.
static int N_Terms = 4;
static MultiIndex3D Derivatives[4] = {D100, D010, D001, D000};
static int SpacesNumbers[4] = {0, 0, 0, 0};
static int N_Matrices = 1, RowSpace[1] = {0}, ColumnSpace[1] = {0};
static int N_Rhs = 1, RhsSpace[1] = {0};
#include <MainUtilities.h>
#include <FEFunction3D.h>
#include <SystemTCD3D.h>
#include <TimeDiscRout.h>
#include <Collection.h>
#include <BaseCell.h>
#include <Vertex.h>
#include <MooNMD_Io.h>

#include <string>
#include <map>
#include <vector>
#include <chrono>
#include <thread>
#include <sys/time.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <sys/stat.h>

// ---------------------------------------------------------------- options
static std::map<std::string, std::string> g_opt;
static double optd(const char *k, double d)
{
  auto it = g_opt.find(k);
  return it == g_opt.end() ? d : atof(it->second.c_str());
}
static std::string opts(const char *k, const char *d)
{
  auto it = g_opt.find(k);
  return it == g_opt.end() ? std::string(d) : it->second;
}
// seconds since the Unix epoch (a clock shared by concurrent processes)
static double epoch()
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static double wall()
{
  return std::chrono::duration<double>(
      std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------- problems
// problem ids: 0 laplace (Examples/CD_3D/Laplace.h), 1 cdsupg (constant
// convection, f=1, u=1 on x=0 else 0), 2 amc (Examples/TCD_3D/amc.h)
static int g_problem = 0;
static double g_eps = 1.0, g_b[3] = {0, 0, 0}, g_c = 0.0, g_f = 1.0;

void ExactFn(double x, double y, double z, double *values)
{
  if (g_problem == 2)
  {
    double t = TDatabase::TimeDB->CURRENTTIME, k = 0.1, e = exp(-k * t);
    values[0] = e * sin(Pi * x) * cos(Pi * y) * cos(Pi * z);
    values[1] = Pi * e * cos(Pi * x) * cos(Pi * y) * cos(Pi * z);
    values[2] = -Pi * e * sin(Pi * x) * sin(Pi * y) * cos(Pi * z);
    values[3] = -Pi * e * sin(Pi * x) * cos(Pi * y) * sin(Pi * z);
    values[4] = -3. * Pi * Pi * e * sin(Pi * x) * cos(Pi * y) * cos(Pi * z);
    return;
  }
  values[0] = sin(Pi * x) * sin(Pi * y) * sin(Pi * z);
  values[1] = Pi * cos(Pi * x) * sin(Pi * y) * sin(Pi * z);
  values[2] = Pi * sin(Pi * x) * cos(Pi * y) * sin(Pi * z);
  values[3] = Pi * sin(Pi * x) * sin(Pi * y) * cos(Pi * z);
  values[4] = -3 * Pi * Pi * sin(Pi * x) * sin(Pi * y) * sin(Pi * z);
}
void InitialFn(double x, double y, double z, double *values)
{
  values[0] = sin(Pi * x) * cos(Pi * y) * cos(Pi * z);
}
void BoundCondFn(int, double, double, double, BoundCond &cond) { cond = DIRICHLET; }
void BoundValueFn(int, double x, double y, double z, double &value)
{
  if (g_problem == 0)
    value = sin(Pi * x) * sin(Pi * y) * sin(Pi * z);
  else if (g_problem == 1)
    value = (fabs(x) < 1e-12) ? 1.0 : 0.0;
  else
  {
    double t = TDatabase::TimeDB->CURRENTTIME;
    value = exp(-0.1 * t) * sin(Pi * x) * cos(Pi * y) * cos(Pi * z);
  }
}
void CoeffsFn(int n_points, double *X, double *Y, double *Z, double **, double **coeffs)
{
  double t = TDatabase::TimeDB->CURRENTTIME;
  for (int i = 0; i < n_points; i++)
  {
    double *c = coeffs[i];
    if (g_problem == 0)
    {
      c[0] = g_eps; c[1] = 0; c[2] = 0; c[3] = 0; c[4] = 0;
      c[5] = 3 * Pi * Pi * g_eps * sin(Pi * X[i]) * sin(Pi * Y[i]) * sin(Pi * Z[i]);
      c[6] = 0;
    }
    else if (g_problem == 1)
    {
      c[0] = g_eps; c[1] = g_b[0]; c[2] = g_b[1]; c[3] = g_b[2]; c[4] = g_c;
      c[5] = g_f;
      c[6] = sqrt(g_b[0] * g_b[0] + g_b[1] * g_b[1] + g_b[2] * g_b[2]);
    }
    else
    {
      c[0] = 1.0; c[1] = 0; c[2] = 0; c[3] = 0; c[4] = 0;
      c[5] = (3. * Pi * Pi - 0.1) * exp(-0.1 * t) * sin(Pi * X[i]) * cos(Pi * Y[i]) * cos(Pi * Z[i]);
      c[6] = 0;
    }
  }
}

// ---------------------------------------------------------------- dumping
static std::string g_out;
static FILE *g_meta = NULL;
template <typename T>
static void dump(const std::string &name, const T *p, long n, const char *dtype)
{
  std::string fn = g_out + "/" + name + ".bin";
  FILE *f = fopen(fn.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", fn.c_str()); exit(2); }
  if (n) fwrite(p, sizeof(T), n, f);
  fclose(f);
  fprintf(g_meta, "%s %s %ld\n", name.c_str(), dtype, n);
}
static void dumpScalar(const std::string &name, double v)
{
  fprintf(g_meta, "%s scalar %.17g\n", name.c_str(), v);
}

static void write_dat(const std::string &fn, int order, int levels, int coarse_steps)
{
  std::string data = opts("data", "");
  FILE *f = fopen(fn.c_str(), "w");
  std::string geo = opts("geo", "Wuerfel");
  fprintf(f, "VERSION: 1\nGEOFILE: %s/%s.GEO\nBNDFILE: %s/Wuerfel.PRM\n", data.c_str(), geo.c_str(), data.c_str());
  fprintf(f, "OUTFILE: %s/ref.out\nLOGFILE: %s/ref.log\n", g_out.c_str(), g_out.c_str());
  fprintf(f, "MESH_TYPE: 0\nUSE_PRM: 1\nWRITE_VTK: 0\nWRITE_PS: 0\nMEASURE_ERRORS: 0\n");
  fprintf(f, "ANSATZ_ORDER: %d\nLEVELS: %d\nUNIFORM_STEPS: %d\n", order, levels, coarse_steps);
  fprintf(f, "SOLVER_TYPE: 1\nSC_MG_TYPE_SCALAR: 0\nSC_VERBOSE: 0\n");
  fclose(f);
}

static void set_solver_params()
{
  TDatabase::ParamDB->SC_SOLVER_SCALAR = 16;
  TDatabase::ParamDB->SC_PRECONDITIONER_SCALAR = 5;
  TDatabase::ParamDB->SC_SMOOTHER_SCALAR = (int)optd("smoother", 3);
  TDatabase::ParamDB->SC_PRE_SMOOTH_SCALAR = (int)optd("pre", 2);
  TDatabase::ParamDB->SC_POST_SMOOTH_SCALAR = (int)optd("post", 2);
  TDatabase::ParamDB->SC_COARSE_SMOOTHER_SCALAR = (int)optd("coarse_smoother", 3);
  TDatabase::ParamDB->SC_COARSE_MAXIT_SCALAR = (int)optd("coarse_maxit", 10);
  TDatabase::ParamDB->SC_COARSE_RED_FACTOR_SCALAR = optd("coarse_red", 0.1);
  TDatabase::ParamDB->SC_LIN_RED_FACTOR_SCALAR = optd("red", 1e-10);
  TDatabase::ParamDB->SC_LIN_RES_NORM_MIN_SCALAR = optd("resmin", 0.0);
  TDatabase::ParamDB->SC_LIN_MAXIT_SCALAR = (int)optd("maxit", 1000);
  TDatabase::ParamDB->SC_GMRES_RESTART = (int)optd("restart", 20);
  TDatabase::ParamDB->SC_FLEXIBLE_KRYLOV_SPACE_SOLVER = 1;
  TDatabase::ParamDB->SC_MG_CYCLE_SCALAR = 1;
  TDatabase::ParamDB->SC_SMOOTH_DAMP_FACTOR_SCALAR = optd("omega", 1.0);
  TDatabase::ParamDB->SC_SMOOTH_DAMP_FACTOR_FINE_SCALAR = optd("omega", 1.0);
  TDatabase::ParamDB->SC_GMG_DAMP_FACTOR_SCALAR = 1.0;
  TDatabase::ParamDB->SC_STEP_LENGTH_CONTROL_ALL_SCALAR = (int)optd("slc_all", 0);
  TDatabase::ParamDB->SC_STEP_LENGTH_CONTROL_FINE_SCALAR = (int)optd("slc_fine", 0);
  TDatabase::ParamDB->SC_MG_TYPE_SCALAR = 0;
  TDatabase::ParamDB->SC_VERBOSE = 0;
}

// level data shared by both modes
struct Level
{
  TFESpace3D *space;
  TSquareStructure3D *structure;
  TSquareMatrix3D *A;
  double *sol, *rhs;
  int N;
};

static void dump_level(int l, Level &L)
{
  char p[64];
  snprintf(p, sizeof p, "L%d_", l);
  std::string pre(p);
  TFESpace3D *sp = L.space;
  TCollection *coll = sp->GetCollection();
  int nc = coll->GetN_Cells();
  int nloc = 0;
  int *gn = sp->GetGlobalNumbers(), *bi = sp->GetBeginIndex();
  nloc = bi[1] - bi[0];
  dumpScalar(pre + "N", L.N);
  dumpScalar(pre + "active_bound", sp->GetActiveBound());
  dumpScalar(pre + "hanging_bound", sp->GetHangingBound());
  dumpScalar(pre + "n_dirichlet", sp->GetN_Dirichlet());
  dumpScalar(pre + "n_cells", nc);
  dumpScalar(pre + "n_loc", nloc);
  int nnz = L.A->GetN_Entries();
  dump(pre + "rowptr", L.A->GetRowPtr(), L.N + 1, "i4");
  dump(pre + "kcol", L.A->GetKCol(), nnz, "i4");
  dump(pre + "entries", L.A->GetEntries(), nnz, "f8");
  dump(pre + "rhs", L.rhs, L.N, "f8");
  std::vector<int> ed((size_t)nc * nloc);
  std::vector<double> cv((size_t)nc * 8 * 3);
  for (int c = 0; c < nc; c++)
  {
    for (int k = 0; k < nloc; k++) ed[(size_t)c * nloc + k] = gn[bi[c] + k];
    TBaseCell *cell = coll->GetCell(c);
    int nv = cell->GetN_Vertices();
    for (int v = 0; v < 8; v++)
    {
      double x = 0, y = 0, z = 0;
      if (v < nv) cell->GetVertex(v)->GetCoords(x, y, z);
      cv[((size_t)c * 8 + v) * 3 + 0] = x;
      cv[((size_t)c * 8 + v) * 3 + 1] = y;
      cv[((size_t)c * 8 + v) * 3 + 2] = z;
    }
  }
  dump(pre + "elem_dof", ed.data(), (long)ed.size(), "i4");
  dump(pre + "cell_vert", cv.data(), (long)cv.size(), "f8");
  std::vector<double> x(L.N), y(L.N), z(L.N), xyz((size_t)L.N * 3);
  sp->GetDOFPosition(x.data(), y.data(), z.data());
  for (int i = 0; i < L.N; i++) { xyz[3 * i] = x[i]; xyz[3 * i + 1] = y[i]; xyz[3 * i + 2] = z[i]; }
  dump(pre + "dof_xyz", xyz.data(), (long)xyz.size(), "f8");
}

// ------------------------------------------------------------------ cd3d
static int run_cd3d()
{
  int order = (int)optd("order", 1), levels = (int)optd("levels", 3);
  int coarse_steps = (int)optd("coarse_steps", 2);
  std::string prob = opts("problem", "laplace");
  g_problem = prob == "laplace" ? 0 : 1;
  int disc = (int)optd("disc", prob == "cdsupg" ? 2 : 1);
  g_eps = optd("eps", 1.0);
  g_b[0] = optd("b1", 0); g_b[1] = optd("b2", 0); g_b[2] = optd("b3", 0);
  g_f = optd("f", 1.0);

  std::string dat = g_out + "/run.dat";
  write_dat(dat, order, levels, coarse_steps);
  TDatabase *Database = new TDatabase();
  TFEDatabase3D *FEDatabase = new TFEDatabase3D();
  TDomain *Domain = new TDomain((char *)dat.c_str());
  OpenFiles();
  TDatabase::ParamDB->INTERNAL_PROBLEM_LINEAR = (int)optd("linear_quad", 1);
  TDatabase::ParamDB->DISCTYPE = disc;
  TDatabase::ParamDB->ANSATZ_ORDER = order;
  TDatabase::ParamDB->INTERNAL_POLYNOMIAL_DEGREE = order;
  if (disc == 2)
  {
    TDatabase::ParamDB->SDFEM_TYPE = 2;
    TDatabase::ParamDB->CELL_MEASURE = 4;
    TDatabase::ParamDB->DELTA0 = 1.0;
  }
  set_solver_params();
  Domain->Init(TDatabase::ParamDB->BNDFILE, TDatabase::ParamDB->GEOFILE);
  for (int i = 0; i < coarse_steps; i++) Domain->RegRefineAll();

  char Name[] = "u", Desc[] = "u";
  // mg_type=1 (SC_MG_TYPE_SCALAR = 1, CD3D_ParMooN.C:258-313): the
  // non-conforming N_Q1 / N_P1 space (order -1) on every geometric level,
  // then the conforming space of `order` on the finest mesh as one more level
  const int mg_type = (int)optd("mg_type", 0), geo_levels = levels;
  if (mg_type) levels = geo_levels + 1;
  std::vector<Level> L(levels);
  TCollection *coll = NULL;
  for (int i = 0; i < levels; i++)
  {
    if (i && i < geo_levels) Domain->RegRefineAll();
    if (i < geo_levels) coll = Domain->GetCollection(It_Finest, 0);
    L[i].space = new TFESpace3D(coll, Name, Desc, BoundCondFn, (mg_type && i < geo_levels) ? -1 : order);
    L[i].N = L[i].space->GetN_DegreesOfFreedom();
    L[i].sol = new double[L[i].N]();
    L[i].rhs = new double[L[i].N]();
  }
  double t0 = wall();
  for (int i = 0; i < levels; i++)
  {
    L[i].structure = new TSquareStructure3D(L[i].space);
    L[i].structure->Sort();
    L[i].A = new TSquareMatrix3D(L[i].structure);
  }
  double t_struct = wall() - t0;

  // discrete form: Galerkin (InitializeDiscreteForms, DiscreteForm3D.C:3039) or
  // SUPG without 2nd derivatives (BilinearAssemble_SD, ConvDiff3D.C:150)
  TDiscreteForm3D *form;
  char cds[] = "CD", gal[] = "Galerkin", sd[] = "SUPG";
  if (disc == 2)
    form = new TDiscreteForm3D(cds, sd, N_Terms, Derivatives, SpacesNumbers,
                               N_Matrices, N_Rhs, RowSpace, ColumnSpace, RhsSpace,
                               BilinearAssemble_SD, CoeffsFn, NULL);
  else
    form = new TDiscreteForm3D(cds, gal, N_Terms, Derivatives, SpacesNumbers,
                               N_Matrices, N_Rhs, RowSpace, ColumnSpace, RhsSpace,
                               BilinearAssemble, CoeffsFn, NULL);

  // Parameters[0] is the smoothers' damping (and the step-length fallback),
  // as TSystemCD3D sets them (SystemCD3D.C:175-177)
  double Parameters[2] = {optd("omega", 1.0), optd("omega", 1.0)};
  TMultiGrid3D *MG = new TMultiGrid3D(1, 2, Parameters);
  // step-length control keeps the old iterate and defect in aux vectors 2, 3
  const int n_aux = (optd("slc_all", 0) != 0 || optd("slc_fine", 0) != 0) ? 4 : 2;
  std::vector<TAssembleMat3D *> asmb(levels);
  BoundCondFunct3D *BC[1] = {BoundCondFn};
  BoundValueFunct3D *BV[1] = {BoundValueFn};
  for (int i = 0; i < levels; i++)
  {
    TFESpace3D *fesp[1] = {L[i].space}, *ferhs[1] = {L[i].space};
    TSquareMatrix3D *SQ[1] = {L[i].A};
    double *RHS[1] = {L[i].rhs};
    TAuxParam3D *aux = new TAuxParam3D(1, 0, 0, 0, fesp, NULL, NULL, NULL, NULL, 0, NULL);
    asmb[i] = new TAssembleMat3D(1, fesp, 1, SQ, 0, NULL, 1, RHS, ferhs, form, BC, BV, aux);
    asmb[i]->Init();
    TMGLevel3D *lev = new TMGLevel3D(i, L[i].A, L[i].rhs, L[i].sol, n_aux, NULL);
    MG->AddLevel(lev);
  }

  // repeat=R: the timing mode of the benchmark.  The hierarchy above is built
  // once; then warmup=W untimed and R timed repetitions of Assemble() of all
  // levels + Solve() from the zero start vector, each bracketed as
  // CD3D_ParMooN.C:418-463 brackets them.  With start_file given, the timed
  // repetitions begin once that file exists (concurrent copies start together).
  const int repeat = (int)optd("repeat", 0);
  if (repeat > 0)
  {
    const int warm = (int)optd("warmup", 0);
    const std::string start = opts("start_file", "");
    const int top = levels - 1, N = L[top].N;
    TItMethod *prec = new TMultiGridScaIte(MatVect_Scalar, Defect_Scalar, NULL, 0, N, MG, 1);
    TItMethod *itm = new TFgmresIte(MatVect_Scalar, Defect_Scalar, prec, 0, N, 1);
    TSquareMatrix *sq[1] = {L[top].A};
    std::vector<double> d(N);
    for (int k = 0; k < warm + repeat; k++)
    {
      if (k == warm)
      {
        if (!start.empty())
        {
          dumpScalar("ready_epoch", epoch());
          fflush(g_meta);
          // bounded wait (one hour) for the go signal
          for (int w = 0; w < 360000; w++)
          {
            FILE *f = fopen(start.c_str(), "r");
            if (f) { fclose(f); break; }
            std::this_thread::sleep_for(std::chrono::milliseconds(10));
          }
        }
        dumpScalar("timed_start_epoch", epoch());
      }
      for (int i = 0; i < levels; i++) memset(L[i].sol, 0, sizeof(double) * L[i].N);
      double a = wall();
      for (int i = 0; i < levels; i++)
      {
        asmb[i]->Reset();
        asmb[i]->Assemble3D();
        int Na = L[i].space->GetActiveBound();
        memcpy(L[i].sol + Na, L[i].rhs + Na, (L[i].N - Na) * sizeof(double));
      }
      double b = wall();
      // Solve() through copies of sol / rhs: the finest MG level aliases the
      // level arrays (TSystemCD3D::Solve copies through Itmethod_sol / _rhs,
      // SystemCD3D.C:377-395)
      std::vector<double> isol(L[top].sol, L[top].sol + N), irhs(L[top].rhs, L[top].rhs + N);
      double r0, r1;
      ScalarDefect(L[top].A, isol.data(), irhs.data(), d.data(), r0);
      int iters = itm->Iterate(sq, NULL, isol.data(), irhs.data());
      memcpy(L[top].sol, isol.data(), sizeof(double) * N);
      double c = wall();
      ScalarDefect(L[top].A, isol.data(), irhs.data(), d.data(), r1);
      if (k >= warm)
      {
        char key[64];
        int j = k - warm;
        snprintf(key, sizeof key, "R%d_t_assemble", j); dumpScalar(key, b - a);
        snprintf(key, sizeof key, "R%d_t_solve", j); dumpScalar(key, c - b);
        snprintf(key, sizeof key, "R%d_iterations", j); dumpScalar(key, iters);
        snprintf(key, sizeof key, "R%d_rel_res", j); dumpScalar(key, r1 / r0);
      }
      printf("repetition %d: assemble %.3f s, solve %.3f s, %d iterations, |r|/|r0| = %.3e\n", k, b - a, c - b,
             iters, r1 / r0);
      fflush(stdout);
    }
    dumpScalar("timed_end_epoch", epoch());
    dumpScalar("fine_nnz", L[top].A->GetN_Entries());
    return 0;
  }

  // Assemble: TSystemCD3D::Assemble (SystemCD3D.C:340-365), timed per level
  std::vector<double> t_asm(levels);
  for (int i = 0; i < levels; i++)
  {
    double a = wall();
    asmb[i]->Reset();
    asmb[i]->Assemble3D();
    int Na = L[i].space->GetActiveBound();
    memcpy(L[i].sol + Na, L[i].rhs + Na, (L[i].N - Na) * sizeof(double));
    t_asm[i] = wall() - a;
  }

  bool do_dump = optd("dump", 1) != 0;
  if (do_dump)
    for (int i = 0; i < levels; i++) dump_level(i, L[i]);
  // parent of every cell of level i in level i-1's collection (the cell
  // itself when both levels share the mesh): what Prolongate walks
  if (do_dump)
    for (int i = 1; i < levels; i++)
    {
      TCollection *cc = L[i - 1].space->GetCollection(), *fc = L[i].space->GetCollection();
      int ncc = cc->GetN_Cells(), nfc = fc->GetN_Cells();
      for (int c = 0; c < ncc; c++) cc->GetCell(c)->SetClipBoard(c);
      std::vector<int> par(nfc);
      for (int c = 0; c < nfc; c++)
      {
        TBaseCell *cell = fc->GetCell(c);
        par[c] = cc == fc ? c : cell->GetParent()->GetClipBoard();
      }
      char k[64];
      snprintf(k, sizeof k, "L%d_parent", i);
      dump(k, par.data(), nfc, "i4");
    }
  for (int i = 0; i < levels; i++)
  {
    char k[64];
    snprintf(k, sizeof k, "L%d_t_assemble", i);
    dumpScalar(k, t_asm[i]);
  }
  dumpScalar("t_structure", t_struct);

  // transfer probes: Prolongate / DefectRestriction between each level pair
  if (do_dump && optd("transfer", 1) != 0)
  {
    for (int i = 1; i < levels; i++)
    {
      int Nc = L[i - 1].N, Nf = L[i].N;
      std::vector<double> c(Nc), f(Nf), d(Nf), r(Nc), aux(std::max(Nc, Nf) * 4 + 16);
      unsigned s = 12345u + i;
      for (int k = 0; k < Nc; k++) { s = s * 1664525u + 1013904223u; c[k] = (s >> 8) * (1.0 / 16777216.0) - 0.5; }
      for (int k = 0; k < Nf; k++) { s = s * 1664525u + 1013904223u; d[k] = (s >> 8) * (1.0 / 16777216.0) - 0.5; }
      char k1[64];
      snprintf(k1, sizeof k1, "T%d_", i);
      std::string pre(k1);
      dump(pre + "coarse_in", c.data(), Nc, "f8");
      dump(pre + "fine_in", d.data(), Nf, "f8");
      Prolongate(L[i - 1].space, L[i].space, c.data(), f.data(), aux.data());
      dump(pre + "prolongated", f.data(), Nf, "f8");
      std::vector<double> d2 = d;
      DefectRestriction(L[i - 1].space, L[i].space, r.data(), d2.data(), aux.data());
      dump(pre + "restricted", r.data(), Nc, "f8");
    }
  }

  if (optd("solve", 1) != 0)
  {
    int N = L[levels - 1].N;
    double *sol = L[levels - 1].sol, *rhs = L[levels - 1].rhs;
    TItMethod *prec = new TMultiGridScaIte(MatVect_Scalar, Defect_Scalar, NULL, 0, N, MG, 1);
    TItMethod *it = new TFgmresIte(MatVect_Scalar, Defect_Scalar, prec, 0, N, 1);
    std::vector<double> isol(sol, sol + N), irhs(rhs, rhs + N);
    TSquareMatrix *sq[1] = {L[levels - 1].A};
    // initial residual (FP64, full system incl. Dirichlet rows)
    std::vector<double> d(N);
    double r0;
    ScalarDefect(L[levels - 1].A, isol.data(), irhs.data(), d.data(), r0);
    double a = wall();
    int iters = it->Iterate(sq, NULL, isol.data(), irhs.data());
    double t_solve = wall() - a;
    double r1;
    ScalarDefect(L[levels - 1].A, isol.data(), irhs.data(), d.data(), r1);
    dumpScalar("solve_iterations", iters);
    dumpScalar("t_solve", t_solve);
    dumpScalar("res0", r0);
    dumpScalar("res_final", r1);
    if (do_dump || optd("dump_solution", 0) != 0) dump("solution", isol.data(), N, "f8");
    if (!do_dump && optd("dump_solution", 0) != 0)
    {
      // the finest level's dof positions, to compare with another dof numbering
      std::vector<double> x(N), y(N), z(N), xyz((size_t)N * 3);
      L[levels - 1].space->GetDOFPosition(x.data(), y.data(), z.data());
      for (int i = 0; i < N; i++) { xyz[3 * i] = x[i]; xyz[3 * i + 1] = y[i]; xyz[3 * i + 2] = z[i]; }
      dump("fine_dof_xyz", xyz.data(), (long)xyz.size(), "f8");
      dumpScalar("fine_active_bound", L[levels - 1].space->GetActiveBound());
    }
    printf("solve: %d iterations, %.3f s, |r|/|r0| = %.3e\n", iters, t_solve, r1 / r0);
  }
  for (int i = 0; i < levels; i++)
    printf("level %d: N=%d nnz=%d assemble %.4f s\n", i, L[i].N, L[i].A->GetN_Entries(), t_asm[i]);
  (void)Database; (void)FEDatabase;
  return 0;
}

// ----------------------------------------------------------------- tcd3d
// Replays the recorded amc.h run (ReadIn/tcd3d_GMG.out): Q1, Crank-Nicolson,
// Galerkin, printing L2 / H1-semi errors per step (TCD3D_ParMooN.C:565-).
static int run_tcd3d()
{
  int order = (int)optd("order", 1), levels = (int)optd("levels", 3);
  int coarse_steps = (int)optd("coarse_steps", 4 - ((int)optd("levels", 3) - 1));
  g_problem = 2;
  std::string dat = g_out + "/run.dat";
  write_dat(dat, order, levels, coarse_steps);
  TDatabase *Database = new TDatabase();
  TFEDatabase3D *FEDatabase = new TFEDatabase3D();
  TDomain *Domain = new TDomain((char *)dat.c_str());
  OpenFiles();
  TDatabase::ParamDB->INTERNAL_PROBLEM_LINEAR = (int)optd("linear_quad", 0);
  TDatabase::ParamDB->DISCTYPE = 1;
  TDatabase::ParamDB->ANSATZ_ORDER = order;
  set_solver_params();
  TDatabase::ParamDB->SC_LIN_RED_FACTOR_SCALAR = 0.0;
  TDatabase::ParamDB->SC_LIN_RES_NORM_MIN_SCALAR = optd("resmin", 1e-13);
  TDatabase::TimeDB->TIME_DISC = 2;
  TDatabase::TimeDB->TIMESTEPLENGTH = optd("tau", 1.082532e-01);
  TDatabase::TimeDB->CURRENTTIMESTEPLENGTH = TDatabase::TimeDB->TIMESTEPLENGTH;
  TDatabase::TimeDB->STARTTIME = 0;
  TDatabase::TimeDB->CURRENTTIME = 0;
  TDatabase::TimeDB->ENDTIME = optd("endtime", 0.3);
  Domain->Init(TDatabase::ParamDB->BNDFILE, TDatabase::ParamDB->GEOFILE);
  for (int i = 0; i < coarse_steps; i++) Domain->RegRefineAll();

  char Name[] = "u", Desc[] = "u", CStr[] = "C";
  TFESpace3D **spaces = new TFESpace3D *[levels];
  double **Sol = new double *[levels], **Rhs = new double *[levels];
  TFEFunction3D *u = NULL;
  int N = 0;
  for (int i = 0; i < levels; i++)
  {
    if (i) Domain->RegRefineAll();
    TCollection *coll = Domain->GetCollection(It_Finest, 0);
    spaces[i] = new TFESpace3D(coll, Name, Desc, BoundCondFn, order);
    N = spaces[i]->GetN_DegreesOfFreedom();
    Sol[i] = new double[N]();
    Rhs[i] = new double[N]();
    u = new TFEFunction3D(spaces[i], CStr, CStr, Sol[i], N);
  }
  double *sol = Sol[levels - 1], *rhs = Rhs[levels - 1];
  std::vector<double> oldrhs(N), oldsol(N);
  u->Interpolate(InitialFn);
  TSystemTCD3D *S = new TSystemTCD3D(levels, spaces, Sol, Rhs, 1, 1);
  S->Init(CoeffsFn, BoundCondFn, BoundValueFn, NULL);
  S->AssembleMRhs();
  memcpy(oldrhs.data(), rhs, N * sizeof(double));

  MultiIndex3D AllDer[4] = {D000, D100, D010, D001};
  TFESpace3D *fesp[1] = {spaces[levels - 1]};
  TAuxParam3D *aux = new TAuxParam3D(1, 0, 0, 0, fesp, NULL, NULL, NULL, NULL, 0, NULL);
  double errors[5];
  std::vector<double> times, l2, h1;
  auto measure = [&]() {
    for (int j = 0; j < 5; j++) errors[j] = 0;
    u->GetErrors(ExactFn, 4, AllDer, 2, L2H1Errors, CoeffsFn, aux, 1, fesp, errors);
    times.push_back(TDatabase::TimeDB->CURRENTTIME);
    l2.push_back(errors[0]);
    h1.push_back(errors[1]);
    printf("time: %.7e L2: %.7e H1-semi: %.7e\n", TDatabase::TimeDB->CURRENTTIME, errors[0], errors[1]);
  };
  measure();
  int m = 0;
  int nsub = GetN_SubSteps();
  double end_time = TDatabase::TimeDB->ENDTIME;
  double t_asm = 0, t_solve = 0;
  while (TDatabase::TimeDB->CURRENTTIME < end_time - 1e-12)
  {
    m++;
    for (int l = 0; l < nsub; l++)
    {
      SetTimeDiscParameters(1);
      memcpy(oldsol.data(), sol, N * sizeof(double));
      TDatabase::TimeDB->CURRENTTIME += TDatabase::TimeDB->CURRENTTIMESTEPLENGTH;
      double a = wall();
      S->AssembleARhs();
      S->AssembleSystMat(oldrhs.data(), oldsol.data(), rhs, sol);
      memcpy(oldrhs.data(), rhs, N * sizeof(double));
      t_asm += wall() - a;
      a = wall();
      S->Solve(sol);
      t_solve += wall() - a;
      S->RestoreMassMat();
    }
    measure();
  }
  dump("times", times.data(), (long)times.size(), "f8");
  dump("l2", l2.data(), (long)l2.size(), "f8");
  dump("h1", h1.data(), (long)h1.size(), "f8");
  dumpScalar("t_assemble_total", t_asm);
  dumpScalar("t_solve_total", t_solve);
  dumpScalar("steps", m);
  (void)Database; (void)FEDatabase;
  return 0;
}

int main(int argc, char **argv)
{
  if (argc < 3)
  {
    fprintf(stderr, "usage: %s cd3d|tcd3d <outdir> key=value...\n", argv[0]);
    return 1;
  }
  std::string mode = argv[1];
  g_out = argv[2];
  mkdir(g_out.c_str(), 0777);
  for (int i = 3; i < argc; i++)
  {
    std::string a = argv[i];
    size_t p = a.find('=');
    if (p != std::string::npos) g_opt[a.substr(0, p)] = a.substr(p + 1);
  }
  if (!g_opt.count("data"))
  {
    // default: the data directory next to the binary
    std::string self = argv[0];
    size_t p = self.rfind('/');
    g_opt["data"] = (p == std::string::npos ? std::string(".") : self.substr(0, p)) + "/data";
  }
  g_meta = fopen((g_out + "/meta.txt").c_str(), "w");
  int rc = 1;
  if (mode == "cd3d") rc = run_cd3d();
  else if (mode == "tcd3d") rc = run_tcd3d();
  else fprintf(stderr, "unknown mode %s\n", mode.c_str());
  fclose(g_meta);
  return rc;
}
