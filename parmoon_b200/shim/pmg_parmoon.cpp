// TPmgSystemCD3D: the reference's TSystemCD3D surface on libpmg_b200 (see pmg_parmoon.h).
#include "pmg_parmoon.h"
#include "../../include/pmg_mesh.h"
#include <Database.h>
#include <FEDatabase3D.h>
#include <Collection.h>
#include <BaseCell.h>
#include <Vertex.h>
#include <FE3D.h>
#include <FEDesc3D.h>
#include <Joint.h>
#include <BoundFace.h>
#include <BoundComp3D.h>
#include <cmath>
#include <cstdio>
#include <cstring>

void TPmgSystemCD3D::check(int rc, const char *what) {
  if (rc != PMG_OK && status == PMG_OK) {
    status = rc;
    fprintf(stderr, "TPmgSystemCD3D: %s failed (%d): %s\n", what, rc, pmg_last_error());
  }
}

TPmgSystemCD3D::TPmgSystemCD3D(int N_levels, TFESpace3D **fespaces, double **sol, double **rhs, int disctype,
                               int solver)
    : N_Levels(N_levels), Disctype(disctype), FeSpaces(fespaces), SolArray(sol), RhsArray(rhs) {
  if (solver != GMG) check(PMG_ERR_UNSUPPORTED, "TPmgSystemCD3D: SOLVER must be GMG");
  if (disctype != GALERKIN && disctype != SDFEM) check(PMG_ERR_UNSUPPORTED, "TPmgSystemCD3D: DISCTYPE");
  // the reference's per-level CSR structure (SystemCD3D.C:106-126)
  for (int i = 0; i < N_Levels; i++) {
    TSquareStructure3D *st = new TSquareStructure3D(FeSpaces[i]);
    st->Sort();
    sqstructure.push_back(st);
    sqmatrixA.push_back(new TSquareMatrix3D(st));
  }
  // solver knobs from TDatabase::ParamDB (Database.C:660-780)
  pmg_params p;
  // a program built against another revision of pmg_b200.h: rebuild it
  if (pmg_params_size() != (int)sizeof(pmg_params)) {
    check(PMG_ERR_ARG, "pmg_params_size (libpmg_b200 and this program disagree on sizeof(pmg_params))");
    return;  // no handle: every later call reports the status
  }
  pmg_default_params(&p);
  TParamDB *db = TDatabase::ParamDB;
  // 1 Jacobi, 2 SOR, 3 SSOR; the sequential reference runs SOR for the codes
  // its switch does not list (MultiGrid3D.C:210-213, 430-440); ILU (4) is not
  // built here and pmg_create rejects it
  {
    const int sm = db->SC_SMOOTHER_SCALAR;
    p.smoother = (sm >= 1 && sm <= 4) ? sm : PMG_SMOOTHER_SOR;
    const int cs = db->SC_COARSE_SMOOTHER_SCALAR;
    // unlisted coarse smoothers run SSOR (MultiGrid3D.C:320-327)
    p.coarse_smoother = (cs >= 1 && cs <= 4) || cs == PMG_COARSE_DIRECT ? cs : PMG_COARSE_SSOR;
  }
  p.slc_all = db->SC_STEP_LENGTH_CONTROL_ALL_SCALAR != 0;
  p.slc_fine = db->SC_STEP_LENGTH_CONTROL_FINE_SCALAR != 0;
  p.pre_smooth = db->SC_PRE_SMOOTH_SCALAR;
  p.post_smooth = db->SC_POST_SMOOTH_SCALAR;
  p.coarse_maxit = db->SC_COARSE_MAXIT_SCALAR;
  p.coarse_red = db->SC_COARSE_RED_FACTOR_SCALAR;
  p.smooth_omega = db->SC_SMOOTH_DAMP_FACTOR_SCALAR;
  p.gmg_damp = db->SC_GMG_DAMP_FACTOR_SCALAR;
  p.lin_red = db->SC_LIN_RED_FACTOR_SCALAR;
  p.lin_res_min = db->SC_LIN_RES_NORM_MIN_SCALAR;
  p.lin_maxit = db->SC_LIN_MAXIT_SCALAR;
  p.restart = db->SC_GMRES_RESTART;
  p.div_factor = db->SC_DIV_FACTOR;
  p.sdfem_type = db->SDFEM_TYPE;
  p.delta0 = db->DELTA0;
  p.poly_degree = db->INTERNAL_POLYNOMIAL_DEGREE;
  p.problem_linear = db->INTERNAL_PROBLEM_LINEAR;
  p.reference_restart_rule = 1;
  check(pmg_create(&h, N_Levels, &p), "pmg_create");
}

TPmgSystemCD3D::~TPmgSystemCD3D() {
  if (h) pmg_destroy(h);
  for (auto *m : sqmatrixA) delete m;
  for (auto *s : sqstructure) delete s;
}

// patterns, meshes, Dirichlet values and transfers of every level
void TPmgSystemCD3D::setup(BoundValueFunct3D *BoundValue) {
  BoundValues = BoundValue;
  dirichlet.assign(N_Levels, DirichletNodes());
  std::vector<std::vector<int>> ed_lv(N_Levels);
  std::vector<std::vector<double>> cv_lv(N_Levels);
  std::vector<int> elem_lv(N_Levels, 0);
  for (int i = 0; i < N_Levels && status == PMG_OK; i++) {
    TFESpace3D *sp = FeSpaces[i];
    TCollection *coll = sp->GetCollection();
    const int nc = coll->GetN_Cells(), N = sp->GetN_DegreesOfFreedom(), Na = sp->GetActiveBound();
    if (sp->GetHangingBound() != Na) check(PMG_ERR_UNSUPPORTED, "hanging nodes");
    TSquareMatrix3D *A = sqmatrixA[i];
    check(pmg_set_level_csr(h, i, N, Na, A->GetRowPtr(), A->GetKCol()), "pmg_set_level_csr");
    // element -> dof map (GlobalNumbers + BeginIndex) and cell vertices
    int *gn = sp->GetGlobalNumbers(), *bi = sp->GetBeginIndex();
    const int nloc = bi[1] - bi[0];
    const int nv = coll->GetCell(0)->GetN_Vertices();
    // Q1 / Q2 / N_Q1 (the non-conforming levels of SC_MG_TYPE_SCALAR = 1) on
    // hexahedra, P1 / P2 on tetrahedra
    const int elem = nv == 8 ? (nloc == 8 ? PMG_ELEM_Q1_HEX : nloc == 6 ? PMG_ELEM_NQ1_HEX : PMG_ELEM_Q2_HEX)
                             : (nloc == 4 ? PMG_ELEM_P1_TET : PMG_ELEM_P2_TET);
    elem_lv[i] = elem;
    std::vector<int> &ed = ed_lv[i];
    std::vector<double> &cv = cv_lv[i];
    ed.resize((size_t)nc * nloc);
    cv.assign((size_t)nc * 24, 0.0);
    bool brick = nv == 8;
    for (int c = 0; c < nc; c++) {
      if (bi[c + 1] - bi[c] != nloc) check(PMG_ERR_UNSUPPORTED, "mixed elements");
      for (int l = 0; l < nloc; l++) ed[(size_t)c * nloc + l] = gn[bi[c] + l];
      TBaseCell *cell = coll->GetCell(c);
      double *v = &cv[(size_t)c * 24];
      for (int k = 0; k < nv; k++) cell->GetVertex(k)->GetCoords(v[3 * k], v[3 * k + 1], v[3 * k + 2]);
      if (nv == 8)  // axis-aligned box: each coordinate takes at most two values over the 8 vertices
        for (int d = 0; d < 3; d++) {
          double a = v[d], b = v[d];
          for (int k = 1; k < 8; k++) {
            const double x = v[3 * k + d];
            if (std::fabs(x - a) < 1e-12 || std::fabs(x - b) < 1e-12) continue;
            if (b == a) b = x;
            else brick = false;
          }
        }
    }
    check(pmg_set_level_mesh(h, i, elem, nc, ed.data(), cv.data(), brick ? 1 : 0), "pmg_set_level_mesh");
    // Dirichlet values: BoundValue(Bd_ID, node) at the dof nodes of every boundary
    // face, Bd_ID the face's boundary component (AssembleMat3D.C:1020-1081)
    std::vector<double> X(N), Y(N), Z(N);
    std::vector<int> bd_id(N - Na, 0);
    sp->GetDOFPosition(X.data(), Y.data(), Z.data());
    for (int c = 0; c < nc; c++) {
      TBaseCell *cell = coll->GetCell(c);
      TFEDesc3D *desc = TFEDatabase3D::GetFE3D(sp->GetFE3D(c, cell))->GetFEDesc3D();
      const int njd = desc->GetN_JointDOF();
      for (int j = 0; j < cell->GetN_Joints(); j++) {
        TJoint *joint = cell->GetJoint(j);
        if (joint->GetType() != BoundaryFace && joint->GetType() != IsoBoundFace) continue;
        const int id = ((TBoundFace *)joint)->GetBoundComp()->GetID();
        const int *jd = desc->GetJointDOF(j);
        for (int k = 0; k < njd; k++) {
          const int dof = gn[bi[c] + jd[k]];
          if (dof >= Na) bd_id[dof - Na] = id;
        }
      }
    }
    DirichletNodes &dn = dirichlet[i];
    dn.id = bd_id;
    dn.xyz.resize((size_t)3 * (N - Na));
    for (int d = Na; d < N; d++) {
      dn.xyz[3 * (size_t)(d - Na)] = X[d];
      dn.xyz[3 * (size_t)(d - Na) + 1] = Y[d];
      dn.xyz[3 * (size_t)(d - Na) + 2] = Z[d];
    }
    if (i == 0 || status != PMG_OK) continue;
    // prolongation from level i-1: the coarse basis of each fine cell's parent
    // evaluated at the fine dofs (Prolongate, MGComponents3D.C:208-488)
    TCollection *ccoll = FeSpaces[i - 1]->GetCollection();
    const int ncc = ccoll->GetN_Cells(), Nc = FeSpaces[i - 1]->GetN_DegreesOfFreedom();
    std::vector<int> saved(ncc);
    for (int c = 0; c < ncc; c++) {
      saved[c] = ccoll->GetCell(c)->GetClipBoard();
      ccoll->GetCell(c)->SetClipBoard(c);
    }
    // the coarse cell of every fine cell: its parent, or the cell itself when
    // both spaces live on one mesh (the conforming level above the N_Q1 levels)
    const bool same_mesh = ccoll == coll;
    std::vector<int> owner(N, -1), par(nc, -1);
    for (int c = 0; c < nc; c++) {
      TBaseCell *parent = same_mesh ? coll->GetCell(c) : coll->GetCell(c)->GetParent();
      const int pc = parent ? parent->GetClipBoard() : -1;
      if (pc < 0 || pc >= ncc || ccoll->GetCell(pc) != parent) {
        check(PMG_ERR_ARG, "levels are not nested (fine cell without a parent on the coarser level)");
        break;
      }
      par[c] = pc;
      for (int l = 0; l < nloc; l++) owner[ed[(size_t)c * nloc + l]] = pc;
    }
    for (int c = 0; c < ncc; c++) ccoll->GetCell(c)->SetClipBoard(saved[c]);
    if (status != PMG_OK) continue;
    if (elem_lv[i - 1] != elem || elem == PMG_ELEM_NQ1_HEX) {
      // different spaces, or the non-conforming N_Q1: Prolongate's cell average
      std::vector<int> prp(N + 1);
      check(pmg_cell_prolongation(elem_lv[i - 1], ncc, ed_lv[i - 1].data(), cv_lv[i - 1].data(), Nc, elem, nc,
                                  ed.data(), cv.data(), par.data(), N, prp.data(), nullptr, nullptr),
            "pmg_cell_prolongation");
      std::vector<int> pcol(prp[N]);
      std::vector<double> pval(prp[N]);
      check(pmg_cell_prolongation(elem_lv[i - 1], ncc, ed_lv[i - 1].data(), cv_lv[i - 1].data(), Nc, elem, nc,
                                  ed.data(), cv.data(), par.data(), N, prp.data(), pcol.data(), pval.data()),
            "pmg_cell_prolongation");
      check(pmg_set_transfer(h, i, N, Nc, prp.data(), pcol.data(), pval.data()), "pmg_set_transfer");
      continue;
    }
    std::vector<double> xyz((size_t)3 * N);
    for (int d = 0; d < N; d++) { xyz[3 * d] = X[d]; xyz[3 * d + 1] = Y[d]; xyz[3 * d + 2] = Z[d]; }
    std::vector<int> prp(N + 1);
    check(pmg_nested_prolongation(elem, ncc, ed_lv[i - 1].data(), cv_lv[i - 1].data(), Nc, N, xyz.data(),
                                  owner.data(), prp.data(), nullptr, nullptr), "pmg_nested_prolongation");
    std::vector<int> pcol(prp[N]);
    std::vector<double> pval(prp[N]);
    check(pmg_nested_prolongation(elem, ncc, ed_lv[i - 1].data(), cv_lv[i - 1].data(), Nc, N, xyz.data(),
                                  owner.data(), prp.data(), pcol.data(), pval.data()), "pmg_nested_prolongation");
    check(pmg_set_transfer(h, i, N, Nc, prp.data(), pcol.data(), pval.data()), "pmg_set_transfer");
  }
}

// BoundValue at every level's Dirichlet nodes, re-evaluated before every
// assembly as Assemble3D does (time-dependent boundary data included)
void TPmgSystemCD3D::update_dirichlet() {
  for (int i = 0; i < N_Levels && status == PMG_OK; i++) {
    const DirichletNodes &dn = dirichlet[i];
    const size_t nd = dn.id.size();
    if (nd == 0) continue;
    std::vector<double> dv(nd);
    for (size_t d = 0; d < nd; d++)
      BoundValues(dn.id[d], dn.xyz[3 * d], dn.xyz[3 * d + 1], dn.xyz[3 * d + 2], dv[d]);
    check(pmg_set_dirichlet_values(h, i, dv.data()), "pmg_set_dirichlet_values");
  }
}

void TPmgSystemCD3D::Init(CoeffFct3D *BilinearCoeffs, BoundCondFunct3D *, BoundValueFunct3D *BoundValue,
                          TAuxParam3D *) {
  if (status != PMG_OK) return;
  Coeffs = BilinearCoeffs;
  pmg_coeff_desc c{};
  c.kind = PMG_COEF_TABLE;
  check(pmg_set_coefficients(h, &c), "pmg_set_coefficients");
  setup(BoundValue);
}

void TPmgSystemCD3D::Init(CoeffFct3D *, BoundCondFunct3D *, BoundValueFunct3D *BoundValue, TAuxParam3D *,
                          const pmg_coeff_desc &device_coeffs) {
  if (status != PMG_OK) return;
  Coeffs = nullptr;
  dev_coeffs = device_coeffs;
  if (device_coeffs.modes && device_coeffs.n_modes > 0)
    dev_modes.assign(device_coeffs.modes, device_coeffs.modes + 8 * (size_t)device_coeffs.n_modes);
  dev_coeffs.modes = dev_modes.empty() ? nullptr : dev_modes.data();
  check(pmg_set_coefficients(h, &dev_coeffs), "pmg_set_coefficients");
  setup(BoundValue);
}

// the CoeffFct3D callback at every cell's quadrature points, one call per
// cell as TDiscreteForm3D::GetLocalForms makes it (DiscreteForm3D.C:264)
void TPmgSystemCD3D::tabulate_coefficients() {
  for (int i = 0; i < N_Levels && status == PMG_OK; i++) {
    int nq = 0;
    check(pmg_quad_points(h, i, &nq, nullptr), "pmg_quad_points");
    const int nc = FeSpaces[i]->GetCollection()->GetN_Cells();
    std::vector<double> xyz((size_t)nc * nq * 3), tab((size_t)nc * nq * 6);
    check(pmg_quad_points(h, i, &nq, xyz.data()), "pmg_quad_points");
    if (status != PMG_OK) return;
    std::vector<double> X(nq), Y(nq), Z(nq), store((size_t)nq * 20), pstore((size_t)nq * 4, 0.0);
    std::vector<double *> coeff(nq), param(nq);
    for (int q = 0; q < nq; q++) {
      coeff[q] = &store[(size_t)q * 20];
      param[q] = &pstore[(size_t)q * 4];
    }
    for (int c = 0; c < nc; c++) {
      for (int q = 0; q < nq; q++) {
        X[q] = xyz[((size_t)c * nq + q) * 3];
        Y[q] = xyz[((size_t)c * nq + q) * 3 + 1];
        Z[q] = xyz[((size_t)c * nq + q) * 3 + 2];
      }
      std::fill(store.begin(), store.end(), 0.0);
      Coeffs(nq, X.data(), Y.data(), Z.data(), param.data(), coeff.data());
      for (int q = 0; q < nq; q++)
        std::memcpy(&tab[((size_t)c * nq + q) * 6], coeff[q], 6 * sizeof(double));
    }
    check(pmg_set_coefficient_table(h, i, tab.data()), "pmg_set_coefficient_table");
  }
}

// assemble one form on every level; rhs of every level and the Dirichlet part
// of every level's solution back to the host arrays (SystemCD3D.C:340-365)
void TPmgSystemCD3D::assemble_form(int form) {
  if (status != PMG_OK) return;
  update_dirichlet();
  if (Coeffs) {
    tabulate_coefficients();
  } else {
    // built-in fields read the time from the descriptor
    dev_coeffs.t = TDatabase::TimeDB->CURRENTTIME;
    check(pmg_set_coefficients(h, &dev_coeffs), "pmg_set_coefficients");
  }
  if (status != PMG_OK) return;
  check(pmg_assemble(h, -1, form, nullptr, nullptr), "pmg_assemble");
  for (int i = 0; i < N_Levels && status == PMG_OK; i++) {
    const int N = FeSpaces[i]->GetN_DegreesOfFreedom(), Na = FeSpaces[i]->GetActiveBound();
    check(pmg_get_rhs(h, i, RhsArray[i]), "pmg_get_rhs");
    // set rhs for Dirichlet nodes (SystemCD3D.C:361)
    std::memcpy(SolArray[i] + Na, RhsArray[i] + Na, (size_t)(N - Na) * sizeof(double));
  }
}

void TPmgSystemCD3D::Assemble() { assemble_form(Disctype == SDFEM ? PMG_FORM_SUPG : PMG_FORM_GALERKIN); }

// TSystemTCD3D::AssembleMRhs (SystemTCD3D.C:208-232): M and f(t) on every level
void TPmgSystemCD3D::AssembleMRhs() { assemble_form(Disctype == SDFEM ? PMG_FORM_MASS_SUPG : PMG_FORM_MASS); }

// TSystemTCD3D::AssembleARhs (SystemTCD3D.C:235-257): A and f(t) on every level
void TPmgSystemCD3D::AssembleARhs() {
  if (syst_assembled) {
    check(PMG_ERR_STATE, "AssembleARhs: the system matrix is assembled; call RestoreMassMat first");
    return;
  }
  assemble_form(Disctype == SDFEM ? PMG_FORM_SUPG : PMG_FORM_GALERKIN);
}

// TSystemTCD3D::AssembleSystMat (SystemTCD3D.C:260-326); rhs is the finest
// level's f(t_new) of the last AssembleARhs, which the device holds
void TPmgSystemCD3D::AssembleSystMat(double *oldrhs, double *oldsol, double *rhs, double *sol) {
  if (status != PMG_OK) return;
  const int F = N_Levels - 1;
  const int N = FeSpaces[F]->GetN_DegreesOfFreedom(), Na = FeSpaces[F]->GetActiveBound();
  const double tau = TDatabase::TimeDB->CURRENTTIMESTEPLENGTH;
  const double theta[4] = {TDatabase::TimeDB->THETA1, TDatabase::TimeDB->THETA2, TDatabase::TimeDB->THETA3,
                           TDatabase::TimeDB->THETA4};
  B.resize(N);
  check(pmg_tcd_system(h, tau, theta, oldrhs, oldsol, B.data()), "pmg_tcd_system");
  if (status != PMG_OK) return;
  // Dirichlet values into the start vector (SystemTCD3D.C:297-298)
  std::memcpy(sol + Na, rhs + Na, (size_t)(N - Na) * sizeof(double));
  syst_assembled = true;
}

// TSystemTCD3D::RestoreMassMat (SystemTCD3D.C:328-347)
void TPmgSystemCD3D::RestoreMassMat() {
  if (status != PMG_OK) return;
  check(pmg_tcd_restore(h), "pmg_tcd_restore");
  syst_assembled = false;
}

// TSystemTCD3D::Solve (SystemTCD3D.C:349-420): sol is the start vector, B the rhs
void TPmgSystemCD3D::Solve(double *sol) {
  if (status != PMG_OK) return;
  if (!syst_assembled) {
    check(PMG_ERR_STATE, "Solve: call AssembleSystMat first");
    return;
  }
  Solve(sol, nullptr);
}

// TSystemTCD3D::GetResidual (SystemTCD3D.C:423-460): |B - (M + tau theta1 A) sol|
double TPmgSystemCD3D::GetResidual(double *sol) {
  if (status != PMG_OK) return 0.0;
  if (!syst_assembled) {
    check(PMG_ERR_STATE, "GetResidual: assemble the system matrix first");
    return 0.0;
  }
  const int F = N_Levels - 1;
  std::vector<double> r(B.size());
  double norm = 0.0;
  check(pmg_defect(h, F, sol, B.data(), r.data(), &norm), "pmg_defect");
  return norm;
}

void TPmgSystemCD3D::Solve(double *sol, double *rhs) {
  if (status != PMG_OK) return;
  const int rc = pmg_solve(h, sol, rhs, &stats);
  if (rc == PMG_OK || rc == PMG_ERR_NOT_CONVERGED) {
    // the reference returns after SC_LIN_MAXIT_SCALAR iterations with the iterate it has
    if (rc != PMG_OK) fprintf(stderr, "TPmgSystemCD3D: no convergence in %d iterations\n", stats.iterations);
  } else {
    check(rc, "pmg_solve");
  }
}

void TPmgSystemCD3D::CopyMatricesToHost() {
  for (int i = 0; i < N_Levels && status == PMG_OK; i++)
    check(pmg_get_matrix(h, i, 0, sqmatrixA[i]->GetEntries()), "pmg_get_matrix");
}
