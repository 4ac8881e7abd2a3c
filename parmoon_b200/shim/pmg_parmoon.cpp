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
  pmg_default_params(&p);
  TParamDB *db = TDatabase::ParamDB;
  p.smoother = db->SC_SMOOTHER_SCALAR == 1 ? PMG_SMOOTHER_JACOBI : PMG_SMOOTHER_SSOR;
  p.pre_smooth = db->SC_PRE_SMOOTH_SCALAR;
  p.post_smooth = db->SC_POST_SMOOTH_SCALAR;
  p.coarse_smoother = db->SC_COARSE_SMOOTHER_SCALAR == PMG_COARSE_DIRECT ? PMG_COARSE_DIRECT : PMG_COARSE_SSOR;
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
  std::vector<std::vector<int>> ed_lv(N_Levels);
  std::vector<std::vector<double>> cv_lv(N_Levels);
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
    const int elem = nv == 8 ? (nloc == 8 ? PMG_ELEM_Q1_HEX : PMG_ELEM_Q2_HEX)
                             : (nloc == 4 ? PMG_ELEM_P1_TET : PMG_ELEM_P2_TET);
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
    std::vector<double> X(N), Y(N), Z(N), dv(N - Na);
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
    for (int d = Na; d < N; d++) BoundValue(bd_id[d - Na], X[d], Y[d], Z[d], dv[d - Na]);
    if (N > Na) check(pmg_set_dirichlet_values(h, i, dv.data()), "pmg_set_dirichlet_values");
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
    std::vector<int> owner(N, -1);
    for (int c = 0; c < nc; c++) {
      TBaseCell *parent = coll->GetCell(c)->GetParent();
      const int pc = parent ? parent->GetClipBoard() : -1;
      if (pc < 0 || pc >= ncc || ccoll->GetCell(pc) != parent) {
        check(PMG_ERR_ARG, "levels are not nested (fine cell without a parent on the coarser level)");
        break;
      }
      for (int l = 0; l < nloc; l++) owner[ed[(size_t)c * nloc + l]] = pc;
    }
    for (int c = 0; c < ncc; c++) ccoll->GetCell(c)->SetClipBoard(saved[c]);
    if (status != PMG_OK) continue;
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
  check(pmg_set_coefficients(h, &device_coeffs), "pmg_set_coefficients");
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

void TPmgSystemCD3D::Assemble() {
  if (status != PMG_OK) return;
  if (Coeffs) tabulate_coefficients();
  if (status != PMG_OK) return;
  check(pmg_assemble(h, -1, Disctype == SDFEM ? PMG_FORM_SUPG : PMG_FORM_GALERKIN, nullptr, nullptr), "pmg_assemble");
  for (int i = 0; i < N_Levels && status == PMG_OK; i++) {
    const int N = FeSpaces[i]->GetN_DegreesOfFreedom(), Na = FeSpaces[i]->GetActiveBound();
    check(pmg_get_rhs(h, i, RhsArray[i]), "pmg_get_rhs");
    // set rhs for Dirichlet nodes (SystemCD3D.C:361)
    std::memcpy(SolArray[i] + Na, RhsArray[i] + Na, (size_t)(N - Na) * sizeof(double));
  }
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
