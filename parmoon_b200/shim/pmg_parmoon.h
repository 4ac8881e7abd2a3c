// pmg_parmoon.h -- drop-in replacement for ParMooN's scalar CD3D system class
// TSystemCD3D (include/System/SystemCD3D.h:121-135, src/System/SystemCD3D.C)
// on top of libpmg_b200.
//
// A ParMooN program keeps building its domain, FE spaces and arrays with the
// reference classes and swaps
//     SystemMatrix = new TSystemCD3D(mg_level, Scalar_FeSpaces, Sol_array, Rhs_array, DISCTYPE, SOLVER);
// for
//     SystemMatrix = new TPmgSystemCD3D(mg_level, Scalar_FeSpaces, Sol_array, Rhs_array, DISCTYPE, SOLVER);
// Init / Assemble / Solve keep their arguments and host-array semantics:
// Assemble() leaves every level's rhs, and the Dirichlet part of every level's
// solution, in Rhs_array / Sol_array; Solve(sol, rhs) writes the solution into
// sol.  Matrices, transfers and the V-cycle stay on the device; the CSR
// patterns are the reference's own (TSquareStructure3D + Sort), so
// CopyMatricesToHost() fills GetAMatrix()[i]->GetEntries() entry for entry.
//
// Coefficients: Init(BilinearCoeffs, ...) evaluates the host callback at the
// device's quadrature points on every Assemble (PMG_COEF_TABLE), so any
// CoeffFct3D works unchanged; the overload taking a pmg_coeff_desc lets the
// device evaluate a built-in field instead (no host work per assembly).
// DISCTYPE GALERKIN (1) and SDFEM/SUPG (2) are built; SOLVER must be GMG (1).
// The time-dependent surface of TSystemTCD3D is here as well; the reference's
// class names are provided by SystemCD3D_pmg.C / SystemTCD3D_pmg.C, which a
// program links instead of src/System/SystemCD3D.C / SystemTCD3D.C.
//
// Build inside a ParMooN tree (the reference headers on the include path,
// -D__3D__) and link libpmg_b200.so.
#pragma once
#include <FESpace3D.h>
#include <SquareMatrix3D.h>
#include <SquareStructure3D.h>
#include <AuxParam3D.h>
#include <Constants.h>
#include "../../include/pmg_b200.h"
#include <vector>

class TPmgSystemCD3D {
 public:
  TPmgSystemCD3D(int N_levels, TFESpace3D **fespaces, double **sol, double **rhs, int disctype, int solver);
  ~TPmgSystemCD3D();

  // TSystemCD3D::Init (SystemCD3D.C:253-337): the callback is evaluated on the host
  void Init(CoeffFct3D *BilinearCoeffs, BoundCondFunct3D *BoundCond, BoundValueFunct3D *BoundValue,
            TAuxParam3D *aux);
  // same, with the coefficients evaluated on the device from a built-in field
  void Init(CoeffFct3D *BilinearCoeffs, BoundCondFunct3D *BoundCond, BoundValueFunct3D *BoundValue,
            TAuxParam3D *aux, const pmg_coeff_desc &device_coeffs);

  // TSystemCD3D::Assemble (SystemCD3D.C:340-365)
  void Assemble();

  // TSystemCD3D::Solve (SystemCD3D.C:368-420), SOLVER = GMG with FGMRES
  void Solve(double *sol, double *rhs);

  // TSystemTCD3D surface (include/System/SystemTCD3D.h, SystemTCD3D.C:208-460):
  // mass and stiffness assembly at TDatabase::TimeDB->CURRENTTIME, the theta-
  // scheme system with THETA1..4 and CURRENTTIMESTEPLENGTH, and its solve
  void AssembleMRhs();
  void AssembleARhs();
  void AssembleSystMat(double *oldrhs, double *oldsol, double *rhs, double *sol);
  void RestoreMassMat();
  void Solve(double *sol);
  double GetResidual(double *sol);

  // device matrices into the TSquareMatrix3D objects, for code that reads GetEntries()
  void CopyMatricesToHost();
  TSquareMatrix3D **GetAMatrix() { return sqmatrixA.data(); }
  TSquareStructure3D **GetStructures() { return sqstructure.data(); }

  // PMG_OK, or the PMG_ERR_* code of the first failed device call (the
  // reference exits; a library caller decides)
  int GetLastStatus() const { return status; }
  const pmg_solve_stats &GetSolveStats() const { return stats; }
  pmg_handle GetHandle() const { return h; }

 private:
  int N_Levels, Disctype, status = PMG_OK;
  bool syst_assembled = false;
  std::vector<double> B;  // theta-scheme rhs of the last AssembleSystMat
  TFESpace3D **FeSpaces;
  double **SolArray, **RhsArray;
  CoeffFct3D *Coeffs = nullptr;
  BoundValueFunct3D *BoundValues = nullptr;
  pmg_coeff_desc dev_coeffs{};
  std::vector<double> dev_modes;
  struct DirichletNodes {
    std::vector<int> id;       // boundary component of each Dirichlet dof
    std::vector<double> xyz;   // its node
  };
  std::vector<DirichletNodes> dirichlet;
  std::vector<TSquareStructure3D *> sqstructure;
  std::vector<TSquareMatrix3D *> sqmatrixA;
  pmg_handle h = nullptr;
  pmg_solve_stats stats{};
  void check(int rc, const char *what);
  void setup(BoundValueFunct3D *BoundValue);
  void tabulate_coefficients();
  void assemble_form(int form);
  void update_dirichlet();
};

// the device system behind a TSystemCD3D / TSystemTCD3D of the link-time
// replacements (SystemCD3D_pmg.C); NULL for any other object
class TSystemCD3D;
TPmgSystemCD3D *PmgDeviceSystem(const TSystemCD3D *s);
// reference-style failure: print the library's message and exit(4711)
void PmgRequireOk(TPmgSystemCD3D *d, const char *where);
