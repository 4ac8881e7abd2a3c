// Link-time replacement of src/System/SystemTCD3D.C: the reference's class
// TSystemTCD3D (include/System/SystemTCD3D.h, unchanged; derived from
// TSystemCD3D) on libpmg_b200.  Link together with SystemCD3D_pmg.o, whose
// TSystemCD3D constructor creates the device system this class drives:
// 3DPrograms/TCD3D_ParMooN.C then runs its time loop (AssembleMRhs, then per
// step AssembleARhs / AssembleSystMat / Solve / RestoreMassMat) on the B200
// without a source change.  M, A and the theta-scheme system stay on the
// device; Rhs_array / Sol_array receive what the reference leaves in them.
#include <SystemTCD3D.h>
#include <Database.h>
#include <MooNMD_Io.h>
#include "pmg_parmoon.h"
#include <cstdlib>

TSystemTCD3D::TSystemTCD3D(int N_levels, TFESpace3D **fespaces, double **sol, double **rhs, int disctype, int solver)
    : TSystemCD3D(N_levels, fespaces, sol, rhs, disctype, solver) {
  N_Matrices++;
  // host mirrors of M on the reference structures (filled on request only)
  sqmatrixM = new TSquareMatrix3D *[N_Levels];
  for (int i = 0; i < N_Levels; i++) sqmatrixM[i] = new TSquareMatrix3D(sqstructure[i]);
  MMatRhsAssemble = nullptr;
  DiscreteFormMRhs = DiscreteFormRhs = nullptr;
  B = new double[N_DOF];
  defect = new double[N_DOF];
  gamma = 0.;
  SystMatAssembled = FALSE;
  Values = NULL; KCol = NULL; Row = NULL; Symbolic = NULL; Numeric = NULL;
  UpdateStiffnessMat = FALSE;
  FirstTime = TRUE;
  factorize = true;
}

TSystemTCD3D::~TSystemTCD3D() {
  for (int i = 0; i < N_Levels; i++) delete sqmatrixM[i];
  delete[] sqmatrixM;
  delete[] B;
  delete[] defect;
}

void TSystemTCD3D::Init(CoeffFct3D *BilinearCoeffs, BoundCondFunct3D *BoundCond, BoundValueFunct3D *BoundValue,
                        TAuxParam3D *aux) {
  BoundaryConditions[0] = BoundCond;
  BoundaryValues[0] = BoundValue;
  TPmgSystemCD3D *d = PmgDeviceSystem(this);
  d->Init(BilinearCoeffs, BoundCond, BoundValue, aux);
  PmgRequireOk(d, "TSystemTCD3D::Init");
}

void TSystemTCD3D::AssembleMRhs() {
  TPmgSystemCD3D *d = PmgDeviceSystem(this);
  d->AssembleMRhs();
  PmgRequireOk(d, "TSystemTCD3D::AssembleMRhs");
}

void TSystemTCD3D::AssembleARhs() {
  TPmgSystemCD3D *d = PmgDeviceSystem(this);
  d->AssembleARhs();
  PmgRequireOk(d, "TSystemTCD3D::AssembleARhs");
}

void TSystemTCD3D::AssembleSystMat(double *oldrhs, double *oldsol, double *rhs, double *sol) {
  if (SystMatAssembled) {
    OutPut("System is has to be restored before calling AssembleSystMat! " << endl);
    exit(0);
  }
  TPmgSystemCD3D *d = PmgDeviceSystem(this);
  d->AssembleSystMat(oldrhs, oldsol, rhs, sol);
  PmgRequireOk(d, "TSystemTCD3D::AssembleSystMat");
  gamma = TDatabase::TimeDB->CURRENTTIMESTEPLENGTH * TDatabase::TimeDB->THETA1;
  SystMatAssembled = TRUE;
}

void TSystemTCD3D::RestoreMassMat() {
  if (!SystMatAssembled) {
    cout << "System is not assembled to restore " << endl;
    exit(0);
  }
  TPmgSystemCD3D *d = PmgDeviceSystem(this);
  d->RestoreMassMat();
  PmgRequireOk(d, "TSystemTCD3D::RestoreMassMat");
  gamma = 0.;
  SystMatAssembled = FALSE;
}

void TSystemTCD3D::Solve(double *sol) {
  TPmgSystemCD3D *d = PmgDeviceSystem(this);
  d->Solve(sol);
  PmgRequireOk(d, "TSystemTCD3D::Solve");
}

double TSystemTCD3D::GetResidual(double *sol) {
  if (!SystMatAssembled) {
    OutPut("Assemble the System Matrix before calculating the GetResidual" << endl);
    exit(4711);
  }
  TPmgSystemCD3D *d = PmgDeviceSystem(this);
  const double r = d->GetResidual(sol);
  PmgRequireOk(d, "TSystemTCD3D::GetResidual");
  return r;
}
