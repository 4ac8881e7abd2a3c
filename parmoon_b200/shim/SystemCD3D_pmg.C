// Link-time replacement of src/System/SystemCD3D.C: the reference's class
// TSystemCD3D (include/System/SystemCD3D.h, unchanged) implemented on
// libpmg_b200 through TPmgSystemCD3D.  A ParMooN program such as
// 3DPrograms/CD3D_ParMooN.C compiles unmodified; linking this object (and
// pmg_parmoon.o, libpmg_b200.so) ahead of the ParMooN library makes its
// TSystemCD3D::{Init, Assemble, Solve} run on the B200.
//
// The reference's members keep their meaning where a subclass could read
// them (N_Levels, FeSpaces, SolArray, RhsArray, Disctype, SOLVER, N_DOF,
// sqstructure, sqmatrixA: the reference's own CSR structures, and matrices on
// them filled by TPmgSystemCD3D::CopyMatricesToHost); the device state lives in a
// TPmgSystemCD3D kept beside each object.  Errors end the program with
// exit(4711) as the reference's do (SystemCD3D.C:201-225, 302-305), after
// printing the library's message.
#include <SystemCD3D.h>
#include <Database.h>
#include <MooNMD_Io.h>
#include "pmg_parmoon.h"
#include <cstdlib>
#include <map>

static std::map<const TSystemCD3D *, TPmgSystemCD3D *> &device_systems() {
  static std::map<const TSystemCD3D *, TPmgSystemCD3D *> m;
  return m;
}

TPmgSystemCD3D *PmgDeviceSystem(const TSystemCD3D *s) {
  auto it = device_systems().find(s);
  return it == device_systems().end() ? nullptr : it->second;
}

static TPmgSystemCD3D *device_of(const TSystemCD3D *s) { return PmgDeviceSystem(s); }

void PmgRequireOk(TPmgSystemCD3D *d, const char *where) {
  if (d->GetLastStatus() != PMG_OK) {
    OutPut(where << " (B200): " << pmg_last_error() << endl);
    exit(4711);
  }
}

static void require_ok(TPmgSystemCD3D *d, const char *where) { PmgRequireOk(d, where); }

TSystemCD3D::TSystemCD3D(int N_levels, TFESpace3D **fespaces, double **sol, double **rhs, int disctype, int solver) {
  N_Levels = N_levels;
  FeSpaces = fespaces;
  SolArray = sol;
  RhsArray = rhs;
  Disctype = disctype;
  SOLVER = solver;
  Start_Level = 0;
  N_Matrices = 1;
  N_DOF = FeSpaces[N_Levels - 1]->GetN_DegreesOfFreedom();
  if (solver != GMG) {
    OutPut("TSystemCD3D (B200): only SOLVER_TYPE = GMG is built" << endl);
    exit(4711);
  }
  TPmgSystemCD3D *d = new TPmgSystemCD3D(N_levels, fespaces, sol, rhs, disctype, solver);
  require_ok(d, "TSystemCD3D::TSystemCD3D");
  device_systems()[this] = d;
  sqstructure = d->GetStructures();
  sqmatrixA = d->GetAMatrix();
  sqmatrices = (TSquareMatrix **)SQMATRICES;
  SQMATRICES[0] = sqmatrixA[N_Levels - 1];
  AMatRhsAssemble = nullptr;
  MG = nullptr;
  MGLevel = nullptr;
  Itmethod = prec = nullptr;
  Itmethod_sol = Itmethod_rhs = nullptr;
  DiscreteFormARhs = nullptr;
}

TSystemCD3D::~TSystemCD3D() {
  TPmgSystemCD3D *d = device_of(this);
  device_systems().erase(this);
  delete d;
}

void TSystemCD3D::Init(CoeffFct3D *BilinearCoeffs, BoundCondFunct3D *BoundCond, BoundValueFunct3D *BoundValue,
                       TAuxParam3D *aux) {
  BoundaryConditions[0] = BoundCond;
  BoundaryValues[0] = BoundValue;
  TPmgSystemCD3D *d = device_of(this);
  d->Init(BilinearCoeffs, BoundCond, BoundValue, aux);
  require_ok(d, "TSystemCD3D::Init");
}

void TSystemCD3D::Assemble() {
  TPmgSystemCD3D *d = device_of(this);
  d->Assemble();
  require_ok(d, "TSystemCD3D::Assemble");
}

void TSystemCD3D::Solve(double *sol, double *rhs) {
  TPmgSystemCD3D *d = device_of(this);
  d->Solve(sol, rhs);
  require_ok(d, "TSystemCD3D::Solve");
}
