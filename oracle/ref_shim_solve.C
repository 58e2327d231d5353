// Test infrastructure only: link stubs for the solver harness library
// (libcpsref_solve.so).  Each names a reference symbol whose defining file
// is not compiled (I/O, parallel transport, gauge force, the MIT zMobius
// preconditioners, the eigensolver entry points); none is reached by the
// harness's calls, and each aborts loudly if it ever is.
#include <config.h>
#include <util/data_types.h>
#include <util/dirac_op.h>
#include <util/lattice.h>
#include <util/pt.h>
#include <util/latrngio.h>
#include <util/ReadLatticePar.h>
#include <util/ReadU1LatticePar.h>
#include <util/zmobius.h>
#include <comms/glb.h>
#include <alg/do_arg.h>
#include <cstdio>
#include <cstdlib>

CPS_START_NAMESPACE
static void not_built(const char *w) {
  fprintf(stderr, "ref_shim_solve: %s is not part of the oracle build\n", w);
  abort();
}
int ParTrans::scope_lock = 0;
unsigned int local_checksum(Float *, int) { not_built("local_checksum"); return 0; }
int NumChkb(RitzMatType) { not_built("NumChkb"); return 0; }
ForceArg Gwilson::EvolveMomGforce(Matrix *, Float) { not_built("Gwilson::EvolveMomGforce"); return ForceArg(); }
void ReadLatticeParallel::read(Lattice &, const QioArg &) { not_built("ReadLatticeParallel::read"); }
void ReadU1LatticeParallel::read(Lattice &, const QioArg &) { not_built("ReadU1LatticeParallel::read"); }
LatRngRead::LatRngRead() {}
LatRngRead::~LatRngRead() {}
LatRngWrite::LatRngWrite() {}
LatRngWrite::~LatRngWrite() {}
void LatRngRead::read(UGrandomGenerator *, UGrandomGenerator *, const QioArg &) { not_built("LatRngRead::read"); }
void LatRngWrite::write(UGrandomGenerator *, UGrandomGenerator *, const QioArg &) { not_built("LatRngWrite::write"); }
bool DoArg::Decode(char *, char *) { not_built("DoArg::Decode"); return false; }
bool MdwfTuning::Decode(char *, char *) { not_built("MdwfTuning::Decode"); return false; }
bool MdwfTuning::Encode(char *, char *) { not_built("MdwfTuning::Encode"); return false; }
int DiracOp::InvLowModeApprox(std::vector<Vector *> &, std::vector<Vector *> &, char *, int) {
  not_built("DiracOp::InvLowModeApprox");
  return 0;
}
int DiracOp::InvEigCg(Vector *, Vector *, Float *, const int, const int, Vector **, const int, Float *, float **,
                      Rcomplex *, const int, const Float *, const int) {
  not_built("DiracOp::InvEigCg");
  return 0;
}
CPS_END_NAMESPACE
