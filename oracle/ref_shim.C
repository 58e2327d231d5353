// Test infrastructure only: definitions the reference kernels link against
// but which live in reference files that cannot be compiled without the
// whole library (Lattice, VML file decoding).  None of these is executed on
// the kernel paths the harness calls; each fails loudly if it ever is.
#include <config.h>
#include <util/data_types.h>
#include <util/dirac_op.h>
#include <util/vector.h>
#include <alg/do_arg.h>
#include <alg/cg_arg.h>
#include <util/zmobius.h>
#include <util/random.h>
#include <comms/glb.h>
#include <cstdio>
#include <cstdlib>

CPS_START_NAMESPACE
// static flop counter of DiracOp (include/util/dirac_op.h:71)
IntFlopCounter DiracOp::CGflops = 0;

bool DoArg::Decode(char *, char *) { fprintf(stderr, "ref_shim: DoArg::Decode\n"); abort(); }
bool MdwfTuning::Decode(char *, char *) { fprintf(stderr, "ref_shim: MdwfTuning::Decode\n"); abort(); }
void ReflectAndMultGamma5(Vector *, const Vector *, int, int) {
  fprintf(stderr, "ref_shim: ReflectAndMultGamma5\n");
  abort();
}
// MIT-variant preconditioners (defined in d_op_zmobius/d_op_zmobius.C);
// only the ZMOB_PC_*_MIT branches of zmobius_m/zmobius_mdag call them.
void zmobius_B_MIT(Vector *, Float, int, Zmobus *, Complex *, Complex *) {
  fprintf(stderr, "ref_shim: zmobius_B_MIT\n");
  abort();
}
void zmobius_Binv_MIT(Vector *, Float, int, Zmobus *, Complex *, Complex *) {
  fprintf(stderr, "ref_shim: zmobius_Binv_MIT\n");
  abort();
}
// eigen_solver.C's Lanczos / Ritz helpers (not the dense eigen_solver the
// harness calls) reference the lattice random generator and slice sums.
void slice_sum(Float *, int, int) {
  fprintf(stderr, "ref_shim: slice_sum\n");
  abort();
}
LatRanGen::LatRanGen() {}
LatRanGen::~LatRanGen() {}
void LatRanGen::SetSigma(IFloat) {
  fprintf(stderr, "ref_shim: LatRanGen::SetSigma\n");
  abort();
}
IFloat LatRanGen::Grand(FermionFieldDimension) {
  fprintf(stderr, "ref_shim: LatRanGen::Grand\n");
  abort();
}
LatRanGen LRG;
CPS_END_NAMESPACE
