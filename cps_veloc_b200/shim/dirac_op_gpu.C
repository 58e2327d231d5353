// The CPS-side shim: the Krylov solve of every DiracOp on the GPU.
//
// Compiled into a CPS build (against CPS's own headers, linked with
// libcpsgpu.so), this file provides DiracOp::InvCgShift
// (d_op_base/comsrc/inv_cg.C:84-448) in place of the reference's: the CG on
// MatPcDagMatPc (+ shift) of the DiracOp in scope runs on the GPU through the
// C ABI (include/cpsgpu.h), with the reference's argument meanings and
// return convention (iterations + 1; *true_res = |src - A sol| / |src|).
// Every caller of InvCg — DiracOp*::MatInv, FmatEvlInv, the force solves —
// then solves on the GPU with its own preconditioning and reconstruction
// left unchanged.  It provides DiracOp::MInvCG (d_op_base/noarch/minvcg.C:
// 47-353) the same way: the multishift CG of FmatEvlMInv and the RHMC
// integrators (the FP32 recurrences with an FP64 refinement of every shift
// under CPSGPU_INNER=single|half).  The reference's InvCgShift and MInvCG
// symbols are removed from their objects (made weak) when they are linked
// together.
//
// What it reads from CPS: the lattice geometry and boundary conditions
// (GJP), the fermion class of the lattice (Lattice::Fclass), the DiracOp's
// CgArg (mass, stop_rsd, max_num_iter) and the gauge field, which while a
// DiracOp is alive is in WILSON order with the BondCond signs applied
// (dirac_op_base.C:95-164).  CPSGPU_INNER=single|half in the environment
// selects a mixed-precision solve (default FP64, as the reference).
#include <config.h>
#include <util/dirac_op.h>
#include <util/error.h>
#include <util/gjp.h>
#include <util/lattice.h>
#include <util/vector.h>
#include <alg/cg_arg.h>

#include <cstdlib>
#include <cstring>

#include <cpsgpu.h>

CPS_START_NAMESPACE

namespace {
cpsgpu_lattice g_lat = nullptr;
cpsgpu_dirac g_op = nullptr;
int g_sites[4] = {0, 0, 0, 0};
cpsgpu_dirac_arg g_arg;

void die(const char *fname) { ERR.General("DiracOp", fname, "cpsgpu: %s\n", cpsgpu_last_error()); }

// the device operator of the DiracOp in scope (rebuilt when the geometry
// or the parameters change) with the gauge field the DiracOp holds now
cpsgpu_dirac device_op(Lattice &lat, const CgArg *arg) {
  const int sites[4] = {GJP.XnodeSites(), GJP.YnodeSites(), GJP.ZnodeSites(), GJP.TnodeSites()};
  if (!g_lat || std::memcmp(sites, g_sites, sizeof(sites)) != 0) {
    if (g_op) cpsgpu_dirac_destroy(g_op);
    if (g_lat) cpsgpu_lattice_destroy(g_lat);
    g_op = nullptr;
    int bc[4];
    for (int mu = 0; mu < 4; mu++) bc[mu] = (GJP.Bc(mu) == BND_CND_APRD) ? -1 : 1;
    if (cpsgpu_lattice_create(sites, bc, &g_lat) != CPSGPU_OK) die("InvCgShift");
    std::memcpy(g_sites, sites, sizeof(sites));
  }
  if (cpsgpu_import_gauge(g_lat, (const double *)lat.GaugeField(), /*signs_applied=*/1) != CPSGPU_OK)
    die("InvCgShift");
  cpsgpu_dirac_arg a;
  std::memset(&a, 0, sizeof(a));
  switch (lat.Fclass()) {
    case F_CLASS_WILSON: a.kind = CPSGPU_WILSON; break;
    case F_CLASS_DWF: a.kind = CPSGPU_DWF; break;
    case F_CLASS_MOBIUS: a.kind = CPSGPU_MOBIUS; break;
    default: ERR.NotImplemented("DiracOp", "InvCgShift (cpsgpu: Wilson, DWF and Mobius fermions)");
  }
  a.ls = (a.kind == CPSGPU_WILSON) ? 1 : GJP.SnodeSites();
  a.mass = arg->mass;
  a.m5 = GJP.DwfHeight();
  a.mobius_b = (a.kind == CPSGPU_MOBIUS) ? GJP.Mobius_b() : 1.0;
  a.mobius_c = (a.kind == CPSGPU_MOBIUS) ? GJP.Mobius_c() : 0.0;
  a.a5_inv = GJP.DwfA5Inv();
  if (!g_op || std::memcmp(&a, &g_arg, sizeof(a)) != 0) {
    if (g_op) cpsgpu_dirac_destroy(g_op);
    if (cpsgpu_dirac_create(g_lat, &a, &g_op) != CPSGPU_OK) die("InvCgShift");
    g_arg = a;
  }
  // the Mobius preconditioning the DiracOp in scope uses (d_op_mobius.C:104)
  if (a.kind == CPSGPU_MOBIUS) {
    int pc = -1;
    if (cpsgpu_dirac_get_pc_type(g_op, &pc) != CPSGPU_OK) die("InvCgShift");
    if (pc != (int)GJP.ZMobius_PC_Type() && cpsgpu_dirac_set_pc_type(g_op, (int)GJP.ZMobius_PC_Type()) != CPSGPU_OK)
      die("InvCgShift");
  }
  return g_op;
}

int inner_precision() {
  const char *e = std::getenv("CPSGPU_INNER");
  if (!e) return CPSGPU_DOUBLE;
  if (!std::strcmp(e, "single")) return CPSGPU_SINGLE;
  if (!std::strcmp(e, "half")) return CPSGPU_HALF;
  return CPSGPU_DOUBLE;
}
}  // namespace

int DiracOp::InvCgShift(Vector *out, Vector *in, Float src_norm_sq, Float *true_res, Float *shift) {
  const char *fname = "InvCgShift(V*,V*,F,F*,F*)";
  cpsgpu_dirac d = device_op(lat, dirac_arg);
  cpsgpu_cg_arg a;
  cpsgpu_cg_arg_default(&a);
  a.stop_rsd = dirac_arg->stop_rsd;
  a.max_num_iter = dirac_arg->max_num_iter;
  a.src_norm_sq = src_norm_sq;
  a.shift = shift ? *shift : 0.0;
  a.precision = inner_precision();
  cpsgpu_cg_result r;
  if (cpsgpu_invcg(d, (double *)out, (const double *)in, &a, &r) != CPSGPU_OK) die(fname);
  // the reference stops on a breakdown (inv_cg.C:326-329); non-finite values too
  if (r.status == CPSGPU_BREAKDOWN) ERR.General(cname, fname, "p.Ap = 0\n");
  if (r.status == CPSGPU_NONFINITE) ERR.General(cname, fname, "non-finite residual\n");
  if (true_res) *true_res = r.true_res;
  return r.iterations;
}

int DiracOp::MInvCG(Vector **psi, Vector *chi, Float chi_norm, Float *mass, int Nmass, int isz, Float *RsdCG,
                    MultiShiftSolveType type, Float *alpha) {
  const char *fname = "MInvCG(V**,V*,F,F*,int,int,F*,MultiShiftSolveType,F*)";
  (void)isz;  // the reference only prints it (minvcg.C:318-324)
  cpsgpu_dirac d = device_op(lat, dirac_arg);
  const int prec = inner_precision() == CPSGPU_DOUBLE ? CPSGPU_DOUBLE : CPSGPU_SINGLE;
  int iters = 0;
  if (cpsgpu_minvcg(d, reinterpret_cast<double *const *>(psi), (const double *)chi, chi_norm, mass, Nmass, RsdCG,
                    (int)type, alpha, dirac_arg->max_num_iter, prec, /*refine=*/1, &iters) != CPSGPU_OK)
    die(fname);
  return iters;
}

CPS_END_NAMESPACE
