// Test infrastructure only: a C-callable harness around the reference's
// own noarch kernels (compiled from the reference sources by
// oracle/Makefile into oracle/_ref/libcpsref.so).  Nothing in the product
// links this; tests/ load it to pin the oracle restatement and the CUDA
// kernels to the reference's arithmetic.
//
// Geometry and parameters are set through the reference's own
// GlobalJobParameter::Initialize(const DoArg&) (include/util/gjp.h:823),
// the Wilson/Dwf workspace through wilson_init / dwf_init
// (d_op_wilson/noarch/wilson_init.C:52, d_op_dwf/noarch/dwf_init.C:41),
// and the Mobius per-s coefficient arrays exactly as the DiracOpMobius
// constructor fills them (d_op_mobius/d_op_mobius.C:105-131).
//
// All vectors are passed in the reference's own storage orders:
//   gauge field  WILSON order, [parity(even first)][cb site][mu][col][row][re,im]
//                (convert_func.C:361-410), boundary signs already applied by
//                the caller (the reference's BondCond, lattice_base.C:5336);
//   fermions     [s][cb site][spin][colour][re,im]  (wilson_dslash.C:60).
#include <config.h>
#include <util/data_types.h>
#include <util/dirac_op.h>
#include <util/vector.h>
#include <util/wilson.h>
#include <util/dwf.h>
#include <util/zmobius.h>
#include <util/mobius.h>
#include <util/lattice/fforce_wilson_type.h>
#include <alg/force_arg.h>
#include <util/gjp.h>
#include <util/sproj_tr.h>
#include <util/fpconv.h>
#include <alg/do_arg.h>
#include <cstring>
#include <vector>

USING_NAMESPACE_CPS

namespace cps {
// the dense symmetric eigensolver eigCG calls (d_op_base/comsrc/eigen_solver.C:40)
int eigen_solver(Float *A, Float *Evec, Float *Eval, int n);
// the tridiagonal helpers of ImpResLanczos (d_op_base/comsrc/eigen_solver.C:206-305, 1442-1498)
int tqri(Float *d, Float *e, int nk, int n, Float **z);
void QRtrf(Float *d, Float *e, int nk, int n, Float **Q, Float dsh, int kmin, int kmax);
void eigsrt(Float *d, int n);
void eigsrt(Float *d, Float **v, int n);
// zmobius_m5inv in-place form (d_op_zmobius/noarch/zmobius_m5inv.C:807)
void zmobius_m5inv(Vector *inout, Float mass, int dag, Zmobus *arg, Complex *K);
}

static Dwf g_dwf;          // DWF and Mobius library argument
static bool g_have_dwf = false;
static Wilson g_wilson;    // Wilson library argument (Fwilson's static struct)
static double g_mobius_b = 1.0, g_mobius_c = 0.0;  // the Mobius b, c of the last ref_init
static bool g_have_wilson = false;

extern "C" {

// Configure the reference for one geometry.  bc_t: 1 periodic, -1 antiperiodic
// (only the BndCndType GJP records; the sign itself is on the links).
int ref_init_a5(int lx, int ly, int lz, int lt, int ls, double m5, double mobius_b, double mobius_c, int bc_t,
                double a5_inv);
int ref_init(int lx, int ly, int lz, int lt, int ls, double m5,
             double mobius_b, double mobius_c, int bc_t) {
  return ref_init_a5(lx, ly, lz, lt, ls, m5, mobius_b, mobius_c, bc_t, 1.0);
}

// the same with DoArg.dwf_a5_inv = a5_inv
int ref_init_a5(int lx, int ly, int lz, int lt, int ls, double m5, double mobius_b, double mobius_c, int bc_t,
                double a5_inv) {
  DoArg d;
  d.x_node_sites = lx; d.y_node_sites = ly; d.z_node_sites = lz;
  d.t_node_sites = lt; d.s_node_sites = ls;
  d.x_nodes = d.y_nodes = d.z_nodes = d.t_nodes = d.s_nodes = 1;
  d.x_bc = d.y_bc = d.z_bc = BND_CND_PRD;
  d.t_bc = (bc_t < 0) ? BND_CND_APRD : BND_CND_PRD;
  d.dwf_height = m5;
  d.dwf_a5_inv = a5_inv;
  GJP.Initialize(d);
  GJP.Mobius_b(mobius_b);
  GJP.Mobius_c(mobius_c);
  g_mobius_b = mobius_b;
  g_mobius_c = mobius_c;
  GJP.ZMobius_PC_Type(ZMOB_PC_SYM2);

  wilson_init(&g_wilson);
  g_have_wilson = true;
  if (ls > 0) {
    dwf_init(&g_dwf);
    g_have_dwf = true;
    // as in DiracOpMobius::DiracOpMobius (d_op_mobius.C:100-131)
    Dwf *m = &g_dwf;
    m->ls = ls;
    m->pc_type = ZMOB_PC_SYM2;
    m->mobius_kappa_b = 1.0 / (2 * (mobius_b * (4 - m5) + a5_inv));
    m->mobius_kappa_c = 1.0 / (2 * (mobius_c * (4 - m5) - a5_inv));
    m->zmobius_b.assign(ls, Complex(mobius_b, 0));
    m->zmobius_c.assign(ls, Complex(mobius_c, 0));
    m->zmobius_kappa_b.assign(ls, Complex(m->mobius_kappa_b, 0));
    m->zmobius_kappa_c.assign(ls, Complex(m->mobius_kappa_c, 0));
    m->zmobius_kappa_ratio.resize(ls);
    for (int i = 0; i < ls; i++)
      m->zmobius_kappa_ratio[i] = m->zmobius_kappa_b[i] / m->zmobius_kappa_c[i];
  }
  return 0;
}

// Complex per-slice coefficients, set as DiracOpZMobius's reset_mobius_arg
// does (d_op_zmobius.C:246-292); b and c hold (re, im) per slice.
void ref_set_zmobius(const double *b, const double *c) {
  Dwf *m = &g_dwf;
  const double m5 = GJP.DwfHeight();
  for (int s = 0; s < m->ls; s++) {
    m->zmobius_b[s] = Complex(b[2 * s], b[2 * s + 1]);
    m->zmobius_c[s] = Complex(c[2 * s], c[2 * s + 1]);
    m->zmobius_kappa_b[s] = 1.0 / (2. * (m->zmobius_b[s] * (4 - m5) + GJP.DwfA5Inv()));
    m->zmobius_kappa_c[s] = 1.0 / (2. * (m->zmobius_c[s] * (4 - m5) - GJP.DwfA5Inv()));
    m->zmobius_kappa_ratio[s] = m->zmobius_kappa_b[s] / m->zmobius_kappa_c[s];
  }
}

double ref_dwf_kappa(void) { return g_dwf.dwf_kappa; }
double ref_mobius_kappa_b(void) { return g_dwf.mobius_kappa_b; }
double ref_mobius_kappa_c(void) { return g_dwf.mobius_kappa_c; }

// ---- Wilson (include/util/wilson.h:226-282) ----
void ref_wilson_dslash(double *chi, double *u, double *psi, int cb, int dag) {
  wilson_dslash(chi, u, psi, cb, dag, &g_wilson);
}
void ref_wilson_m(double *chi, double *u, double *psi, double kappa) {
  wilson_m(chi, u, psi, kappa, &g_wilson);
}
void ref_wilson_mdag(double *chi, double *u, double *psi, double kappa) {
  wilson_mdag(chi, u, psi, kappa, &g_wilson);
}
void ref_wilson_mdagm(double *chi, double *u, double *psi, double *dot, double kappa) {
  wilson_mdagm(chi, u, psi, dot, kappa, &g_wilson);
}

// ---- Shamir DWF (include/util/dwf.h:97-248) ----
void ref_dwf_dslash(double *out, double *u, double *in, double mass, int cb, int dag) {
  dwf_dslash((Vector *)out, (Matrix *)u, (Vector *)in, mass, cb, dag, &g_dwf);
}
void ref_dwf_dslash_4(double *out, double *u, double *in, int cb, int dag) {
  dwf_dslash_4((Vector *)out, (Matrix *)u, (Vector *)in, cb, dag, &g_dwf);
}
void ref_dwf_dslash_5_plus(double *out, double *in, double mass, int dag) {
  dwf_dslash_5_plus((Vector *)out, (Vector *)in, mass, dag, &g_dwf);
}
void ref_dwf_m(double *out, double *u, double *in, double mass) {
  dwf_m((Vector *)out, (Matrix *)u, (Vector *)in, mass, &g_dwf);
}
void ref_dwf_mdag(double *out, double *u, double *in, double mass) {
  dwf_mdag((Vector *)out, (Matrix *)u, (Vector *)in, mass, &g_dwf);
}
void ref_dwf_mdagm(double *out, double *u, double *in, double *dot, double mass) {
  dwf_mdagm((Vector *)out, (Matrix *)u, (Vector *)in, dot, mass, &g_dwf);
}

// ---- Mobius through the zMobius kernels (include/util/zmobius.h:66-229) ----
void ref_zmobius_dslash_4(double *out, double *u, double *in, int cb, int dag, double mass) {
  zmobius_dslash_4((Vector *)out, (Matrix *)u, (Vector *)in, cb, dag, &g_dwf, mass);
}
void ref_zmobius_m5inv(double *inout, double mass, int dag) {
  zmobius_m5inv((Vector *)inout, mass, dag, &g_dwf, g_dwf.zmobius_kappa_ratio.data());
}
// zmobius_dslash_5_plus.C:125: out += the kappa-ratio-weighted fifth-direction hop of in
void ref_zmobius_kappa_dslash_5_plus(double *out, double *in, double mass, int dag) {
  zmobius_kappa_dslash_5_plus_cmplx((Vector *)out, (Vector *)in, mass, dag, &g_dwf,
                                    g_dwf.zmobius_kappa_ratio.data());
}
void ref_zmobius_m(double *out, double *u, double *in, double mass) {
  zmobius_m((Vector *)out, (Matrix *)u, (Vector *)in, mass, &g_dwf);
}
void ref_zmobius_mdag(double *out, double *u, double *in, double mass) {
  zmobius_mdag((Vector *)out, (Matrix *)u, (Vector *)in, mass, &g_dwf);
}
void ref_zmobius_mdagm(double *out, double *u, double *in, double *dot, double mass) {
  zmobius_mdagm((Vector *)out, (Matrix *)u, (Vector *)in, dot, mass, &g_dwf);
}

// ---- NERSC archives: FPConv::checksum (fpconv.C:320-360) of n_words file
// values in the given FP_FORMAT (the enum order of fpconv.C:12-22)
unsigned int ref_fp_checksum(char *data, int n_values, int format) {
  FPConv fp;
  fp.setFileFormat((FP_FORMAT)format);
  return fp.checksum(data, n_values, (FP_FORMAT)format);
}

// ---- Mobius through DiracOpMobius's own kernels (d_op_mobius/noarch) ----
void ref_mobius_dslash_4(double *out, double *u, double *in, int cb, int dag, double mass) {
  mobius_dslash_4((Vector *)out, (Matrix *)u, (Vector *)in, cb, dag, &g_dwf, mass);
}
void ref_mobius_m5inv(double *out, double *in, double mass, int dag) {
  mobius_m5inv((Vector *)out, (Vector *)in, mass, dag, &g_dwf);
}
// mobius_Booee (mobius_dslash_4.C:40-88) as its two steps: out = b in, then
// out += c x the fifth-direction hop of in.  mobius_Booee reads b and c
// through GJP.Mobius_b() / Mobius_c(), which dereference the DoArgExt that
// only a full CPS start-up provides, so the harness passes the values
// ref_init recorded instead.
void ref_mobius_booee(double *out, double *in, double mass) {
  const size_t n = (size_t)12 * GJP.VolNodeSites() * GJP.SnodeSites();
  for (size_t k = 0; k < n; k++) out[k] = g_mobius_b * in[k];
  mobius_kappa_dslash_5_plus((Vector *)out, (Vector *)in, mass, 0, &g_dwf, g_mobius_c);
}
// out += fact x the fifth-direction hop of in (mobius_dslash_5_plus.C:119)
void ref_mobius_kappa_dslash_5_plus(double *out, double *in, double mass, int dag, double fact) {
  mobius_kappa_dslash_5_plus((Vector *)out, (Vector *)in, mass, dag, &g_dwf, fact);
}
void ref_mobius_m(double *out, double *u, double *in, double mass) {
  mobius_m((Vector *)out, (Matrix *)u, (Vector *)in, mass, &g_dwf);
}
// FforceWilsonType(mom, gauge, v1, v2, Ls, coef).run() (fforce_wilson_type.C):
// CANONICAL mom and gauge (boundary signs on the links, as Fmobius applies
// BondCond around it), v1 / v2 in the S_INNER order [4D site][s][24]
void ref_fforce_wilson_type(double *mom, double *u, double *v1, double *v2, int ls, double coef, double *out) {
  FforceWilsonType f((Matrix *)mom, (Matrix *)u, v1, v2, ls, coef);
  ForceArg a = f.run();
  out[0] = a.L1;
  out[1] = a.L2;
  out[2] = a.Linf;
}

// ---- eigCG: eigen_solver (packed lower triangle in, Evec[k n + i] = component k of eigenvector i)
int ref_eigen_solver(double *A, double *Evec, double *Eval, int n) { return eigen_solver(A, Evec, Eval, n); }

// ---- ImpResLanczos helpers; Q row-major, n x n, passed as row pointers ----
static std::vector<Float *> rows_of(double *Q, int n) {
  std::vector<Float *> r(n);
  for (int i = 0; i < n; i++) r[i] = Q + (size_t)i * n;
  return r;
}
int ref_tqri(double *d, double *e, int nk, int n, double *Q) { return tqri(d, e, nk, n, rows_of(Q, n).data()); }
void ref_qrtrf(double *d, double *e, int nk, int n, double *Q, double dsh, int kmin, int kmax) {
  QRtrf(d, e, nk, n, rows_of(Q, n).data(), dsh, kmin, kmax);
}
void ref_eigsrt(double *d, double *Q, int n) {
  if (Q) eigsrt(d, rows_of(Q, n).data(), n);
  else eigsrt(d, n);
}

// ---- HMC fermion force pieces ----
// sprojTr{X,Y,Z,T}{m,p} (f_wilson_types/noarch/sproj_tr.C), indexed as the
// SprojType enum orders them (alg/enum_int.h: XM..TM = 0..3, XP..TP = 4..7)
void ref_sproj_tr(int which, double *f, double *v, double *w, int nblk, int v_stride, int w_stride) {
  typedef void (*fn)(IFloat *, IFloat *, IFloat *, int, int, int);
  static const fn tab[8] = {sprojTrXm, sprojTrYm, sprojTrZm, sprojTrTm,
                            sprojTrXp, sprojTrYp, sprojTrZp, sprojTrTp};
  tab[which](f, v, w, nblk, v_stride, w_stride);
}
// the per-link steps of the force loop through the reference's Matrix
// (util/vector.h): F = U T, F = TrLessAntiHerm with F^dag, F *= coeff, norm()
void ref_force_matrix(double *f, double *norm, double *U, double *T, double coeff) {
  Matrix a, b;
  a.DotMEqual(*(const Matrix *)U, *(const Matrix *)T);
  b.Dagger(a);
  a.TrLessAntiHermMatrix(b);
  a *= coeff;
  *norm = a.norm();
  std::memcpy(f, &a, 18 * sizeof(double));
}

}  // extern "C"
