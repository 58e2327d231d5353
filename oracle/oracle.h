/* Test infrastructure only: the CPU oracle.
 *
 * A plain-C, FP64 restatement of the reference's fermion-solve hot path
 * (Wilson / Shamir-DWF / Mobius even-odd preconditioned operators and the
 * CG / multishift-CG loops).  Only tests/, the smoke check and the bench's
 * CPU-baseline leg use it, always as the checker, never as the product.
 *
 * Storage orders are the reference's own (so reference outputs compare
 * element by element):
 *   gauge   WILSON order: u[72*(i + Vh*p) + 18*mu + 2*(row + 3*col) + re/im],
 *           p = 4D parity (even first), i = checkerboard index
 *           (x/2) + (Lx/2)*(y + Ly*(z + Lz*t))      (convert_func.C:361-410,
 *           wilson_dslash.C:54, :288, :307)
 *   fermion f[24*(s*Vh + i) + 2*(colour + 3*spin) + re/im]  (wilson_dslash.C:60)
 * Unlike the reference, the gauge field here carries NO boundary signs: the
 * per-direction sign bc[mu] is applied to every hop that wraps the lattice in
 * direction mu (the reference bakes the same sign into the links at
 * x_mu = L_mu - 1 with Lattice::BondCond, lattice_base.C:5336).
 */
#ifndef CPS_ORACLE_H
#define CPS_ORACLE_H
#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int L[4];      /* local lattice extent x,y,z,t (all even) */
  int ls;        /* fifth-dimension extent (1 for Wilson) */
  double bc[4];  /* +1 periodic, -1 antiperiodic, per direction */
  double a5_inv; /* DoArg.dwf_a5_inv (0 reads as the default 1) */
} orc_geom;

/* Wilson hopping term (wilson_dslash.C:173-515): reads psi on checkerboard
 * cb, writes chi on 1-cb; dag selects D^dagger. */
void orc_wilson_dslash(const orc_geom *g, double *chi, const double *u,
                       const double *psi, int cb, int dag);
/* wilson_m.C:49, wilson_mdag.C:50, wilson_mdagm.C:83 */
void orc_wilson_m(const orc_geom *g, double *chi, const double *u,
                  const double *psi, double kappa, int dag);
void orc_wilson_mdagm(const orc_geom *g, double *chi, const double *u,
                      const double *psi, double kappa, double *dot);

/* Shamir DWF, 5D even-odd (dwf_dslash.C:32, dwf_dslash_4.C:68,
 * dwf_dslash_5_plus_omp.C:115, dwf_m.C:31, dwf_mdag.C:32, dwf_mdagm.C:32).
 * a5inv = g->a5_inv (dwf_dslash_5_plus_omp.C:137-138, dwf_init.C:97-98). */
void orc_dwf_dslash(const orc_geom *g, double *out, const double *u,
                    const double *in, double mass, int cb, int dag);
void orc_dwf_m(const orc_geom *g, double *out, const double *u,
               const double *in, double mass, double m5, int dag);
void orc_dwf_mdagm(const orc_geom *g, double *out, const double *u,
                   const double *in, double mass, double m5, double *dot);

/* Mobius through the complex-coefficient (zMobius) kernels, 4D even-odd,
 * SYM2 preconditioning.  b, c, kappa_b, K = kappa_b/kappa_c per s.
 * zmobius_dslash_4.C:34-221, zmobius_dslash_5_plus.C:125-374,
 * zmobius_m5inv.C:247-396 and :534-679, zmobius_m-sym2.h:5-127,
 * zmobius_mdag-sym2.h:4-109, zmobius_mdagm.C:32-59. */
typedef struct {
  double complex b[64], c[64], kappa_b[64], K[64];
} orc_mobius;
void orc_mobius_params(orc_mobius *mp, int ls, double b, double c, double m5);
/* the same with the fifth-direction spacing: kappa_b = 1/(2(b(4-M5)+a5inv)),
 * kappa_c = 1/(2(c(4-M5)-a5inv)) (d_op_mobius.C:105-108) */
void orc_mobius_params_a5(orc_mobius *mp, int ls, double b, double c, double m5, double a5_inv);
void orc_mobius_dslash_4(const orc_geom *g, const orc_mobius *mp, double *out,
                         const double *u, const double *in, int cb, int dag,
                         double mass);
void orc_mobius_m5inv(const orc_geom *g, const orc_mobius *mp, double *inout,
                      double mass, int dag);
void orc_mobius_m(const orc_geom *g, const orc_mobius *mp, double *out,
                  const double *u, const double *in, double mass, int dag);
void orc_mobius_mdagm(const orc_geom *g, const orc_mobius *mp, double *out,
                      const double *u, const double *in, double mass,
                      double *dot);

/* M5 = 1 + K D5 applied in place (the fifth-direction part with the
 * kappa ratio K per s): what DiracOpMobius::MatInv applies to the initial
 * guess for SYM2 (d_op_mobius.C:505-515 via zmobius_kappa_dslash_5_plus_cmplx,
 * zmobius_dslash_5_plus.C:125-374, which accumulates into its output). */
void orc_mobius_m5(const orc_geom *g, const orc_mobius *mp, double *inout, double mass);
/* every preconditioning type of zmobius_m / zmobius_mdag (zmobius_m.C:40-74,
 * zmobius_mdag.C:41-69; enum ZMobiusPCType, dwf.h:42-48) */
enum { ORC_PC_ORIG = 0, ORC_PC_SYM1 = 1, ORC_PC_SYM2 = 2, ORC_PC_SYM1_MIT = 3, ORC_PC_SYM2_MIT = 4, ORC_PC_SYM3 = 5 };
void orc_mobius_m_pc(const orc_geom *g, const orc_mobius *mp, double *out, const double *u, const double *in,
                     double mass, int dag, int pc);
void orc_mobius_mdagm_pc(const orc_geom *g, const orc_mobius *mp, double *out, const double *u, const double *in,
                         double mass, double *dot, int pc);

/* CG on MatPcDagMatPc (+shift): DiracOp::InvCgShift, inv_cg.C:84-448.
 * The operator is a callback: out = MdagM in, *dot = |M in|^2 when dot!=0.
 * Returns itr+1 as the reference does; *true_res = |b - A x| / |b|. */
typedef void (*orc_mdagm_fn)(void *ctx, double *out, const double *in,
                             double *dot);
int orc_invcg(orc_mdagm_fn op, void *ctx, long n, double *sol,
              const double *src, double src_norm_sq, double stop_rsd,
              int max_num_iter, double *true_res, const double *shift);

/* Multishift CG: DiracOp::MInvCG, minvcg.C:47-353.  type 0 SINGLE,
 * 1 MULTI, 2 GENERAL (enum_int.h:233-238).  RsdCG is overwritten with the
 * achieved residuals; returns the iteration count k as the reference does. */
int orc_minvcg(orc_mdagm_fn op, void *ctx, long n, double **psi,
               const double *chi, double chi_norm, const double *shift,
               int nshift, double *rsdcg, int type, const double *alpha,
               int max_num_iter);

/* BiCGstab(n) on MatPc (not the normal equations): DiracOpWilsonTypes::
 * BiCGstab, bicgstab.C:35-229, step for step (complex dot products
 * <a, b> = sum conj(a) b).  Returns the reference's k (the loop counter after
 * the loop); *true_res = |r| (absolute, as the reference reports it), set
 * only when converged.  matpc(ctx, out, in): out = MatPc in. */
typedef void (*orc_matpc_fn)(void *ctx, double *out, const double *in);
int orc_bicgstab(orc_matpc_fn matpc, void *ctx, long f_size, double *psi, const double *chi, double chi_norm,
                 int n, double stop_rsd, int max_num_iter, double *true_res);

/* Full-lattice solves, DiracOp*::MatInv with the CG inverter.  in and out
 * hold both checkerboards, half = 24*ls*Vh reals each: Wilson and DWF put
 * the odd checkerboard (the one the CG solves on) first, Mobius the even
 * one first, as the reference does.  out holds the initial guess of the
 * CG's checkerboard on entry.  Returns the CG's iteration count.
 *   orc_wilson_matinv  d_op_wilson.C:257-334  (kappa = Wilson kappa)
 *   orc_dwf_matinv     d_op_dwf.C:316-492     (kappa = DWF kappa_5)
 *   orc_mobius_matinv  d_op_mobius.C:407-700  (SYM2) */
int orc_wilson_matinv(const orc_geom *g, double *out, const double *u, const double *in, double kappa,
                      double stop_rsd, int max_num_iter, double *true_res);
int orc_dwf_matinv(const orc_geom *g, double *out, const double *u, const double *in, double mass, double m5,
                   double stop_rsd, int max_num_iter, double *true_res);
int orc_mobius_matinv(const orc_geom *g, const orc_mobius *mp, double *out, const double *u, const double *in,
                      double mass, double stop_rsd, int max_num_iter, double *true_res);
/* the same for the preconditioning pc (ORIG, SYM1, SYM2, SYM3; -1 for the
 * MIT ones, which the reference does not implement) */
int orc_mobius_matinv_pc(const orc_geom *g, const orc_mobius *mp, double *out, const double *u, const double *in,
                         double mass, double stop_rsd, int max_num_iter, double *true_res, int pc);

/* DiracOp::MinResExt (minresext.C): the chronological initial guess over an
 * MatPcDagMatPc callback; v[] is orthonormalised in place, vm[i] = A v[i].
 * At most 16 previous solutions. */
void orc_minresext(orc_mdagm_fn op, void *ctx, long n, double *psi, const double *phi, double **v, double **vm,
                   int degree, double *error);

/* eigCG (inv_eig_cg.C): the dense symmetric eigensolver it needs (cyclic
 * Jacobi; eigen_solver.C's layout) and DiracOp::InvEigCg over an
 * MatPcDagMatPc callback; see oracle.c. */
void orc_sym_eigen(const double *Ap, double *Evec, double *Eval, int n);
int orc_inveigcg(orc_mdagm_fn op, void *ctx, long n, double *sol, const double *src, double stop_rsd, int max_iter,
                 int nev, int m, double **V, double *M, int def_len, double **U, const double *invH,
                 const double *restart, int restart_len, double *true_res);

/* DiracOp::Ritz (ritz.C:152-532) over an MatPcDagMatPc callback (negated
 * when neg); see oracle.c. */
int orc_ritz(orc_mdagm_fn op, void *ctx, int neg, long n, double **psi_all, int N_eig, double RsdR_a,
             double RsdR_r, double Rsdlam, double Cutl_zero, int n_renorm, int Kalk_Sim, int N_min, int N_max,
             double Cv_fact, int MaxCG, int ProjApsiP, double *lambda_out);

/* DiracOp::Jacobi (jacobi.C:48-268) and DiracOpWilsonTypes::RitzEig
 * (eigen_wilson.C:89-586); see oracle.c. */
int orc_jacobi(double **psi, long n, int N_eig, double *lambda, double *off_diag_ri, double Toler, int N_max);
int orc_ritz_eig(orc_mdagm_fn op, void *ctx, int neg, long n, double **psi, int N_eig, double RsdR_a,
                 double RsdR_r, double Rsdlam, double Cv_fact, int n_renorm, int Kalk_Sim, int N_min, int N_max,
                 int MaxCG, int ProjApsiP, int N_KS_max, double *lambda_H, int *valid_eig);

/* HMC fermion force (Fwilson / FdwfBase::EvolveMomFforce): sprojTr, the
 * per-link matrix steps and the whole force loop; see oracle.c. */
void orc_sproj_tr(int mu, int sign, double *f, const double *v, const double *w, int nblk, int v_stride,
                  int w_stride);
void orc_force_matrix(double *f, double *norm, const double *U, const double *T, double coeff);
void orc_fforce(const orc_geom *g, double *mom, const double *u, const double *v1, const double *v2, double dt,
                double out[3]);
/* mobius_Booee and the force loop Fmobius uses (FforceWilsonType::run) */
void orc_mobius_booee(const orc_geom *g, const orc_mobius *mp, double *out, const double *in, double mass);
void orc_fforce_wilson_type(const orc_geom *g, double *mom, const double *u, const double *v1, const double *v2,
                            double coef, double out[3]);

/* Implicitly restarted Lanczos, DiracOp::ImpResLanczos (lanczos.C:193-745)
 * with the Chebyshev-filtered RitzMat (d_op_dwf.C:852-960), and its
 * tridiagonal helpers tqri / QRtrf / eigsrt (eigen_solver.C); see oracle.c.
 * Q is row-major with leading dimension ld. */
void orc_qrtrf(double *d, double *e, int nk, double *Q, int ld, double dsh, int kmin, int kmax);
int orc_tqri(double *d, double *e, int nk, int n, double *Q, int ld);
void orc_eigsrt(double *d, double *Q, int ld, int n);
int orc_lanczos(orc_mdagm_fn op, void *ctx, int neg_lanczos, int neg_conv, long n, float **V, double *alpha, int nk,
                int nt, int np, int maxiters, double stop_res, int conv_check, int Npol, double p0, double p1,
                double eigen_shift);

/* DiracOp::InvLowModeApprox (inv_lowmode_approx.C:272-512); see oracle.c */
void orc_inv_lowmode_approx(double **out, double **in, int len, float **evecs, const double *evals, int neig,
                            long n, int square);

#ifdef __cplusplus
}
#endif

#endif
