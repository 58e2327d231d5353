/* cpsgpu: B200-native fermion-solve hot path of CPS (Columbia Physics System)
 * behind a C ABI.
 *
 * The library keeps the gauge field and fermion fields resident on one GPU
 * and implements, as hand-written sm_100a kernels, the even-odd
 * preconditioned Wilson, Shamir domain-wall and Mobius operators and the CG
 * and multishift-CG solvers that CPS's DiracOp classes run on the CPU.
 * A CPS build calls these entry points from a thin C++ shim that overrides
 * the DiracOp methods; every function replaces the reference interface cited
 * in its comment (paths relative to the reference's cps_pp tree).
 *
 * Conventions shared with the reference:
 *   - vectors are host arrays of doubles in CPS storage order:
 *       Wilson:  [cb site][spin][colour][re,im], 24 reals per site, the
 *                preconditioned (odd) checkerboard (convert_func.C:452-490);
 *       DWF:     [s][cb site][24], slice s on 4D parity (s+cb)%2
 *                (dwf_dslash_4.C:107-137, convert.C:728-760);
 *       Mobius:  [s][cb site][24], every slice on one 4D parity
 *                (DWF_4D_EOPREC_EE, convert.C:797-851);
 *     with cb site = (x/2) + (Lx/2)*(y + Ly*(z + Lz*t));
 *   - the gauge field is in WILSON order, [parity (even first)][cb site]
 *     [mu][3x3 complex, element (row,col) at 2*(row+3*col)]
 *     (convert_func.C:361-410, wilson_dslash.C:54);
 *   - boundary conditions are per direction (+1 periodic, -1 antiperiodic).
 *     The reference multiplies the boundary links by the sign while a DiracOp
 *     is alive (Lattice::BondCond, lattice_base.C:5336); pass signs_applied=1
 *     to cpsgpu_import_gauge for such a field.  The library removes the signs
 *     from its copy and applies them to the hops instead, which keeps every
 *     stored link in SU(3) so 12-real compression stays exact.
 *
 * Errors: every function returns CPSGPU_OK (0) or a negative code, with a
 * message from cpsgpu_last_error().  Where the reference exits the process
 * (ERR.General, CG breakdown at inv_cg.C:326-329), the library returns a
 * status instead; the shim maps it back to ERR.* to keep CPS's behaviour.
 */
#ifndef CPSGPU_H
#define CPSGPU_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CPSGPU_OK 0
#define CPSGPU_ERR_ARG (-1)
#define CPSGPU_ERR_UNSUPPORTED (-2)
#define CPSGPU_ERR_CUDA (-3)
#define CPSGPU_ERR_STATE (-4)

/* solver status (cpsgpu_cg_result.status) */
#define CPSGPU_CONVERGED 1
#define CPSGPU_MAX_ITER 2
#define CPSGPU_BREAKDOWN 3 /* p.Ap == 0 */
#define CPSGPU_NONFINITE 4

/* fermion actions */
#define CPSGPU_WILSON 0
#define CPSGPU_DWF 1
#define CPSGPU_MOBIUS 2

/* precisions */
#define CPSGPU_DOUBLE 0
#define CPSGPU_SINGLE 1
#define CPSGPU_HALF 2 /* FP16 storage with a per-site FP32 norm, FP32 arithmetic */

/* multishift solve types (enum MultiShiftSolveType, include/alg/enum_int.h:233-238) */
#define CPSGPU_MS_SINGLE 0
#define CPSGPU_MS_MULTI 1
#define CPSGPU_MS_GENERAL 2

typedef struct cpsgpu_lattice_s *cpsgpu_lattice;
typedef struct cpsgpu_dirac_s *cpsgpu_dirac;
typedef struct cpsgpu_field_s *cpsgpu_field;

/* ---- version and errors ---- */
const char *cpsgpu_version(void);
const char *cpsgpu_last_error(void);
int cpsgpu_device_count(int *count);
/* select the CUDA device for objects created afterwards on this thread */
int cpsgpu_set_device(int device);
/* The end of a job (CPS's End(), after the DiracOps and Lattice are gone):
 * waits for the current device's work and forgets the launch shapes the
 * autotuner recorded.  Lattices, operators and fields are released by their
 * own destroy calls, before it; the library may be used again afterwards. */
int cpsgpu_finalize(void);

/* ---- geometry and gauge field ---- */
/* Local lattice geometry on the current CUDA device.  Replaces the GJP
 * geometry (GlobalJobParameter::Initialize, include/util/gjp.h:823) and the
 * Lattice constructor's gauge allocation (lattice_base.C:320-325). */
int cpsgpu_lattice_create(const int node_sites[4], const int bc[4], cpsgpu_lattice *lat);
int cpsgpu_lattice_destroy(cpsgpu_lattice lat);
/* Upload a WILSON-order gauge field (the field Lattice::Convert(WILSON)
 * produces, convert.C:141-260).  Stores FP64 (18- and 12-real), FP32 and
 * FP16 12-real copies on the device. */
int cpsgpu_import_gauge(cpsgpu_lattice lat, const double *u_wilson, int signs_applied);
/* max |row2 - conj(row0 x row1)| over all links, and whether FP64 uses 12 reals */
int cpsgpu_gauge_info(cpsgpu_lattice lat, double *recon_err, int *fp64_recon12);
int cpsgpu_synchronize(cpsgpu_lattice lat);
/* Stored link form of the FP32 or FP16 operator: 12 reals (third row rebuilt
 * in registers) or 18, in the operator's precision; the FP16 operator may
 * also read FP32 links (CPSGPU_LINKS_F32_12 / _18: no conversions in the
 * kernel).  cpsgpu_autotune picks the fastest; this overrides it. */
#define CPSGPU_LINKS_F32_12 112
#define CPSGPU_LINKS_F32_18 118
int cpsgpu_set_link_reals(cpsgpu_lattice lat, int prec, int reals);
int cpsgpu_get_link_reals(cpsgpu_lattice lat, int prec, int *reals);

/* ---- storage orders on the host (no device work) ----
 * StrOrdType values (enum_int.h:87-97).  Fields hold both checkerboards.
 *   cpsgpu_fconvert  FwilsonTypes::Fconvert / FdwfBase::Fconvert
 *                    (convert.C:444-562, :639-1000): fermion, 24*ls*vol reals
 *                    in place; ls = 1 for a 4D field.  4D WILSON order puts
 *                    the odd checkerboard first; 5D WILSON is the DWF
 *                    even-odd order (odd part: slice s holds the 4D sites of
 *                    parity (s+1)%2).
 *   cpsgpu_gconvert  Lattice::Convert for the gauge field (convert.C:141-420):
 *                    72*vol reals in place; WILSON = even parity first, each
 *                    link stored transposed (col, row).
 *   cpsgpu_four2five / cpsgpu_five2four  FdwfBase::Ffour2five / Ffive2four
 *                    (f_dwf_base.C:961, :1068): the upper spin half of slice
 *                    s_u and the lower one of slice s_l carry the 4D field;
 *                    ncb = 2 for both checkerboards, 1 for one. */
#define CPSGPU_STR_CANONICAL 0
#define CPSGPU_STR_WILSON 2
int cpsgpu_fconvert(const int node_sites[4], int ls, double *f, int to, int from);
int cpsgpu_gconvert(const int node_sites[4], double *u, int to, int from);
int cpsgpu_four2five(const int node_sites[4], int ls, double *five, const double *four, int s_u, int s_l, int ncb);
int cpsgpu_five2four(const int node_sites[4], int ls, double *four, const double *five, int s_u, int s_l, int ncb);
/* The same four conversions on device memory (FP64 device pointers of the
 * caller, e.g. cudaMalloc'd or a framework's tensors), out of place
 * (dst != src), for the geometry of lat (a whole lattice, not a t slab),
 * asynchronous on lat's stream (cpsgpu_synchronize waits for them). */
int cpsgpu_fconvert_device(cpsgpu_lattice lat, int ls, double *dst, const double *src, int to, int from);
int cpsgpu_gconvert_device(cpsgpu_lattice lat, double *dst, const double *src, int to, int from);
int cpsgpu_four2five_device(cpsgpu_lattice lat, int ls, double *five, const double *four, int s_u, int s_l, int ncb);
int cpsgpu_five2four_device(cpsgpu_lattice lat, int ls, double *four, const double *five, int s_u, int s_l, int ncb);

/* ---- Dirac operators ---- */
typedef struct {
  int kind;        /* CPSGPU_WILSON / CPSGPU_DWF / CPSGPU_MOBIUS */
  int ls;          /* fifth-dimension extent (ignored for Wilson) */
  double mass;     /* CgArg.mass (cg_arg.h:17-36) */
  double m5;       /* DoArg.dwf_height */
  double mobius_b; /* DoArgExt.mobius_b_coeff */
  double mobius_c; /* DoArgExt.mobius_c_coeff */
  double a5_inv;   /* DoArg.dwf_a5_inv, the fifth-direction inverse lattice
                      spacing (DWF, Mobius); 0 selects the default 1 */
} cpsgpu_dirac_arg;

/* Replaces the DiracOpWilson / DiracOpDwf / DiracOpMobius constructors
 * (d_op_wilson.C:54-137, d_op_dwf.C:67-100, d_op_mobius.C:57-140): kappa
 * = 1/(2(m+4)) (Wilson), 1/(2(4 + a5_inv - M5)) (DWF, dwf_init.C:97-98),
 * kappa_b = 1/(2(b(4-M5) + a5_inv)) and kappa_c = 1/(2(c(4-M5) - a5_inv))
 * (Mobius, d_op_mobius.C:105-108); the DWF fifth-direction hop weighs 2 a5_inv
 * and -2 m_f a5_inv at the walls (dwf_dslash_5_plus_omp.C:137-138). */
int cpsgpu_dirac_create(cpsgpu_lattice lat, const cpsgpu_dirac_arg *arg, cpsgpu_dirac *d);
int cpsgpu_dirac_destroy(cpsgpu_dirac d);
/* Complex per-slice Mobius coefficients (DiracOpZMobius, d_op_zmobius.C
 * :246-292): b and c hold 2*Ls doubles each, (re, im) of b_s and c_s.
 * kappa_b(s) = 1/(2(b_s(4 - M5) + 1)), kappa_c(s) = 1/(2(c_s(4 - M5) - 1)).
 * Every operator and solver of the Mobius handle then uses them;
 * cpsgpu_matinv stays real-only (it scales by the real kappa_b). */
int cpsgpu_dirac_set_zmobius(cpsgpu_dirac d, const double *b, const double *c);
int cpsgpu_dirac_info(cpsgpu_dirac d, double *kappa, double *kappa_c);

/* Host-vector operators; vectors hold one preconditioned checkerboard in
 * CPS order, n = 24 * Ls * Vol/2 doubles; prec selects the device precision
 * (inputs and outputs are FP64 on the host either way). */
/* Wilson: wilson_dslash (wilson.h:226, wilson_dslash.C:173-515).
 * DWF: dwf_dslash = 4D hop of every slice + fifth-direction hop
 * (dwf_dslash.C:32-51).  Reads cb, writes 1-cb. */
int cpsgpu_dslash(cpsgpu_dirac d, double *out, const double *in, int cb, int dag, int prec);
/* DiracOp*::MatPc / MatPcDag: wilson_m / wilson_mdag (wilson_m.C:49, wilson_mdag.C:50),
 * dwf_m / dwf_mdag (dwf_m.C:31, dwf_mdag.C:32), zmobius_m_sym2 /
 * zmobius_mdag_sym2 (zmobius_m-sym2.h:5, zmobius_mdag-sym2.h:4). */
int cpsgpu_matpc(cpsgpu_dirac d, double *out, const double *in, int dag, int prec);
/* DiracOp*::MatPcDagMatPc(out, in, dot): wilson_mdagm (wilson_mdagm.C:83),
 * dwf_mdagm (dwf_mdagm.C:32), zmobius_mdagm (zmobius_mdagm.C:32).
 * *dot = |MatPc in|^2 when dot is non-null. */
int cpsgpu_matpc_dag_matpc(cpsgpu_dirac d, double *out, const double *in, double *dot, int prec);
/* No counterpart in the reference.  The same FP64 MatPcDagMatPc for callers
 * that cannot allocate device memory when they apply the operator (their
 * device memory belongs to their own pool allocator, or they cannot take the
 * device-wide synchronisation of cudaMalloc/cudaFree).  in_dev and out_dev are
 * caller-owned device pointers holding one FP64 field in the library's
 * device layout: reals (2g, 2g+1) of CPS site i in slice s at
 * double2 index (s*12 + g)*Vol/2 + i.  Every temporary lives in one fixed
 * 64 MiB device array that the library holds on each GPU it is used on until
 * the process exits, so the call allocates nothing; operators whose two FP64
 * fields do not fit in it (more than about 170k 5D sites) are rejected with
 * CPSGPU_ERR_ARG.  Wilson and DWF only.  The first call on a device looks up
 * that array's address, so make it before any stream capture.  All calls
 * share the array: calls that overlap on the GPU (from several threads or
 * streams) race.  *dot = |MatPc in|^2 when dot is non-null.  Returns when the
 * result is in out_dev; the caller must have finished writing in_dev. */
int cpsgpu_matpc_dag_matpc_noalloc(cpsgpu_dirac d, double *out_dev, const double *in_dev, double *dot);
/* DiracOp*::Mat (dag 0) / MatDag (dag 1), the unpreconditioned operator on
 * full vectors of both checkerboards, 2 n doubles ([odd][even] halves for
 * Wilson and DWF, [even][odd] for Mobius): Wilson d_op_wilson.C:362-424,
 * DWF d_op_dwf.C:541-627, Mobius Mat d_op_mobius.C:735-795 (out = (1 +
 * a5_inv K D5) in - kappa_b Dslash_4 of the other half).  Mobius MatDag
 * returns CPSGPU_ERR_ARG: the reference's stops with an error
 * (d_op_mobius.C:879).  FP64. */
int cpsgpu_mat(cpsgpu_dirac d, double *out, const double *in, int dag);
/* DiracOp*::MatHerm: gamma_5 Mat (Wilson, d_op_wilson.C:426-443),
 * gamma_5 R Mat with R the reflection s -> Ls-1-s of FdwfBase::Freflex
 * (DWF d_op_dwf.C:629-660, Mobius d_op_mobius.C:915-942); gamma_5 =
 * diag(1, 1, -1, -1) (MultGamma 15).  Full vectors as cpsgpu_mat.  FP64. */
int cpsgpu_mat_herm(cpsgpu_dirac d, double *out, const double *in);
/* DiracOpMobius::MatPcDagMatPcShift with eigen_shift mu (d_op_mobius.C:235,
 * zmobius_mdagm_shift zmobius_mdagm.C:79-135): out = M^+ M in - 2 mu R g5
 * M in + mu^2 in, M = MatPc, R g5 = ReflectAndMultGamma5 within the
 * checkerboard; *dot = |M in|^2 when dot is non-null.  Mobius only. */
int cpsgpu_matpc_dag_matpc_shift(cpsgpu_dirac d, double *out, const double *in, double mu, double *dot, int prec);
/* Mobius pieces: zmobius_dslash_4 (zmobius_dslash_4.C:209) and the
 * out-of-place zmobius_m5inv (zmobius_m5inv.C:822). */
int cpsgpu_mobius_dslash_4(cpsgpu_dirac d, double *out, const double *in, int cb, int dag, int prec);
int cpsgpu_mobius_m5inv(cpsgpu_dirac d, double *out, const double *in, int dag, int prec);
/* The Mobius operator's preconditioning, GJP.ZMobius_PC_Type (DoArgExt
 * zmobius_pc_type; enum ZMobiusPCType, dwf.h:42-48): 0 ORIG, 1 SYM1, 2 SYM2
 * (the default), 3 SYM1_MIT, 4 SYM2_MIT, 5 SYM3, as zmobius_m / zmobius_mdag
 * dispatch on it (zmobius_m.C:40-74, zmobius_mdag.C:41-69).  MatPc, MatPcDag,
 * MatPcDagMatPc and the CG and multishift solvers follow it; MatInv
 * supports ORIG, SYM1, SYM2 and SYM3 (d_op_mobius.C:477-663; the MIT forms
 * stop there with an error, and return one here).  The forms other than
 * SYM2 need real b, c, the same on every slice.  SYM3 is reproduced as the
 * reference computes it: its rescaling of GJP's b, c does not reach the
 * hops, which read the operator's own copies (zmobius_dslash_4.C:61-62). */
int cpsgpu_dirac_set_pc_type(cpsgpu_dirac d, int pc_type);
int cpsgpu_dirac_get_pc_type(cpsgpu_dirac d, int *pc_type);
/* No counterpart in the reference: the kernel of the Mobius operator's
 * standalone Ls x Ls mixings (M5^-1, the first step of MatPc).
 *   0 (the default): for FP16 fields the register-tiled arithmetic of 3 on
 *     input tiles staged in shared memory by bulk asynchronous copies, two
 *     stages per persistent block (mix_bulk.cu; Ls 8, 10, 12, 16, sites per
 *     checkerboard slice a multiple of 32, real b, c), else as 3;
 *   1: for FP16 fields, mma.sync m16n8k16 contractions on the tensor cores
 *     (FP16 operands with the matrix split into high and low parts, FP32
 *     accumulation, mix_tc.cu; Ls <= 16, real b, c), else as 0;
 *   2: CUDA cores, the spinors staged in shared memory (blas.cu), the form
 *     every case outside the others uses (complex zMobius coefficients,
 *     other Ls);
 *   3: for FP32 and FP16 fields, CUDA cores, register-tiled (mix_reg.cu):
 *     the two real matrices are a kernel parameter, every thread computes
 *     all Ls output slices of a block of reals with packed FP32 multiply-adds
 *     (Ls 8, 10, 12, 16, 20, 24; real b, c); FP64 fields as 2.
 * Every form but 1 gives the same bits. */
int cpsgpu_set_mix_impl(cpsgpu_dirac d, int impl);

/* ---- solvers ---- */
typedef struct {
  double stop_rsd;     /* CgArg.stop_rsd: stop when |r| <= stop_rsd |b| */
  int max_num_iter;    /* CgArg.max_num_iter */
  double src_norm_sq;  /* 0: computed (inv_cg.C:166-169) */
  double shift;        /* solve (MatPcDagMatPc + shift) x = b */
  int precision;       /* CPSGPU_DOUBLE: plain FP64 CG; SINGLE / HALF: mixed precision */
  double delta;        /* reliable-update threshold (mixed precision); 0: 0.01 for FP32, 0.1 for FP16 */
  int chunk;           /* iterations per CUDA-graph launch; 0: default 8 */
  int use_graph;       /* capture the iteration chunk in a CUDA graph */
} cpsgpu_cg_arg;

typedef struct {
  int iterations;       /* as DiracOp::InvCg returns it: iterations done + 1 */
  int status;           /* CPSGPU_CONVERGED / MAX_ITER / BREAKDOWN / NONFINITE */
  double true_res;      /* |b - A x| / |b|, recomputed in FP64 (inv_cg.C:403-415) */
  int reliable_updates; /* mixed precision only */
  double seconds;       /* device time of the solve (CUDA events on the library stream) */
  long long kernels;    /* kernels this library executed for the solve */
} cpsgpu_cg_result;

void cpsgpu_cg_arg_default(cpsgpu_cg_arg *arg);

/* DiracOp::InvCg(out, in, src_norm_sq, true_res) -> InvCgShift
 * (inv_cg.C:84-454): sol holds the initial guess on entry. */
int cpsgpu_invcg(cpsgpu_dirac d, double *sol, const double *src, const cpsgpu_cg_arg *arg,
                 cpsgpu_cg_result *res);
/* nrhs independent solves in one batched launch sequence (each gauge link
 * load serves every right-hand side); the multi-source
 * DiracOpMobius::MatInv(std::vector<Vector*>...) (d_op_mobius.C:407) loops
 * InvCg over the same set. res has nrhs entries. */
int cpsgpu_invcg_multi(cpsgpu_dirac d, double *const *sol, const double *const *src, int nrhs,
                       const cpsgpu_cg_arg *arg, cpsgpu_cg_result *res);
/* ---- gauge configurations ----
 * Plaquette and link trace of the resident (unsigned) links, normalised as
 * the NERSC header and ReadLatticeParallel's check use them:
 * plaq = Lattice::SumReTrPlaq() / (18 V) (lattice_base.C:2878-3060),
 * link_trace = sum over links of Re tr U / (12 V). */
int cpsgpu_gauge_plaquette(cpsgpu_lattice lat, double *plaq, double *link_trace);

/* NERSC archive format (ReadLatticePar.C, WriteLatticePar.C, latheader.C,
 * fpconv.C); fp formats in the reference's FP_FORMAT order. */
#define CPSGPU_FP_IEEE32 3
#define CPSGPU_FP_IEEE32BIG 4
#define CPSGPU_FP_IEEE32LITTLE 5
#define CPSGPU_FP_IEEE64 6
#define CPSGPU_FP_IEEE64BIG 7
#define CPSGPU_FP_IEEE64LITTLE 8
typedef struct {
  int dims[4];
  int recon_row_3;           /* 1: DATATYPE = 4D_SU3_GAUGE (two rows stored), 0: 4D_SU3_GAUGE_3x3 */
  int fp_format;             /* CPSGPU_FP_* */
  double plaquette;          /* PLAQUETTE (read: as the reference parses it, %f) */
  double link_trace;         /* LINK_TRACE */
  unsigned int checksum;     /* CHECKSUM */
  int sequence_number;
  char ensemble_id[128], ensemble_label[128], creator[128];
} cpsgpu_nersc_header;
/* ReadLatticeParallel::read without the lattice: parse the header, check
 * the dimensions, read the links (u: CANONICAL [site][mu][3][3][re, im]),
 * verify the checksum (error on a mismatch) and rebuild the third rows of
 * a two-row file. */
int cpsgpu_nersc_read(const char *path, const int node_sites[4], double *u, cpsgpu_nersc_header *hdr);
/* WriteLatticeParallel::write of a CANONICAL host field: header (plaquette
 * and link trace computed from u, periodic boundaries as the reference
 * records them, meta: ensemble id / label / sequence number / creator, may
 * be NULL) and data in fp_format, two rows per link when recon_row_3. */
int cpsgpu_nersc_write(const char *path, const int node_sites[4], const double *u, int recon_row_3, int fp_format,
                       const cpsgpu_nersc_header *meta, cpsgpu_nersc_header *out);
/* ReadLatticeParallel::read into the lattice: read (as above), import the
 * links (no boundary signs) and fail when the plaquette of the imported
 * field deviates from the header's by more than check_precision (relative;
 * the reference's default is 0.01).  *plaq = the computed plaquette. */
int cpsgpu_lattice_load_nersc(cpsgpu_lattice lat, const char *path, double check_precision, cpsgpu_nersc_header *hdr,
                              double *plaq);

/* ---- HMC fermion force (Wilson and Shamir DWF) ----
 * The reference's ForceArg (alg/force_arg.h): L1 = mean |F|, L2 = rms |F|,
 * Linf = max |F| over links, |F|^2 = Matrix::norm() = -2 Re tr F^2. */
typedef struct {
  double L1, L2, Linf;
} cpsgpu_force_arg;
/* DiracOpWilson / DiracOpDwf::CalcHmdForceVecs(chi) (d_op_wilson.C:466-507,
 * d_op_dwf.C:682-733): f_out = (chi, D chi), f_in = (-kappa^2 MatPc chi,
 * D^dag of it), full fields in WILSON order ([odd half][even half], before
 * the reference's conversion to CANONICAL); chi is the odd half.
 * Mobius (real b, c; SYM2): the vectors Fmobius::EvolveMomFforce builds,
 * DiracOpMobius::CalcHmdForceVecs(f_out, f_in, MatPc chi, chi)
 * (d_op_mobius.C:1015-1100, f_mobius.C:847-887), [even half][odd half];
 * chi is left unchanged (the reference overwrites it with M5^-1 chi). */
int cpsgpu_calc_hmd_force_vecs(cpsgpu_dirac d, double *f_out, double *f_in, const double *chi);
/* Fwilson::EvolveMomFforce(mom, chi, mass, dt) (f_wilson.C:470-687),
 * FdwfBase::EvolveMomFforce (f_dwf_base_force.C:41-300) and
 * Fmobius::EvolveMomFforce(mom, frm, mass, step_size) (f_mobius.C:847-887,
 * FforceWilsonType): mom += the fermion force of the pseudofermion solution
 * chi (the preconditioned half, WILSON order) for a step dt; mom is the
 * CANONICAL Matrix field [site][mu][3][3][re, im] with the lexicographic site
 * x + Lx (y + Ly (z + Lz t)).  The operator's own mass plays the reference's
 * mass argument.  Mobius: real b, c (not zMobius). */
int cpsgpu_evolve_mom_fforce(cpsgpu_dirac d, double *mom, const double *chi, double dt, cpsgpu_force_arg *out);
/* Fwilson / FdwfBase::RHMC_EvolveMomFforce(mom, sol, degree, isz, alpha,
 * mass, dt, sol_d, force_measure) (f_wilson.C:689-757, f_dwf_base.C:1424):
 * mom += sum over the poles k < degree of the force of sol[k] with step
 * dt alpha[k].  force_measure != 0 (FORCE_MEASURE_YES): the poles are summed
 * into a zeroed field first, *out = the ForceArg of that sum, then it is
 * added to mom; otherwise they accumulate into mom directly and *out = 0. */
int cpsgpu_rhmc_evolve_mom_fforce(cpsgpu_dirac d, double *mom, const double *const *sol, int degree,
                                  const double *alpha, double dt, int force_measure, cpsgpu_force_arg *out);
/* Device timing of CalcHmdForceVecs + the force update on a Gaussian chi
 * (ms per call, ms of the force kernel alone, its algorithmic bytes). */
int cpsgpu_time_fforce(cpsgpu_dirac d, int reps, double *ms_total, double *ms_kernel, double *kernel_bytes);

/* DiracOp::Ritz(psi_all, N_eig, lambda, RsdR_a, RsdR_r, Rsdlam, Cutl_zero,
 * n_renorm, Kalk_Sim, N_min, N_max, Cv_fact, MaxCG, ProjApsiP)
 * (d_op_base/comsrc/ritz.C:152-532): the N_eig-th lowest eigenpair of
 * MatPcDagMatPc (RitzMatOper MATPCDAG_MATPC; neg != 0: of its negative,
 * NEG_MATPCDAG_MATPC) by conjugate-gradient minimisation of the Ritz
 * functional orthogonal to psi_all[0..N_eig-1) (previous eigenvectors),
 * starting from psi_all[N_eig-1], which receives the eigenvector; *lambda
 * its eigenvalue, *iterations the reference's count.  Returns
 * CPSGPU_MAX_ITER (the reference exits) after MaxCG iterations. */
typedef struct {
  double RsdR_a, RsdR_r, Rsdlam, Cutl_zero, Cv_fact;
  int n_renorm, Kalk_Sim, N_min, N_max, MaxCG, ProjApsiP, neg;
} cpsgpu_ritz_arg;
int cpsgpu_ritz(cpsgpu_dirac d, double *const *psi_all, int N_eig, const cpsgpu_ritz_arg *arg, double *lambda,
                int *iterations);
/* DiracOp::Jacobi(psi, N_eig, lambda, off_diag, Toler, N_max)
 * (d_op_base/comsrc/jacobi.C:48-268): Jacobi rotations of the vectors psi
 * (in place) that diagonalise the small hermitian matrix with diagonal
 * lambda and off-diagonal elements off_diag[j(j-1)/2 + i] = <psi_i, A psi_j>
 * (i < j; (re, im) pairs), then the pairs sorted by |lambda|.  *sweeps = the
 * reference's count; CPSGPU_MAX_ITER after N_max sweeps. */
int cpsgpu_jacobi(cpsgpu_dirac d, double *const *psi, int N_eig, double *lambda, double *off_diag, double toler,
                  int n_max, int *sweeps);
/* DiracOpWilsonTypes::RitzEig(psi, lambda_H, valid_eig, eig_arg)
 * (d_op_wilson_types/eigen_wilson.C:89-586) with RitzMatOper
 * MATPCDAG_MATPC (arg->neg = 0) or NEG_MATPCDAG_MATPC (arg->neg = 1):
 * Kalkreuter-Simma sweeps of Ritz (Kalk_Sim stopping rules) and Jacobi
 * until the largest relative eigenvalue change is <= arg->Rsdlam, at most
 * N_KS_max sweeps (successive Ritz calls when N_eig = 1 or
 * arg->Kalk_Sim = 0); then the projection stage: vectors failing the
 * reference's row-norm test replaced by (1 +- A / sqrt|lambda|) psi, a
 * normalised Gram-Schmidt pass and a last Jacobi (tolerance 1e-5).
 * psi (in place): start vectors in, eigenvectors out; lambda_H[0..N_eig):
 * the eigenvalues, lambda_H[N_eig..2 N_eig): the Ritz / KS eigenvalues
 * (the reference's layout); valid_eig[N_eig].  *iterations = the total
 * Ritz count, or with CPSGPU_MAX_ITER returned the reference's -1 (MaxCG) /
 * -2 (N_KS_max), or -3 when a Jacobi call ran out (the reference exits).
 * The reference's text dump of the matrix to eig_arg->fname is not made. */
int cpsgpu_ritz_eig(cpsgpu_dirac d, double *const *psi, int N_eig, const cpsgpu_ritz_arg *arg, int N_KS_max,
                    double *lambda_H, int *valid_eig, int *iterations);

/* RitzMatType values (include/alg/enum_int.h:210-222) the eigensolvers take */
#define CPSGPU_RITZ_MAT_HERM 1
#define CPSGPU_RITZ_MATPC_HERM 2
#define CPSGPU_RITZ_MATPCDAG_MATPC 3
#define CPSGPU_RITZ_NEG_MATPCDAG_MATPC 4
/* LanczosArg (include/alg/lanczos_arg.h:32-53) with its MatrixPolynomialArg
 * (Npol, params[0..1]); mass, precision, save and file fields are the
 * operator's or the caller's business */
typedef struct {
  int RitzMat_lanczos, RitzMat_convcheck; /* CPSGPU_RITZ_* */
  int nk_lanczos_vectors, nt_lanczos_vectors, np_lanczos_vectors;
  double eigen_shift, stop_residual;
  int maxiters, conv_check;
  int Npol;
  double params[2];
} cpsgpu_lanczos_arg;
/* DiracOp::ImpResLanczos(V, alpha, lanczos_arg) (d_op_base/comsrc/lanczos.C:193-745)
 * with the Chebyshev-filtered RitzMat of DiracOpDwf / DiracOpMobius
 * (d_op_dwf.C:852-960, d_op_mobius.C:1279): T_Npol of
 * (2 A - (a+b)) / (a-b), a = params[0]^2, b = (params[1] + |eigen_shift|)^2.
 * V: nk + np float vectors of the operator's half-checkerboard size in
 * WILSON order, V[0] the start vector; on return the Ritz vectors of the
 * leading nk block, V[0..nt) the wanted eigenvectors; alpha[nk + np]: the
 * first nt their eigenvalues of the unfiltered RitzMat_convcheck operator.
 * *restarts = the restart count (maxiters when not converged, as the
 * reference returns it).  CPSGPU_ERR_UNSUPPORTED for Wilson fermions (the
 * reference's DiracOp::RitzMat(V*,V*,MP*) is NotImplemented) and other
 * RitzMat types; CPSGPU_NONFINITE on a NaN residual (the reference exits);
 * Npol >= 2. */
int cpsgpu_imp_res_lanczos(cpsgpu_dirac d, float *const *V, double *alpha, const cpsgpu_lanczos_arg *arg,
                           int *restarts);

/* Eigenvector cache: the reference's EigenCache list (util/eigen_container.h,
 * EigenCacheListSearch at :432; filled from disk by EigenContainer) as
 * named caches on the lattice, resident in device memory (FP32).  load:
 * neig float eigenvectors of d's half-checkerboard size in WILSON order and
 * their eigenvalues under name (a cache of the same name is replaced);
 * clear: drop every cache of the lattice. */
int cpsgpu_eigencache_load(cpsgpu_dirac d, const char *name, int neig, const float *const *evecs,
                           const double *evals);
int cpsgpu_eigencache_clear(cpsgpu_lattice lat);
/* DiracOp::InvLowModeApprox(out, in, fname_eig_root, neig)
 * (d_op_base/comsrc/inv_lowmode_approx.C:272-512, the path of a cache of
 * exactly neig vectors): out[i] = sum_k <v_k, in[i]> / lambda_k v_k for the
 * len sources, with lambda_k squared when ritz_mat_oper is MAT_HERM or
 * MATPC_HERM (CPSGPU_RITZ_*, RitzMatType values 1..9 accepted as the
 * reference does).  CPSGPU_ERR_ARG when no cache has this name and neig
 * (the reference exits).  The compressed-cache path (blockProj2) is not
 * part of this call. */
int cpsgpu_inv_lowmode_approx(cpsgpu_dirac d, double *const *out, const double *const *in, int len, const char *name,
                              int neig, int ritz_mat_oper);
/* DiracOp::InvEigCg(sol, src, true_res, nev, m, V, vec_len, M, U, invH,
 * def_len, restart, restart_len) (d_op_base/comsrc/inv_eig_cg.C:129-635):
 * CG on MatPcDagMatPc (FP64, arg->stop_rsd, arg->max_num_iter) from zero or
 * from the deflated guess U invH U^dag src, with the eigCG bookkeeping when
 * nev > 0 (m > 2 nev Lanczos vectors in V, restarted to 2 nev Ritz vectors;
 * on return V[0..2 nev) the last restart's Ritz vectors, M their Ritz
 * values, 0 past the rank) and deflated restarts at |r| < restart[i] |src|.
 * U: def_len FP32 deflation vectors; invH: (U^dag A U)^-1, complex,
 * row-major, (re, im) pairs.  *iterations = the reference's iter;
 * *true_res = |src - A sol| / |src|.  Unlike the reference's eigen_solver,
 * whose QL step leaves the eigenvectors uncomputed (eigen_solver.C:180-185),
 * the small eigenproblems here return true eigenvectors. */
int cpsgpu_inveigcg(cpsgpu_dirac d, double *sol, const double *src, const cpsgpu_cg_arg *arg, int nev, int m,
                    double *const *V, double *M, float *const *U, const double *invH, int def_len,
                    const double *restart, int restart_len, int *iterations, double *true_res);
/* DiracOp::MinResExt(psi, phi, v, vm, degree) (minresext.C:30-150): the
 * chronological initial guess psi for MatPcDagMatPc psi = phi from degree
 * previous solutions v[] (orthonormalised in place, as the reference does),
 * vm[i] = MatPcDagMatPc v[i] written; *error = |phi - A psi| / |phi| (the
 * reference prints it).  degree 0: psi = 0. */
int cpsgpu_minresext(cpsgpu_dirac d, double *psi, const double *phi, double *const *v, double *const *vm,
                     int degree, double *error);
/* DiracOpWilsonTypes::BiCGstab(psi, chi, chi_norm, n, true_res)
 * (bicgstab.C:35-229): BiCGstab(n) on MatPc itself (not the normal
 * equations), psi the initial guess, stop |r|^2 < stop_rsd^2 chi_norm with
 * arg->stop_rsd and arg->max_num_iter (chi_norm 0: computed).  *iterations
 * is the reference's k; *true_res = |r| (absolute, as the reference reports
 * it; 0 when not converged).  FP64 on the device; the solver's complex
 * scalars are host recurrences. */
int cpsgpu_bicgstab(cpsgpu_dirac d, double *psi, const double *chi, double chi_norm, int n, const cpsgpu_cg_arg *arg,
                    int *iterations, double *true_res);
/* DiracOp*::MatInv(out, in, true_res) with the CG inverter
 * (d_op_wilson.C:257-334, d_op_dwf.C:316-492, d_op_mobius.C:407-700, SYM2):
 * the solve on both checkerboards.  in and out hold 2 * 24*Ls*Vh reals in
 * the reference's order: Wilson and DWF [odd | even], Mobius [even | odd];
 * out's CG checkerboard (odd) is the initial guess.  The source is not
 * modified (PRESERVE_YES).  res describes the CG on the odd checkerboard. */
int cpsgpu_matinv(cpsgpu_dirac d, double *out, const double *in, const cpsgpu_cg_arg *arg, cpsgpu_cg_result *res);
/* InverterType values (include/alg/enum_int.h:707-716) MatInv takes */
#define CPSGPU_INV_CG 0
#define CPSGPU_INV_LOWMODEAPPROX 3
#define CPSGPU_INV_CG_LOWMODE_DEFL 4
/* MatInv with CgArg.Inverter LOWMODEAPPROX (the CG's solution replaced by
 * the low-mode approximation of InvLowModeApprox, from the cache eig_name
 * holding neig vectors; res: 0 iterations, true_res 0 as the reference
 * reports) or CG_LOWMODE_DEFL (that approximation as CG's initial guess):
 * d_op_dwf.C:468-476, d_op_mobius.C:566-590.  CG: as cpsgpu_matinv. */
int cpsgpu_matinv_lowmode(cpsgpu_dirac d, double *out, const double *in, const cpsgpu_cg_arg *arg, int inverter,
                          const char *eig_name, int neig, cpsgpu_cg_result *res);
/* DiracOp::MInvCG (minvcg.C:47-353): multishift CG on MatPcDagMatPc +
 * shift[k].  rsdcg[k] in: stop residuals, out: achieved residuals; returns
 * the iteration count through *iterations as the reference returns it.
 * precision CPSGPU_DOUBLE runs the reference's FP64 recurrences; SINGLE runs
 * them in FP32 and then refines every shift with FP64-true-residual CG to
 * rsdcg[k] (refine != 0). */
int cpsgpu_minvcg(cpsgpu_dirac d, double *const *psi, const double *chi, double chi_norm, const double *shift,
                  int nshift, double *rsdcg, int type, const double *alpha, int max_num_iter, int precision,
                  int refine, int *iterations);
/* Where the operator's last cpsgpu_minvcg spent its time (no counterpart in
 * the reference): host wall seconds of the source / guess upload, the
 * shifted recurrences, the FP64 refinement and the solutions' download
 * (each phase ends with a stream synchronisation), and the refinement's
 * iterations (largest over the shifts, and their sum). */
typedef struct {
  double upload_s, recurrence_s, refine_s, download_s;
  int refine_iterations_max, refine_iterations_sum;
} cpsgpu_minvcg_stats;
int cpsgpu_get_minvcg_stats(cpsgpu_dirac d, cpsgpu_minvcg_stats *stats);

/* ---- device-resident fields ---- */
int cpsgpu_field_create(cpsgpu_dirac d, int precision, int nrhs, cpsgpu_field *f);
int cpsgpu_field_destroy(cpsgpu_field f);
int cpsgpu_field_upload(cpsgpu_field f, const double *host);
int cpsgpu_field_download(cpsgpu_field f, double *host);
int cpsgpu_field_gaussian(cpsgpu_field f, unsigned long long seed);
/* out = dslash(in) (precision of the fields, which must match) */
int cpsgpu_dslash_field(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in, int cb, int dag);
int cpsgpu_mdagm_field(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in);

/* ---- t-slab domain decomposition of the dslash ----
 * Replaces the QMP halo exchange of wilson_dslash_vec
 * (d_op_wilson/qmp/wilson_dslash_vec.C:184-278, 486-493) for a lattice
 * split along t over nodes_t ranks (GJP.Nodes(3)), one slab per rank:
 * lat holds slab coor_t with its own node_sites (an even number of
 * t-slices) and its own links.  While partitioned, only these calls apply
 * the operator (every other operator, solver and the plaquette return
 * CPSGPU_ERR_STATE).  One dslash: pack the input's two t faces (FP64 or
 * FP32 fields) into device buffers of cpsgpu_dd_face_bytes each; move
 * to_prev to the previous rank's from_next and to_next to the next rank's
 * from_prev (periodically, by NCCL, peer copies or MPI: the caller's
 * transport); then cpsgpu_dslash_dd.  Faces are spin-projected half
 * spinors (12 reals per site and slice), the backward one already
 * multiplied by the sending slab's link, so no gauge halo is needed; the
 * antiperiodic t sign applies only at the lattice's own t ends.  Both calls
 * return once their kernels have finished. */
int cpsgpu_lattice_set_t_partition(cpsgpu_lattice lat, int nodes_t, int coor_t);
int cpsgpu_dd_face_bytes(cpsgpu_dirac d, int precision, int nrhs, size_t *bytes);
int cpsgpu_dslash_dd_pack(cpsgpu_dirac d, cpsgpu_field in, int cb, int dag, void *to_prev, void *to_next);
int cpsgpu_dslash_dd(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in, int cb, int dag, const void *from_next,
                     const void *from_prev);
/* cpsgpu_dslash_dd in two parts, so that the faces move while the device
 * computes (the local / non-local split of wilson_dslash_vec,
 * wilson_dslash_vec.C:184-278): _interior applies the hop to the slab's
 * t-slices 1 .. Lt-2, which read no halo, and returns as soon as it is
 * enqueued on lat's stream (call it after cpsgpu_dslash_dd_pack, before
 * the exchange); _boundary then applies it to the first and last t-slices,
 * reading the received faces, and returns once both parts have finished.
 * Together they write what cpsgpu_dslash_dd writes, bit for bit. */
int cpsgpu_dslash_dd_interior(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in, int cb, int dag);
int cpsgpu_dslash_dd_boundary(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in, int cb, int dag,
                              const void *from_next, const void *from_prev);
/* BLAS-1 on FP64 device fields (vector_util.C:727-922): out = a x + y
 * (fTimesV1PlusV2), and this rank's part of <a, b> = sum conj(a) b
 * (compDotProduct without its global sum: a decomposed solver adds the
 * ranks' parts, as glb_sum does).  Both return once done. */
int cpsgpu_field_axpby(cpsgpu_field out, double a, cpsgpu_field x, cpsgpu_field y);
int cpsgpu_field_dot(cpsgpu_field a, cpsgpu_field b, double *re, double *im);
/* No counterpart in the reference (whose solver loop runs on the host): a
 * decomposed solver that keeps its scalars on the device.  set_stream makes
 * every launch for lat go to the caller's CUDA stream (a cudaStream_t;
 * NULL restores the library's own stream, so the legacy default stream is
 * named cudaStreamLegacy), after synchronising the old one; while it is set, cpsgpu_dslash_dd_pack, cpsgpu_dslash_dd,
 * cpsgpu_dslash_dd_boundary and cpsgpu_field_axpby only enqueue (no host
 * synchronisation), so they order with the caller's own work on that
 * stream (face copies, NCCL collectives) and can be captured in a CUDA
 * graph.  field_dot_device writes this rank's <a, b> (re, im) to dev_out
 * (device memory, 2 doubles), and field_axpby_device computes
 * out = (scale * dev_a[0]) x + y with the coefficient read on the device;
 * both only enqueue. */
int cpsgpu_lattice_set_stream(cpsgpu_lattice lat, void *stream);
int cpsgpu_field_dot_device(cpsgpu_field a, cpsgpu_field b, double *dev_out);
int cpsgpu_field_axpby_device(cpsgpu_field out, const double *dev_a, double scale, cpsgpu_field x, cpsgpu_field y);
/* solve with FP64 fields already on the device (sol: initial guess in,
 * solution out); arg->precision selects plain or mixed CG */
int cpsgpu_invcg_field(cpsgpu_dirac d, cpsgpu_field sol, cpsgpu_field src, const cpsgpu_cg_arg *arg,
                       cpsgpu_cg_result *res);
/* n independent DiracOp::InvCg solves (InvCgShift, inv_cg.C:84-448) of
 * different operators (their own lattices, masses, kinds) as ONE CUDA graph
 * launch: every solve's iteration loop is a root branch of the graph, so the
 * systems run concurrently on the GPU and each stops at its own convergence.
 * The reference runs such solves one after another (FdwfBase::FmatEvlInv per
 * mass, f_dwf_base.C:189-275).  sol[k] (initial guesses in, solutions out)
 * and src[k] are FP64 device fields of ops[k]; args[k] its CgArg and
 * precision (mixed precision as cpsgpu_invcg).  An operator may appear once
 * per precision (several right-hand sides of one operator go in one field).
 * res holds one result per right-hand side, solve after solve. */
int cpsgpu_solve_batch(int n, const cpsgpu_dirac *ops, const cpsgpu_field *sol, const cpsgpu_field *src,
                       const cpsgpu_cg_arg *args, cpsgpu_cg_result *res);

/* ---- tuning ---- */
/* Time candidate block shapes of every hop kernel the operator uses, at
 * precision prec, and keep the fastest; with nrhs > 1 also the right-hand-
 * side tile.  Returns the number of tuned keys. */
int cpsgpu_autotune(cpsgpu_dirac d, int prec, int nrhs, int *tuned);
/* Right-hand-side tile of batched hops at precision prec (no counterpart in
 * the reference): consecutive thread blocks apply the same links to `tile`
 * solves before moving on.  get returns the tile a launch of nrhs right-hand
 * sides uses; set overrides the autotuner (0 restores the default). */
int cpsgpu_get_rhs_tile(cpsgpu_dirac d, int prec, int nrhs, int *tile);
int cpsgpu_set_rhs_tile(cpsgpu_dirac d, int prec, int tile);
/* Launch shape of the operator's non-mixing hop kernels at precision prec
 * and its current link form (no counterpart in the reference): `sites`
 * consecutive checkerboard sites x `slices` slices per block, and
 * `slices_per_thread` 1 or 2 (2: DWF at FP32 arithmetic, Ls a multiple of
 * 4 * slices — each thread computes two same-parity slices with shared
 * links), and the site order in which the grid's blocks take the lattice:
 * CPSGPU_ORDER_SLICES (consecutive blocks: every slice group of one block
 * of sites) or CPSGPU_ORDER_SITES (consecutive blocks: the site blocks of
 * one slice group, lexicographically).  get returns the shape in use; set
 * overrides the autotuner.  The shape table (like the autotuner's) is shared by every
 * operator of the same kind, Ls, precision and link form. */
enum { CPSGPU_ORDER_SLICES = 0, CPSGPU_ORDER_SITES = 1 };
int cpsgpu_get_hop_shape(cpsgpu_dirac d, int prec, int *sites, int *slices, int *slices_per_thread, int *order);
int cpsgpu_set_hop_shape(cpsgpu_dirac d, int prec, int sites, int slices, int slices_per_thread, int order);

/* ---- measurement ----
 * Time `reps` back-to-back launches of the operator's hop kernel
 * (Dslash for Wilson / DWF, the Wilson hop of every slice for Mobius) at
 * precision prec, with CUDA events on the library's stream.  The launches
 * rotate over enough distinct input/output fields that the working set
 * exceeds the L2 cache, so every launch streams from HBM.  Returns the mean
 * device time per launch and the algorithmic bytes one launch must move
 * (input and output spinors once, every link once). */
int cpsgpu_time_dslash(cpsgpu_dirac d, int prec, int cb, int dag, int reps, double *ms_per_launch,
                       double *bytes_per_launch);
/* Same for one MatPcDagMatPc application (all its kernels); bytes counts
 * every kernel's compulsory traffic. */
int cpsgpu_time_mdagm(cpsgpu_dirac d, int prec, int reps, double *ms_per_apply, double *bytes_per_apply);
/* Same for the Mobius M5^-1 alone (zmobius_m5inv, zmobius_m5inv.C:534):
 * the dense Ls x Ls contraction per chirality on the CUDA cores; bytes =
 * input and output spinors once. */
int cpsgpu_time_m5inv(cpsgpu_dirac d, int prec, int reps, double *ms_per_apply, double *bytes_per_apply);

/* ---- pinned host memory for fast host<->device copies ---- */
int cpsgpu_host_alloc(size_t bytes, void **ptr);
int cpsgpu_host_free(void *ptr);

/* ---- seeded synthetic inputs (host code, no GPU needed) ---- */
/* U = exp(i width H), H a Gaussian Hermitian traceless 3x3 per link, then
 * reunitarised to SU(3); written in WILSON order without boundary signs.
 * Deterministic in (seed, site, mu). */
int cpsgpu_gen_gauge(const int node_sites[4], unsigned long long seed, double width, double *u_wilson);
/* n unit-variance Gaussian reals, deterministic in (seed, stream, index) */
int cpsgpu_gen_gaussian(double *out, long n, unsigned long long seed, unsigned int stream);

#ifdef __cplusplus
}
#endif
#endif
