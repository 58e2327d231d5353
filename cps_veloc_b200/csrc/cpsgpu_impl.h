// Host-side structures of the library behind the C ABI (include/cpsgpu.h).
#pragma once
#include <complex>
#include <cuda_runtime.h>
#include <stdexcept>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "fields.cuh"
#include "reduce.cuh"

namespace cpsgpu {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CPSGPU_CUDA(call)                                                                   \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      throw ::cpsgpu::Error(-3, std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

// Owning device allocation.
struct DeviceBuffer {
  void *ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t n) { alloc(n); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
  DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
    if (this != &o) { release(); ptr = o.ptr; bytes = o.bytes; o.ptr = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DeviceBuffer() { release(); }
  void alloc(size_t n) {
    release();
    if (n) CPSGPU_CUDA(cudaMalloc(&ptr, n));
    bytes = n;
  }
  void ensure(size_t n) { if (n > bytes) alloc(n); }
  void release() { if (ptr) cudaFree(ptr); ptr = nullptr; bytes = 0; }
  template <typename T> T *as() const { return reinterpret_cast<T *>(ptr); }
};

// A fermion field in one precision: nrhs x ls slices of vh sites.
struct Field {
  int prec = PREC_DOUBLE;
  long vh = 0;
  int ls = 1, nrhs = 1;
  DeviceBuffer data, norm;
  Field() = default;
  Field(int p, long vh_, int ls_, int nrhs_) { create(p, vh_, ls_, nrhs_); }
  void create(int p, long vh_, int ls_, int nrhs_);
  size_t site_bytes() const;
  size_t sites() const { return (size_t)vh * ls * nrhs; }
  SpinorView view() const {
    SpinorView v;
    v.data = data.ptr;
    v.norm = norm.as<float>();
    v.vh = vh;
    v.ls = ls;
    v.nrhs = nrhs;
    return v;
  }
  // view of right-hand side k alone
  SpinorView view_rhs(int k) const;
};

enum DiracKind { KIND_WILSON = 0, KIND_DWF = 1, KIND_MOBIUS = 2 };

struct EigenCacheDev;  // lowmode.cu

struct Lattice {
  int L[4];
  long vh;
  double bc[4];
  int device = 0;
  cudaStream_t stream = nullptr;       // where every launch for this lattice goes
  cudaStream_t own_stream = nullptr;   // the library's stream, created with the lattice
  bool caller_stream = false;          // stream is the caller's (cpsgpu_lattice_set_stream)
  // gauge field copies: FP64 full and compressed, FP32 and FP16 compressed
  DeviceBuffer gD18, gD12, gS12, gH12;
  DeviceBuffer gS18, gH18;  // full-link FP32 / FP16 copies (fields.cuh LinkIO<.., 18>)
  bool have_gauge = false;
  double recon_err = 0.0;  // max |row2 - conj(row0 x row1)| over all links
  bool use_recon12 = true; // FP64 operator reads 12-real links
  DeviceBuffer staging;    // CPS-order host mirror on the device
  DeviceBuffer partials;   // per-block reduction partials
  DeviceBuffer scratch_st; // SolverScalars for operator-only reductions
  double *pinned = nullptr;  // small pinned host buffer for scalars
  std::vector<std::shared_ptr<EigenCacheDev>> eig_caches;  // named low-mode caches (lowmode.cu)
  int t_nodes = 1, t_coor = 0;  // t-slab decomposition: this lattice is slab t_coor of t_nodes (dd.cu)
  Lattice(const int L_[4], const double bc_[4]);
  ~Lattice();
  GaugeView gauge(int prec) const;
  // reals per stored link a precision reads: FP64 uses 12 when the links are
  // SU(3); FP32 / FP16 use sloppy_recon[prec] (12 or 18, set by the autotuner;
  // the FP16 operator may also read FP32 links, LINK_F32_12 / LINK_F32_18)
  int sloppy_recon[3] = {12, 18, 18};
  int recon(int prec) const {
    if (prec == PREC_DOUBLE) return use_recon12 ? 12 : 18;
    return sloppy_recon[prec];
  }
};

struct OpWork {
  Field t1, t2, t0, t3;  // operator temporaries, one precision
};

// Mobius preconditionings (GJP.ZMobius_PC_Type, dwf.h:42-48)
enum MobiusPc { PC_ORIG = 0, PC_SYM1 = 1, PC_SYM2 = 2, PC_SYM1_MIT = 3, PC_SYM2_MIT = 4, PC_SYM3 = 5 };
// MatPc (plan[0]) or MatPc^dagger (plan[1]) of a Mobius operator as
//   out = X + Last W_cb0( Mid W_cb1( Pre in ) ),   X = in, or Xmix in,
// every matrix s-local ([2][ls][ls] per chirality, the layout of the mixing
// kernels); a null Pre / Xmix is the identity, a null Last the scalar coef.
struct MobiusPlan {
  const double *pre = nullptr, *mid = nullptr, *last = nullptr, *xmix = nullptr;
  double coef = 0.0;
};

// Multishift CG workspace (multishift.cu), kept across calls on one operator.
struct CgSolver;
// an instantiated graph and the configuration it was captured for
struct CachedGraph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  long long body_kernels = 0;  // kernels of one body of its WHILE node
  std::vector<long long> counts;  // kernels of the graph's other parts (its builder's bookkeeping)
  std::vector<long long> key;
  CachedGraph() = default;
  CachedGraph(const CachedGraph &) = delete;
  CachedGraph &operator=(const CachedGraph &) = delete;
  ~CachedGraph() { drop(); }
  void drop() {
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    ge = nullptr;
    g = nullptr;
    key.clear();
  }
};

struct MsWork {
  Field chi, r, tmp;
  std::vector<Field> p, psi;
  DeviceBuffer st, ms, pv, psiv;
  OpWork w;
  // the recurrences' loop: a WHILE node over chunks of iterations, ctl its
  // [bodies run, bound] counters
  CachedGraph loop;
  // the FP32 recurrences and the FP64 refinement of every shift as one graph
  CachedGraph full;
  DeviceBuffer ctl;
  // the batched refinement solver of the sloppy path, kept with its fields
  // and its instantiated graph while the number of shifts stays the same
  std::shared_ptr<CgSolver> refine;
  int refine_n = 0;
  // the last call's phases: wall seconds and refinement iterations
  double upload_s = 0, recurrence_s = 0, refine_s = 0, download_s = 0;
  int refine_max = 0, refine_sum = 0;
};

struct Dirac {
  Lattice *lat;
  int kind;
  int ls;
  double mass, m5, b, c;
  double a5inv = 1.0;  // DoArg.dwf_a5_inv: the fifth-direction inverse lattice spacing
  double kappa;  // Wilson kappa, DWF kappa_5, Mobius kappa_b
  double kappa_c;
  // Mobius s-mixing matrices, each [2][ls][ls] (upper, lower chirality):
  //   P = B M5inv, Q = B M5inv kappa_b, R = kappa_b M5inv^+ B^+ (-kappa_b),
  //   S = M5inv^+ B^+, and the pieces B, B^+, M5inv, M5inv^+ on their own.
  DeviceBuffer mixP, mixQ, mixR, mixS, mixB, mixBd, mixM5i, mixM5id, mixM5;
  // 1 + a5inv K D5: the fifth-direction term of the unpreconditioned Mat
  // (mobius_dslash_5_plus weights the hop by a5inv, d_op_mobius.C:735-795)
  DeviceBuffer mixM5a;
  // complex per-slice b_s, c_s (zMobius): every matrix above is complex,
  // stored [2][ls][ls][re, im], and the -kappa_b(s) of MatPc is the complex
  // diagonal mixKb applied in a mixing epilogue
  bool cplx = false;
  bool uniform_bc = true;  // the same b, c on every slice
  DeviceBuffer mixKb;
  std::vector<double> hM5i, hM5id, hB, hBd;  // host copies of the packed M5^-1 and B matrices
  // host copy of every real mixing matrix uploaded for this operator, by
  // device address (launch_mix passes the matrix as a kernel parameter)
  std::unordered_map<const void *, std::vector<double>> mix_host;
  Dirac(Lattice *l, int kind_, int ls_, double mass_, double m5_, double b_, double c_, double a5inv_ = 1.0);
  // (re)build the Mobius matrices from per-slice coefficients
  void build_mobius(const std::vector<std::complex<double>> &bs, const std::vector<std::complex<double>> &cs);
  // right-hand sides per hop tile (consecutive blocks share links across
  // this many solves), per precision, set by the autotuner; 0 = untuned
  int rtile[3] = {0, 0, 0};
  // the standalone Ls x Ls mixings of FP16 fields on the tensor cores
  // (mix_tc.cu) instead of the CUDA cores
  bool mix_tc = false;
  // the register-tiled mixing kernel (mix_reg.cu) where it applies; off:
  // the shared-memory kernel (blas.cu)
  bool mix_reg = true;
  // the bulk-copy staged kernel (mix_bulk.cu) for FP16 fields where it applies
  bool mix_bulk = true;
  DeviceBuffer mixTcFrag;  // the tensor-core form's A fragments of the matrix being applied
  // the preconditioning of MatPc (Mobius) and its two plans; the matrices
  // of the non-SYM2 forms live in pc_bufs
  int pc_type = PC_SYM2;
  MobiusPlan plan[2];
  std::vector<DeviceBuffer> pc_bufs;
  void set_pc_type(int pc);
  MsWork ms;  // multishift workspace
  int rhs_tile(int prec, int nrhs) const {
    const int t = rtile[prec];
    return t > 0 ? t : (nrhs < 4 ? nrhs : 4);
  }
};

// ---- kernels / launchers (hop.cu, blas.cu) ----
// Launch one hop with epilogue; see hop.cuh for the meaning of each field.
struct HopLaunch {
  int prec = PREC_DOUBLE;   // hop precision
  int pr = PREC_DOUBLE;     // r/p precision (CG/RES)
  int px = PREC_DOUBLE;     // sol precision (CG)
  int ep = 0;
  int cb = 0, dag = 0;
  int norm = 0, red_op = 0, gate = 0;
  const double *mix = nullptr;
  std::vector<double> coef;  // per slice
  const void *halo_fwd = nullptr, *halo_bwd = nullptr;  // t halos of a decomposed lattice (dd.cu)
  int sub = 0;  // HopSub: all sites, or (decomposed lattice) the interior or the two t-end slices
  double *partials = nullptr;  // the reduction's per-block partials (null: the lattice's buffer)
};
void launch_hop(const Dirac &D, const HopLaunch &L, const SpinorView &in, const SpinorView &out,
                const SpinorView &x, const SpinorView &r, const SpinorView &sol, const SpinorView &p,
                const SpinorView &b, SolverScalars *st);

// Everything of the Mobius MatPc (dag 0) or MatPc^dagger (dag 1) before its
// last hop (D.plan[dag]: the pre-mixing, the first hop with its mixing, the
// X term): the caller launches out = x + Last W_cb0(hop_in) with the
// epilogue it needs (mix = Last, or the scalar coef when mix is null).
// Lh carries precision, gate and partials; uses w.t0, w.t1, w.t3.
struct MobiusTail {
  SpinorView hop_in, x;
  const double *mix;
  double coef;
};
MobiusTail mobius_head(const Dirac &D, int prec, int dag, const SpinorView &in, OpWork &w, HopLaunch Lh,
                       SolverScalars *st);

// the tensor-core form of launch_mix (mix_tc.cu): FP16 fields, real
// matrices, Ls <= 16
bool mix_tc_applies(const Dirac &D, int prec);
void launch_mix_tc(const Dirac &D, const double *mix, const SpinorView &in, const SpinorView &out,
                   const SolverScalars *st, int gate);
// out = Mix in (per chirality Ls x Ls), all slices
// the register-tiled form of launch_mix (mix_reg.cu): real matrices whose
// host copy is in D.mix_host and Ls among the instantiated sizes; false when
// it does not apply
bool launch_mix_reg(const Dirac &D, int prec, const double *mix, const SpinorView &in, const SpinorView &out,
                    const SolverScalars *st, int gate);
// the bulk-copy staged form (mix_bulk.cu): FP16 fields, real matrices,
// vh a multiple of 32, Ls 8, 10, 12 or 16; false when it does not apply
bool launch_mix_bulk(const Dirac &D, int prec, const double *mix, const SpinorView &in, const SpinorView &out,
                     const SolverScalars *st, int gate);
int mix_bulk_error();  // nonzero once a bounded wait of the bulk kernel ran out (the read clears it)
void launch_mix(const Dirac &D, int prec, const double *mix, const SpinorView &in, const SpinorView &out,
                const SolverScalars *st = nullptr, int gate = 0);

// vector kernels
// out = a x + y and f *= a, FP64 fields
void launch_axpby(cudaStream_t s, const SpinorView &out, double a, const SpinorView &x, const SpinorView &y);
void launch_axpby_dev(cudaStream_t s, const SpinorView &out, const double *a, double scale, const SpinorView &x,
                      const SpinorView &y);
void launch_scale(cudaStream_t s, double a, const SpinorView &f);
void launch_convert(cudaStream_t s, int pdst, const SpinorView &dst, int psrc, const SpinorView &src);
void launch_zero(cudaStream_t s, const Field &f);
// p = r + beta p (gated on st->done)
void launch_xpay(cudaStream_t s, int prec, const SpinorView &p, const SpinorView &r, SolverScalars *st, int nrhs);
// x64 += xs; xs = 0 (gated on st->reliable)
void launch_accum_reliable(cudaStream_t s, const SpinorView &x64, int pxs, const SpinorView &xs, SolverScalars *st, int nrhs,
                           int force);
// |f|^2 (+ finalize op)
void launch_norm(cudaStream_t s, int prec, const SpinorView &f, SolverScalars *st, double *partials, int op, int gate);
// sum the per-block partials (nv values each, nblk blocks per solve) of the
// preceding reducing kernel and update each solve's scalars with op
void launch_finalize(cudaStream_t s, int nv, const double *partials, SolverScalars *st, int op, unsigned nblk,
                     int nsolves, int gate);
// st[k] <- value (host-side init through a kernel so graphs can replay it)
void launch_init_scalars(cudaStream_t s, SolverScalars *st, int nrhs, const SolverScalars &init);

// CPS order <-> device layout
void launch_import_fermion(cudaStream_t s, int prec, const SpinorView &dst, const double *staging);
void launch_export_fermion(cudaStream_t s, int prec, const SpinorView &src, double *staging);
void import_gauge(Lattice &L, const double *host_wilson_order, int signs_applied);

// operators (operators.cu)
void op_dslash(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int cb, int dag);
void op_matpc(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int dag, OpWork &w,
              SolverScalars *st, int norm, int red_op);
void op_mdagm(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, OpWork &w,
              SolverScalars *st, int red_op_dot);
// fullops.cu: the unpreconditioned operators on both checkerboards (halves 0
// and 1 in the reference's full-vector order) and the shifted Mobius
// MatPcDagMatPc (st->sum[0] = |MatPc in|^2 when st is given)
void op_mat(const Dirac &D, int prec, const SpinorView &out0, const SpinorView &out1, const SpinorView &in0,
            const SpinorView &in1, int dag, OpWork &w);
void op_mat_herm(const Dirac &D, int prec, const SpinorView &out0, const SpinorView &out1, const SpinorView &in0,
                 const SpinorView &in1, OpWork &w);
void op_mdagm_shift(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, double mu, OpWork &w,
                    SolverScalars *st);
void op_mobius_dslash4(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int cb, int dag,
                       OpWork &w);
void op_mobius_m5inv(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int dag);

// DiracOp::Ritz parameters (krylov.cu)
struct RitzArgs {
  double RsdR_a, RsdR_r, Rsdlam, Cutl_zero, Cv_fact;
  int n_renorm, Kalk_Sim, N_min, N_max, MaxCG, ProjApsiP, neg;
};

// t-slab domain decomposition (dd.cu)
size_t dd_face_bytes(const Dirac &D, int prec, int nrhs);
void dd_pack(const Dirac &D, int prec, const SpinorView &in, int cb, int dag, void *to_prev, void *to_next);
// sub: 0 every site, 1 the interior t-slices (no halos read; may run while
// the faces move), 2 the first and last t-slices (reading the halos)
void dd_dslash(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int cb, int dag,
               const void *from_next, const void *from_prev, int sub = 0);
void field_dot(Lattice &L, const SpinorView &a, const SpinorView &b, double *re, double *im);
void field_dot_device(Lattice &L, const SpinorView &a, const SpinorView &b, double *dev_out);

// low-mode deflation (lowmode.cu)
void eigencache_store(Lattice &L, const std::string &name, std::vector<Field> &&evecs, const double *evals);
void eigencache_clear(Lattice &L);
void inv_lowmode_approx(Dirac &D, const std::vector<SpinorView> &out, const std::vector<SpinorView> &in,
                        const std::string &name, int neig, bool square);

// DiracOp::ImpResLanczos (krylov.cu): LanczosArg with the Chebyshev filter's
// MatrixPolynomialArg; neg_*: RitzMatOper NEG_MATPCDAG_MATPC for the filter /
// the convergence check
struct LanczosArgs {
  int neg_lanczos, neg_conv, nk, nt, np, maxiters, conv_check, Npol;
  double stop_res, p0, p1, eigen_shift;
};

// HMC fermion force (force.cu): CalcHmdForceVecs' four half fields and the
// force loop of EvolveMomFforce on a CANONICAL momentum field in device memory
struct ForceVecs {
  Field v1o, v1e, v2o, v2e;
  Field t1, t2;  // Mobius temporaries
  OpWork w;
};
void calc_hmd_force_vecs(const Dirac &D, ForceVecs &fv, const SpinorView &chi);
void fforce_update(const Dirac &D, const ForceVecs &fv, double *mom, double dt, double out[3]);
double fforce_bytes(const Dirac &D);
// plaquette and link-trace sums of the resident links (gauge.cu) and of a
// CANONICAL host field (nersc.cpp)
void gauge_sums(Lattice &L, double *sum_plaq, double *sum_link);
void host_gauge_sums(const int L[4], const double *u, double *sum_plaq, double *sum_link);
// ForceArg of a whole momentum field (per-link Matrix::norm) and mom += x
void mom_norms(Lattice &L, const double *mom, double out[3]);
void mom_add(Lattice &L, double *mom, const double *x);

// kernels enqueued by this library (graph replays counted by the solver)
long long &launch_counter();

// workspace sizing helper
void ensure_field(Field &f, int prec, long vh, int ls, int nrhs);

}  // namespace cpsgpu
