// The C ABI (include/cpsgpu.h): argument checking, object lifetimes,
// host <-> device staging in CPS storage order, and error translation.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cpsgpu.h"
#include "cpsgpu_impl.h"
#include "hop.cuh"
#include "tune.h"
#include "solver.h"

namespace cpsgpu {
void gen_gauge(const int L[4], uint64_t seed, double width, double *out);
void gen_gaussian(double *out, long n, uint64_t seed, unsigned stream);
int autotune(Dirac &D, int prec, int nrhs);
double time_dslash(Dirac &D, int prec, int cb, int dag, int reps, double *bytes);
double time_mdagm(Dirac &D, int prec, int reps, double *bytes);
double time_m5inv(Dirac &D, int prec, int reps, double *bytes);
double matpc_dag_matpc_noalloc(const Dirac &D, double *out, const double *in);
int bicgstab(Dirac &D, Field &psi, const Field &chi, double chi_norm, int nn, double stop_rsd, int max_num_iter,
             double *true_res);
void fconvert(const int node_sites[4], int ls, double *f, int to, int from);
void minresext(Dirac &D, Field &psi, const Field &phi, std::vector<Field> &v, std::vector<Field> &vm,
               double *error);
int ritz(Dirac &D, std::vector<Field> &psi_all, int N_eig, const RitzArgs &ra, double *lambda_out);
int jacobi(Dirac &D, std::vector<Field> &psi, int N_eig, double *lambda, std::vector<std::complex<double>> &off,
           double Toler, int N_max);
int ritz_eig(Dirac &D, std::vector<Field> &psi, const RitzArgs &ra0, int N_KS_max, double *lambda_H,
             int *valid_eig);
int imp_res_lanczos(Dirac &D, std::vector<Field> &V, double *alpha, const LanczosArgs &a);
int inveigcg(Dirac &D, Field &sol, const Field &src, double stop_rsd, int max_iter, int nev, int m,
             std::vector<Field> &V, double *M, std::vector<Field> &U, const std::vector<std::complex<double>> &invH,
             const double *restart, int restart_len, double *true_res);
void nersc_read(const char *path, const int node_sites[4], double *u, cpsgpu_nersc_header *hdr);
void nersc_write(const char *path, const int node_sites[4], const double *u, int recon_row_3, int fp_format,
                 const cpsgpu_nersc_header *meta, cpsgpu_nersc_header *out);
void gconvert(const int node_sites[4], double *u, int to, int from);
void four2five(const int node_sites[4], int ls, double *five, const double *four, int s_u, int s_l, int ncb);
void five2four(const int node_sites[4], int ls, double *four, const double *five, int s_u, int s_l, int ncb);
void fconvert_device(const Lattice &lat, int ls, double *dst, const double *src, int to, int from);
void gconvert_device(const Lattice &lat, double *dst, const double *src, int to, int from);
void four2five_device(const Lattice &lat, int ls, double *five, const double *four, int s_u, int s_l, int ncb);
void five2four_device(const Lattice &lat, int ls, double *four, const double *five, int s_u, int s_l, int ncb);
int minvcg(Dirac &D, double *const *psi, const double *chi, double chi_norm, const double *shift, int nshift,
           double *rsdcg, int type, const double *alpha, int max_num_iter, int precision, int refine);
}  // namespace cpsgpu

using namespace cpsgpu;

struct cpsgpu_lattice_s {
  std::unique_ptr<Lattice> L;
};

struct cpsgpu_dirac_s {
  cpsgpu_lattice_s *lat;
  std::unique_ptr<Dirac> D;
  // host-path workspace
  Field in[3], out[3];
  OpWork w[3];
  std::unique_ptr<CgSolver> solvers[3];
  // both checkerboards of the full-vector operators (in 0, in 1, out 0, out 1)
  std::unique_ptr<Field[]> full;
  // HMC force workspace: CalcHmdForceVecs' fields and the momentum field
  std::unique_ptr<ForceVecs> fv;
  DeviceBuffer mom;
};

struct cpsgpu_field_s {
  cpsgpu_dirac_s *d;
  Field f;
};

namespace {
// the operator's instantiated graphs (CG solvers, the multishift loop and its
// refinement) hold the launches of the form they were captured for: after a
// change of matrices, kernels or launch shapes they are captured again
void drop_captured(cpsgpu_dirac_s *d) {
  for (auto &s : d->solvers) s.reset();
  d->D->ms.refine.reset();
  d->D->ms.refine_n = 0;
  d->D->ms.loop.drop();
  d->D->ms.full.drop();
}
}  // namespace

namespace {
thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

template <typename F>
int guarded(F &&f) {
  try {
    g_err.clear();
    return f();
  } catch (const Error &e) {
    return fail(e.code, e.what());
  } catch (const std::exception &e) {
    return fail(CPSGPU_ERR_STATE, e.what());
  }
}

int check_prec(int p) {
  if (p != CPSGPU_DOUBLE && p != CPSGPU_SINGLE && p != CPSGPU_HALF) throw Error(CPSGPU_ERR_ARG, "bad precision");
  return p;
}

size_t vec_reals(const cpsgpu_dirac_s *d) { return (size_t)24 * d->D->ls * d->D->lat->vh; }

// upload a CPS-order host vector (nrhs copies at `stride` reals apart, or an
// array of pointers) into f
void upload(Lattice &L, Field &f, const double *const *host, int nrhs) {
  size_t n = (size_t)24 * f.vh * f.ls;
  L.staging.ensure(n * nrhs * sizeof(double));
  for (int k = 0; k < nrhs; k++)
    CPSGPU_CUDA(cudaMemcpyAsync(L.staging.as<double>() + n * k, host[k], n * sizeof(double), cudaMemcpyHostToDevice,
                                L.stream));
  launch_import_fermion(L.stream, f.prec, f.view(), L.staging.as<double>());
}

void download(Lattice &L, const Field &f, double *const *host, int nrhs) {
  size_t n = (size_t)24 * f.vh * f.ls;
  L.staging.ensure(n * nrhs * sizeof(double));
  launch_export_fermion(L.stream, f.prec, f.view(), L.staging.as<double>());
  for (int k = 0; k < nrhs; k++)
    CPSGPU_CUDA(cudaMemcpyAsync(host[k], L.staging.as<double>() + n * k, n * sizeof(double), cudaMemcpyDeviceToHost,
                                L.stream));
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
}

void need_gauge(const cpsgpu_dirac_s *d) {
  if (!d->D->lat->have_gauge) throw Error(CPSGPU_ERR_STATE, "no gauge field imported");
  if (d->D->lat->t_nodes > 1)
    throw Error(CPSGPU_ERR_STATE, "t-partitioned lattice: only the decomposed dslash (cpsgpu_dslash_dd) applies");
}

void ensure_partials(Lattice &L, int ls, int nrhs) {
  size_t nblk = (size_t)((L.vh + 31) / 32) * ls + 1024;
  L.partials.ensure(nblk * 2 * nrhs * sizeof(double));
}

CgArgs to_args(const cpsgpu_cg_arg *a) {
  CgArgs c;
  c.stop_rsd = a->stop_rsd;
  c.max_num_iter = a->max_num_iter;
  c.src_norm_sq = a->src_norm_sq;
  c.shift = a->shift;
  // reliable-update threshold: measured on DWF 16^3x32, Ls=16, the FP32 inner
  // solve is fastest at 0.01 (fewer FP64 updates, no extra iterations), the
  // FP16 one at 0.1 (smaller values inflate its iteration count)
  c.delta = a->delta > 0 ? a->delta : (a->precision == CPSGPU_SINGLE ? 0.01 : 0.1);
  c.chunk = a->chunk > 0 ? a->chunk : 8;
  c.use_graph = a->use_graph;
  return c;
}

void to_result(const CgResult &r, cpsgpu_cg_result *o) {
  o->iterations = r.iterations;
  o->status = r.status;
  o->true_res = r.true_res;
  o->reliable_updates = r.reliable_updates;
  o->seconds = r.seconds;
  o->kernels = r.kernels;
}

CgSolver &solver_for(cpsgpu_dirac_s *d, int prec, int nrhs) {
  auto &s = d->solvers[prec];
  if (!s) s.reset(new CgSolver(*d->D, prec));
  if (s->nrhs != nrhs || !s->b64.data.ptr) s->setup(nrhs);
  return *s;
}
}  // namespace

extern "C" {

const char *cpsgpu_version(void) { return "cpsgpu 0.1 (sm_100a)"; }
const char *cpsgpu_last_error(void) { return g_err.c_str(); }

int cpsgpu_device_count(int *count) {
  return guarded([&] {
    if (!count) throw Error(CPSGPU_ERR_ARG, "null count");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    *count = (e == cudaSuccess) ? n : 0;
    if (e != cudaSuccess) cudaGetLastError();
    return CPSGPU_OK;
  });
}

int cpsgpu_set_device(int device) {
  return guarded([&] {
    CPSGPU_CUDA(cudaSetDevice(device));
    return CPSGPU_OK;
  });
}

int cpsgpu_finalize(void) {
  return guarded([&] {
    CPSGPU_CUDA(cudaDeviceSynchronize());
    tune_clear();
    return CPSGPU_OK;
  });
}

int cpsgpu_lattice_create(const int node_sites[4], const int bc[4], cpsgpu_lattice *lat) {
  return guarded([&] {
    if (!node_sites || !bc || !lat) throw Error(CPSGPU_ERR_ARG, "null argument");
    double b[4];
    for (int k = 0; k < 4; k++) {
      if (bc[k] != 1 && bc[k] != -1) throw Error(CPSGPU_ERR_ARG, "bc must be +1 or -1");
      b[k] = bc[k];
    }
    auto *l = new cpsgpu_lattice_s;
    try {
      l->L.reset(new Lattice(node_sites, b));
    } catch (...) {
      delete l;
      throw;
    }
    *lat = l;
    return CPSGPU_OK;
  });
}

int cpsgpu_lattice_destroy(cpsgpu_lattice lat) {
  return guarded([&] {
    delete lat;
    return CPSGPU_OK;
  });
}

int cpsgpu_import_gauge(cpsgpu_lattice lat, const double *u, int signs_applied) {
  return guarded([&] {
    if (!lat || !u) throw Error(CPSGPU_ERR_ARG, "null argument");
    import_gauge(*lat->L, u, signs_applied);
    return CPSGPU_OK;
  });
}

int cpsgpu_gauge_info(cpsgpu_lattice lat, double *recon_err, int *recon12) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    if (recon_err) *recon_err = lat->L->recon_err;
    if (recon12) *recon12 = lat->L->use_recon12 ? 1 : 0;
    return CPSGPU_OK;
  });
}

int cpsgpu_set_link_reals(cpsgpu_lattice lat, int prec, int reals) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    if (prec != CPSGPU_SINGLE && prec != CPSGPU_HALF) throw Error(CPSGPU_ERR_ARG, "FP32 or FP16 only");
    const bool f32 = (reals == CPSGPU_LINKS_F32_12 || reals == CPSGPU_LINKS_F32_18);
    if (reals != 12 && reals != 18 && !(f32 && prec == CPSGPU_HALF))
      throw Error(CPSGPU_ERR_ARG, "reals must be 12 or 18 (or FP32 links for the FP16 operator)");
    lat->L->sloppy_recon[prec] = reals;
    return CPSGPU_OK;
  });
}

int cpsgpu_get_link_reals(cpsgpu_lattice lat, int prec, int *reals) {
  return guarded([&] {
    if (!lat || !reals) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (prec != CPSGPU_SINGLE && prec != CPSGPU_HALF) throw Error(CPSGPU_ERR_ARG, "FP32 or FP16 only");
    *reals = lat->L->sloppy_recon[prec];
    return CPSGPU_OK;
  });
}

// ---- gauge configurations (gauge.cu, nersc.cpp)
int cpsgpu_gauge_plaquette(cpsgpu_lattice lat, double *plaq, double *link_trace) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    Lattice &L = *lat->L;
    if (!L.have_gauge) throw Error(CPSGPU_ERR_STATE, "no gauge field imported");
    double sp = 0.0, sl = 0.0;
    gauge_sums(L, &sp, &sl);
    const double vol = 2.0 * (double)L.vh;
    if (plaq) *plaq = sp / (18.0 * vol);
    if (link_trace) *link_trace = sl / (12.0 * vol);
    return CPSGPU_OK;
  });
}

int cpsgpu_nersc_read(const char *path, const int node_sites[4], double *u, cpsgpu_nersc_header *hdr) {
  return guarded([&] {
    nersc_read(path, node_sites, u, hdr);
    return CPSGPU_OK;
  });
}

int cpsgpu_nersc_write(const char *path, const int node_sites[4], const double *u, int recon_row_3, int fp_format,
                       const cpsgpu_nersc_header *meta, cpsgpu_nersc_header *out) {
  return guarded([&] {
    nersc_write(path, node_sites, u, recon_row_3, fp_format, meta, out);
    return CPSGPU_OK;
  });
}

int cpsgpu_lattice_load_nersc(cpsgpu_lattice lat, const char *path, double check_precision, cpsgpu_nersc_header *hdr,
                              double *plaq) {
  return guarded([&] {
    if (!lat || !path) throw Error(CPSGPU_ERR_ARG, "null argument");
    Lattice &L = *lat->L;
    const long vol = 2 * L.vh;
    std::vector<double> u((size_t)vol * 72);
    cpsgpu_nersc_header h;
    nersc_read(path, L.L, u.data(), &h);
    gconvert(L.L, u.data(), CPSGPU_STR_WILSON, CPSGPU_STR_CANONICAL);
    import_gauge(L, u.data(), 0);
    double sp = 0.0;
    gauge_sums(L, &sp, nullptr);
    const double p = sp / (18.0 * (double)vol);
    if (plaq) *plaq = p;
    if (hdr) *hdr = h;
    if (std::fabs((p - h.plaquette) / p) > check_precision) {
      char msg[128];
      std::snprintf(msg, sizeof msg, "plaquette check failed: computed %.10g, header %.10g", p, h.plaquette);
      throw Error(CPSGPU_ERR_ARG, msg);
    }
    return CPSGPU_OK;
  });
}

// ---- host-side storage orders (convert.cpp)
int cpsgpu_fconvert(const int node_sites[4], int ls, double *f, int to, int from) {
  return guarded([&] {
    fconvert(node_sites, ls, f, to, from);
    return CPSGPU_OK;
  });
}

int cpsgpu_gconvert(const int node_sites[4], double *u, int to, int from) {
  return guarded([&] {
    gconvert(node_sites, u, to, from);
    return CPSGPU_OK;
  });
}

int cpsgpu_four2five(const int node_sites[4], int ls, double *five, const double *four, int s_u, int s_l, int ncb) {
  return guarded([&] {
    four2five(node_sites, ls, five, four, s_u, s_l, ncb);
    return CPSGPU_OK;
  });
}

int cpsgpu_five2four(const int node_sites[4], int ls, double *four, const double *five, int s_u, int s_l, int ncb) {
  return guarded([&] {
    five2four(node_sites, ls, four, five, s_u, s_l, ncb);
    return CPSGPU_OK;
  });
}

int cpsgpu_fconvert_device(cpsgpu_lattice lat, int ls, double *dst, const double *src, int to, int from) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    fconvert_device(*lat->L, ls, dst, src, to, from);
    return CPSGPU_OK;
  });
}

int cpsgpu_gconvert_device(cpsgpu_lattice lat, double *dst, const double *src, int to, int from) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    gconvert_device(*lat->L, dst, src, to, from);
    return CPSGPU_OK;
  });
}

int cpsgpu_four2five_device(cpsgpu_lattice lat, int ls, double *five, const double *four, int s_u, int s_l, int ncb) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    four2five_device(*lat->L, ls, five, four, s_u, s_l, ncb);
    return CPSGPU_OK;
  });
}

int cpsgpu_five2four_device(cpsgpu_lattice lat, int ls, double *four, const double *five, int s_u, int s_l, int ncb) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    five2four_device(*lat->L, ls, four, five, s_u, s_l, ncb);
    return CPSGPU_OK;
  });
}

int cpsgpu_synchronize(cpsgpu_lattice lat) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    CPSGPU_CUDA(cudaStreamSynchronize(lat->L->stream));
    return CPSGPU_OK;
  });
}

int cpsgpu_dirac_create(cpsgpu_lattice lat, const cpsgpu_dirac_arg *a, cpsgpu_dirac *d) {
  return guarded([&] {
    if (!lat || !a || !d) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (a->kind < CPSGPU_WILSON || a->kind > CPSGPU_MOBIUS) throw Error(CPSGPU_ERR_ARG, "unknown fermion kind");
    auto *o = new cpsgpu_dirac_s;
    o->lat = lat;
    try {
      o->D.reset(new Dirac(lat->L.get(), a->kind, a->ls, a->mass, a->m5, a->mobius_b, a->mobius_c,
                           a->a5_inv != 0.0 ? a->a5_inv : 1.0));
      ensure_partials(*lat->L, o->D->ls, 1);
    } catch (...) {
      delete o;
      throw;
    }
    *d = o;
    return CPSGPU_OK;
  });
}

int cpsgpu_dirac_set_zmobius(cpsgpu_dirac d, const double *b, const double *c) {
  return guarded([&] {
    if (!d || !b || !c) throw Error(CPSGPU_ERR_ARG, "null argument");
    Dirac &D = *d->D;
    if (D.kind != KIND_MOBIUS) throw Error(CPSGPU_ERR_ARG, "complex b_s, c_s: Mobius operators only");
    if (D.pc_type != PC_SYM2) throw Error(CPSGPU_ERR_ARG, "per-slice b_s, c_s: SYM2 preconditioning only");
    std::vector<std::complex<double>> bs(D.ls), cs(D.ls);
    for (int s = 0; s < D.ls; s++) {
      bs[s] = {b[2 * s], b[2 * s + 1]};
      cs[s] = {c[2 * s], c[2 * s + 1]};
    }
    CPSGPU_CUDA(cudaStreamSynchronize(D.lat->stream));  // no launch may still read the old matrices
    D.build_mobius(bs, cs);
    drop_captured(d);  // captured graphs hold the old matrices
    return CPSGPU_OK;
  });
}

int cpsgpu_dirac_destroy(cpsgpu_dirac d) {
  return guarded([&] {
    delete d;
    return CPSGPU_OK;
  });
}

int cpsgpu_dirac_info(cpsgpu_dirac d, double *kappa, double *kappa_c) {
  return guarded([&] {
    if (!d) throw Error(CPSGPU_ERR_ARG, "null operator");
    if (kappa) *kappa = d->D->kappa;
    if (kappa_c) *kappa_c = d->D->kappa_c;
    return CPSGPU_OK;
  });
}

// ---- host-vector operators
int cpsgpu_dslash(cpsgpu_dirac d, double *out, const double *in, int cb, int dag, int prec) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    if ((cb != 0 && cb != 1) || (dag != 0 && dag != 1)) throw Error(CPSGPU_ERR_ARG, "cb and dag must be 0 or 1");
    check_prec(prec);
    need_gauge(d);
    if (d->D->kind == KIND_MOBIUS) throw Error(CPSGPU_ERR_ARG, "Mobius: use cpsgpu_mobius_dslash_4");
    Lattice &L = *d->D->lat;
    ensure_field(d->in[prec], prec, L.vh, d->D->ls, 1);
    ensure_field(d->out[prec], prec, L.vh, d->D->ls, 1);
    upload(L, d->in[prec], &in, 1);
    op_dslash(*d->D, prec, d->out[prec].view(), d->in[prec].view(), cb, dag);
    download(L, d->out[prec], &out, 1);
    return CPSGPU_OK;
  });
}

int cpsgpu_matpc(cpsgpu_dirac d, double *out, const double *in, int dag, int prec) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    check_prec(prec);
    need_gauge(d);
    Lattice &L = *d->D->lat;
    ensure_field(d->in[prec], prec, L.vh, d->D->ls, 1);
    ensure_field(d->out[prec], prec, L.vh, d->D->ls, 1);
    upload(L, d->in[prec], &in, 1);
    op_matpc(*d->D, prec, d->out[prec].view(), d->in[prec].view(), dag ? 1 : 0, d->w[prec], nullptr, 0, 0);
    download(L, d->out[prec], &out, 1);
    return CPSGPU_OK;
  });
}

int cpsgpu_matpc_dag_matpc(cpsgpu_dirac d, double *out, const double *in, double *dot, int prec) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    check_prec(prec);
    need_gauge(d);
    Lattice &L = *d->D->lat;
    ensure_field(d->in[prec], prec, L.vh, d->D->ls, 1);
    ensure_field(d->out[prec], prec, L.vh, d->D->ls, 1);
    upload(L, d->in[prec], &in, 1);
    SolverScalars *st = L.scratch_st.as<SolverScalars>();
    CPSGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(SolverScalars), L.stream));
    op_mdagm(*d->D, prec, d->out[prec].view(), d->in[prec].view(), d->w[prec], st, RED_STORE);
    download(L, d->out[prec], &out, 1);
    if (dot) {
      SolverScalars h;
      CPSGPU_CUDA(cudaMemcpy(&h, st, sizeof(h), cudaMemcpyDeviceToHost));
      *dot = h.sum[0];
    }
    return CPSGPU_OK;
  });
}

namespace {
// a full vector's halves in the reference's order: [odd][even] (Wilson,
// DWF), [even][odd] (Mobius); the library's fields hold one checkerboard
void full_op(cpsgpu_dirac d, double *out, const double *in, int which, int dag) {
  if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
  need_gauge(d);
  Dirac &D = *d->D;
  Lattice &L = *D.lat;
  const int prec = PREC_DOUBLE;
  if (!d->full) d->full.reset(new Field[4]);
  Field *f = d->full.get();
  for (int k = 0; k < 4; k++) ensure_field(f[k], prec, L.vh, D.ls, 1);
  const size_t half = (size_t)24 * L.vh * D.ls;
  const double *h0 = in, *h1 = in + half;
  upload(L, f[0], &h0, 1);
  upload(L, f[1], &h1, 1);
  if (which == 0) op_mat(D, prec, f[2].view(), f[3].view(), f[0].view(), f[1].view(), dag, d->w[prec]);
  else op_mat_herm(D, prec, f[2].view(), f[3].view(), f[0].view(), f[1].view(), d->w[prec]);
  double *o0 = out, *o1 = out + half;
  download(L, f[2], &o0, 1);
  download(L, f[3], &o1, 1);
}
}  // namespace

int cpsgpu_mat(cpsgpu_dirac d, double *out, const double *in, int dag) {
  return guarded([&] {
    if (dag != 0 && dag != 1) throw Error(CPSGPU_ERR_ARG, "dag must be 0 or 1");
    full_op(d, out, in, 0, dag);
    return CPSGPU_OK;
  });
}

int cpsgpu_mat_herm(cpsgpu_dirac d, double *out, const double *in) {
  return guarded([&] {
    full_op(d, out, in, 1, 0);
    return CPSGPU_OK;
  });
}

int cpsgpu_matpc_dag_matpc_shift(cpsgpu_dirac d, double *out, const double *in, double mu, double *dot, int prec) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    check_prec(prec);
    need_gauge(d);
    if (d->D->kind != KIND_MOBIUS) throw Error(CPSGPU_ERR_ARG, "MatPcDagMatPcShift: Mobius operators only");
    Lattice &L = *d->D->lat;
    ensure_field(d->in[prec], prec, L.vh, d->D->ls, 1);
    ensure_field(d->out[prec], prec, L.vh, d->D->ls, 1);
    upload(L, d->in[prec], &in, 1);
    SolverScalars *st = L.scratch_st.as<SolverScalars>();
    CPSGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(SolverScalars), L.stream));
    op_mdagm_shift(*d->D, prec, d->out[prec].view(), d->in[prec].view(), mu, d->w[prec], st);
    download(L, d->out[prec], &out, 1);
    if (dot) {
      SolverScalars h;
      CPSGPU_CUDA(cudaMemcpy(&h, st, sizeof(h), cudaMemcpyDeviceToHost));
      *dot = h.sum[0];
    }
    return CPSGPU_OK;
  });
}

int cpsgpu_matpc_dag_matpc_noalloc(cpsgpu_dirac d, double *out_dev, const double *in_dev, double *dot) {
  return guarded([&] {
    if (!d || !out_dev || !in_dev) throw Error(CPSGPU_ERR_ARG, "null argument");
    need_gauge(d);
    const double r = matpc_dag_matpc_noalloc(*d->D, out_dev, in_dev);
    if (dot) *dot = r;
    return CPSGPU_OK;
  });
}

int cpsgpu_mobius_dslash_4(cpsgpu_dirac d, double *out, const double *in, int cb, int dag, int prec) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    if ((cb != 0 && cb != 1) || (dag != 0 && dag != 1)) throw Error(CPSGPU_ERR_ARG, "cb and dag must be 0 or 1");
    check_prec(prec);
    need_gauge(d);
    Lattice &L = *d->D->lat;
    ensure_field(d->in[prec], prec, L.vh, d->D->ls, 1);
    ensure_field(d->out[prec], prec, L.vh, d->D->ls, 1);
    upload(L, d->in[prec], &in, 1);
    op_mobius_dslash4(*d->D, prec, d->out[prec].view(), d->in[prec].view(), cb, dag, d->w[prec]);
    download(L, d->out[prec], &out, 1);
    return CPSGPU_OK;
  });
}

int cpsgpu_mobius_m5inv(cpsgpu_dirac d, double *out, const double *in, int dag, int prec) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    check_prec(prec);
    Lattice &L = *d->D->lat;
    ensure_field(d->in[prec], prec, L.vh, d->D->ls, 1);
    ensure_field(d->out[prec], prec, L.vh, d->D->ls, 1);
    upload(L, d->in[prec], &in, 1);
    op_mobius_m5inv(*d->D, prec, d->out[prec].view(), d->in[prec].view(), dag ? 1 : 0);
    download(L, d->out[prec], &out, 1);
    return CPSGPU_OK;
  });
}

// ---- solvers
void cpsgpu_cg_arg_default(cpsgpu_cg_arg *a) {
  if (!a) return;
  a->stop_rsd = 1e-8;
  a->max_num_iter = 10000;
  a->src_norm_sq = 0.0;
  a->shift = 0.0;
  a->precision = CPSGPU_DOUBLE;
  a->delta = 0.0;
  a->chunk = 8;
  a->use_graph = 1;
}

int cpsgpu_invcg_multi(cpsgpu_dirac d, double *const *sol, const double *const *src, int nrhs,
                       const cpsgpu_cg_arg *arg, cpsgpu_cg_result *res) {
  return guarded([&] {
    if (!d || !sol || !src || !arg || !res || nrhs < 1) throw Error(CPSGPU_ERR_ARG, "bad argument");
    if (nrhs > 64) throw Error(CPSGPU_ERR_ARG, "at most 64 right-hand sides per call");
    if (arg->max_num_iter < 1) throw Error(CPSGPU_ERR_ARG, "max_num_iter must be >= 1");
    for (int k = 0; k < nrhs; k++)
      if (!sol[k] || !src[k]) throw Error(CPSGPU_ERR_ARG, "null vector");
    check_prec(arg->precision);
    need_gauge(d);
    Lattice &L = *d->D->lat;
    CgSolver &S = solver_for(d, arg->precision, nrhs);
    upload(L, S.b64, src, nrhs);
    upload(L, S.x64, sol, nrhs);
    std::vector<CgResult> r;
    S.run(to_args(arg), r);
    download(L, S.x64, sol, nrhs);
    for (int k = 0; k < nrhs; k++) to_result(r[k], res + k);
    return CPSGPU_OK;
  });
}

int cpsgpu_invcg(cpsgpu_dirac d, double *sol, const double *src, const cpsgpu_cg_arg *arg, cpsgpu_cg_result *res) {
  return cpsgpu_invcg_multi(d, &sol, &src, 1, arg, res);
}

// DiracOp*::MatInv with the CG inverter, both checkerboards on the device.
//   Wilson / DWF (d_op_wilson.C:257-334, d_op_dwf.C:316-492), halves [odd | even]:
//     temp = kappa Dslash(in_e, CHKB_EVEN) + in_o;  b = MatPcDag temp;  CG;
//     out_e = kappa Dslash(out_o, CHKB_ODD) + in_e
//   Mobius (d_op_mobius.C:407-700), halves [even | odd]:
//     temp = kappa_b Dslash_4(M5^-1 in_e, CHKB_EVEN) + in_o;  SYM1: temp <- M5^-1 temp;
//     SYM2, SYM3: guess out_o <- M5 out_o;  b = MatPcDag temp;  CG;
//     SYM2, SYM3: out_o <- M5^-1 out_o;
//     out_e = M5^-1 (kappa_b Dslash_4(out_o, CHKB_ODD) + in_e);  out *= 2 kappa_b
//   (the MIT preconditionings: not implemented, as in the reference)
namespace {
// DiracOp*::MatInv for Inverter CG, LOWMODEAPPROX or CG_LOWMODE_DEFL
// (d_op_dwf.C:316-500, d_op_mobius.C:407-620); eig_name / neig: the
// low-mode cache of the last two
int matinv_impl(cpsgpu_dirac d, double *out, const double *in, const cpsgpu_cg_arg *arg, cpsgpu_cg_result *res,
                int inverter, const char *eig_name, int neig) {
  return guarded([&] {
    if (!d || !out || !in || !arg || !res) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (inverter != CPSGPU_INV_CG && inverter != CPSGPU_INV_LOWMODEAPPROX && inverter != CPSGPU_INV_CG_LOWMODE_DEFL)
      throw Error(CPSGPU_ERR_UNSUPPORTED, "InverterType not implemented");
    if (inverter != CPSGPU_INV_CG && !eig_name) throw Error(CPSGPU_ERR_ARG, "null eigenvector cache name");
    if (arg->max_num_iter < 1) throw Error(CPSGPU_ERR_ARG, "max_num_iter must be >= 1");
    check_prec(arg->precision);
    need_gauge(d);
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    const cudaStream_t s = L.stream;
    const size_t half = vec_reals(d);
    const bool mob = (D.kind == KIND_MOBIUS);
    if (D.cplx) throw Error(CPSGPU_ERR_ARG, "MatInv: real Mobius coefficients only");
    // the CG's checkerboard and the other one, as the reference orders them
    const double *in_cg = mob ? in + half : in, *in_other = mob ? in : in + half;
    double *out_cg = mob ? out + half : out, *out_other = mob ? out : out + half;
    Field fo(PREC_DOUBLE, L.vh, D.ls, 1), t1(PREC_DOUBLE, L.vh, D.ls, 1), t2(PREC_DOUBLE, L.vh, D.ls, 1);
    OpWork &w = d->w[PREC_DOUBLE];
    CgSolver &S = solver_for(d, arg->precision, 1);
    upload(L, fo, &in_other, 1);  // in_e
    upload(L, t2, &in_cg, 1);     // in_o
    if (!mob) {
      op_dslash(D, PREC_DOUBLE, t1.view(), fo.view(), 0, 0);
      launch_axpby(s, t1.view(), D.kappa, t1.view(), t2.view());
    } else {
      if (D.pc_type == PC_SYM1_MIT || D.pc_type == PC_SYM2_MIT)
        throw Error(CPSGPU_ERR_UNSUPPORTED, "MatInv: the MIT preconditionings are not implemented (d_op_mobius.C:477-495)");
      op_mobius_m5inv(D, PREC_DOUBLE, t1.view(), fo.view(), 0);
      Field t3(PREC_DOUBLE, L.vh, D.ls, 1);
      op_mobius_dslash4(D, PREC_DOUBLE, t3.view(), t1.view(), 0, 0, w);
      launch_axpby(s, t1.view(), D.kappa, t3.view(), t2.view());
      if (D.pc_type == PC_SYM1) {  // SYM1: the source gets M5^-1 (d_op_mobius.C:519-530)
        op_mobius_m5inv(D, PREC_DOUBLE, t3.view(), t1.view(), 0);
        CPSGPU_CUDA(cudaMemcpyAsync(t1.data.ptr, t3.data.ptr, t1.data.bytes, cudaMemcpyDeviceToDevice, s));
      }
    }
    op_matpc(D, PREC_DOUBLE, S.b64.view(), t1.view(), 1, w, nullptr, 0, 0);
    std::vector<CgResult> r;
    if (inverter == CPSGPU_INV_CG) {
      upload(L, S.x64, &out_cg, 1);
      if (mob && (D.pc_type == PC_SYM2 || D.pc_type == PC_SYM3)) {  // guess: x <- M5 x (d_op_mobius.C:498-515)
        launch_mix(D, PREC_DOUBLE, D.mixM5.as<double>(), S.x64.view(), t1.view());
        CPSGPU_CUDA(cudaMemcpyAsync(S.x64.data.ptr, t1.data.ptr, t1.data.bytes, cudaMemcpyDeviceToDevice, s));
      }
    } else {
      // the low-mode part of (MatPcDagMatPc)^-1 applied to MatPcDag in_o
      inv_lowmode_approx(D, {S.x64.view()}, {S.b64.view()}, eig_name, neig, false);
    }
    if (inverter != CPSGPU_INV_LOWMODEAPPROX) {
      S.run(to_args(arg), r);
    } else {
      // no CG: the reference reports true_res = 0 (dirac_op.h:96-106)
      CgResult lm;
      lm.iterations = 0;
      lm.status = CPSGPU_CONVERGED;
      lm.true_res = 0.0;
      r.push_back(lm);
    }
    if (!mob) {
      op_dslash(D, PREC_DOUBLE, t1.view(), S.x64.view(), 1, 0);
      launch_axpby(s, t2.view(), D.kappa, t1.view(), fo.view());
      download(L, S.x64, &out_cg, 1);
      download(L, t2, &out_other, 1);
    } else {
      // out_o: M5^-1 x for SYM2 / SYM3, x itself for ORIG / SYM1 (d_op_mobius.C:627-663)
      if (D.pc_type == PC_SYM2 || D.pc_type == PC_SYM3) op_mobius_m5inv(D, PREC_DOUBLE, t1.view(), S.x64.view(), 0);
      else CPSGPU_CUDA(cudaMemcpyAsync(t1.data.ptr, S.x64.data.ptr, t1.data.bytes, cudaMemcpyDeviceToDevice, s));
      op_mobius_dslash4(D, PREC_DOUBLE, t2.view(), t1.view(), 1, 0, w);
      launch_axpby(s, t2.view(), D.kappa, t2.view(), fo.view());
      op_mobius_m5inv(D, PREC_DOUBLE, fo.view(), t2.view(), 0);     // out_e
      launch_scale(s, 2.0 * D.kappa, t1.view());
      launch_scale(s, 2.0 * D.kappa, fo.view());
      download(L, t1, &out_cg, 1);
      download(L, fo, &out_other, 1);
    }
    to_result(r[0], res);
    return CPSGPU_OK;
  });
}
}  // namespace

int cpsgpu_matinv(cpsgpu_dirac d, double *out, const double *in, const cpsgpu_cg_arg *arg, cpsgpu_cg_result *res) {
  return matinv_impl(d, out, in, arg, res, CPSGPU_INV_CG, nullptr, 0);
}

int cpsgpu_matinv_lowmode(cpsgpu_dirac d, double *out, const double *in, const cpsgpu_cg_arg *arg, int inverter,
                          const char *eig_name, int neig, cpsgpu_cg_result *res) {
  return matinv_impl(d, out, in, arg, res, inverter, eig_name, neig);
}

namespace {
ForceVecs &force_vecs(cpsgpu_dirac d, const double *chi) {
  Dirac &D = *d->D;
  Lattice &L = *D.lat;
  if (D.kind == KIND_MOBIUS && D.cplx) throw Error(CPSGPU_ERR_ARG, "the fermion force is built for real Mobius b, c");
  if (D.kind == KIND_MOBIUS && D.pc_type != PC_SYM2)
    throw Error(CPSGPU_ERR_UNSUPPORTED, "the fermion force is built for the SYM2 preconditioning");
  if (!d->fv) d->fv.reset(new ForceVecs());
  ensure_field(d->in[PREC_DOUBLE], PREC_DOUBLE, L.vh, D.ls, 1);
  upload(L, d->in[PREC_DOUBLE], &chi, 1);
  calc_hmd_force_vecs(D, *d->fv, d->in[PREC_DOUBLE].view());
  return *d->fv;
}
}  // namespace

int cpsgpu_calc_hmd_force_vecs(cpsgpu_dirac d, double *f_out, double *f_in, const double *chi) {
  return guarded([&] {
    if (!d || !f_out || !f_in || !chi) throw Error(CPSGPU_ERR_ARG, "null argument");
    need_gauge(d);
    ForceVecs &fv = force_vecs(d, chi);
    Lattice &L = *d->D->lat;
    const size_t half = (size_t)24 * L.vh * d->D->ls;
    // WILSON order of the halves: [odd][even] (Wilson, DWF), [even][odd] (Mobius)
    const bool mob = d->D->kind == KIND_MOBIUS;
    double *o1 = mob ? f_out + half : f_out, *e1 = mob ? f_out : f_out + half;
    double *o2 = mob ? f_in + half : f_in, *e2 = mob ? f_in : f_in + half;
    download(L, fv.v1o, &o1, 1);
    download(L, fv.v1e, &e1, 1);
    download(L, fv.v2o, &o2, 1);
    download(L, fv.v2e, &e2, 1);
    return CPSGPU_OK;
  });
}

int cpsgpu_evolve_mom_fforce(cpsgpu_dirac d, double *mom, const double *chi, double dt, cpsgpu_force_arg *out) {
  return guarded([&] {
    if (!d || !mom || !chi) throw Error(CPSGPU_ERR_ARG, "null argument");
    need_gauge(d);
    ForceVecs &fv = force_vecs(d, chi);
    Lattice &L = *d->D->lat;
    const size_t bytes = (size_t)2 * L.vh * 4 * 18 * sizeof(double);
    d->mom.ensure(2 * bytes);
    CPSGPU_CUDA(cudaMemcpyAsync(d->mom.ptr, mom, bytes, cudaMemcpyHostToDevice, L.stream));
    double f[3];
    fforce_update(*d->D, fv, d->mom.as<double>(), dt, f);
    CPSGPU_CUDA(cudaMemcpyAsync(mom, d->mom.ptr, bytes, cudaMemcpyDeviceToHost, L.stream));
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    if (out) {
      out->L1 = f[0];
      out->L2 = f[1];
      out->Linf = f[2];
    }
    return CPSGPU_OK;
  });
}

int cpsgpu_rhmc_evolve_mom_fforce(cpsgpu_dirac d, double *mom, const double *const *sol, int degree,
                                  const double *alpha, double dt, int force_measure, cpsgpu_force_arg *out) {
  return guarded([&] {
    if (!d || !mom || (degree > 0 && (!sol || !alpha))) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (degree < 0) throw Error(CPSGPU_ERR_ARG, "degree must be >= 0");
    for (int k = 0; k < degree; k++)
      if (!sol[k]) throw Error(CPSGPU_ERR_ARG, "null solution vector");
    need_gauge(d);
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    if (D.kind == KIND_MOBIUS && D.cplx) throw Error(CPSGPU_ERR_ARG, "the fermion force is built for real Mobius b, c");
    if (D.kind == KIND_MOBIUS && D.pc_type != PC_SYM2)
      throw Error(CPSGPU_ERR_UNSUPPORTED, "the fermion force is built for the SYM2 preconditioning");
    const size_t bytes = (size_t)2 * L.vh * 4 * 18 * sizeof(double);
    d->mom.ensure(2 * bytes);
    double *m = d->mom.as<double>(), *tmp = m + bytes / sizeof(double);
    CPSGPU_CUDA(cudaMemcpyAsync(m, mom, bytes, cudaMemcpyHostToDevice, L.stream));
    // FORCE_MEASURE_YES: the poles accumulate into a zeroed field whose norms
    // are measured before it is added to mom (f_wilson.C:689-757)
    double *acc = force_measure ? tmp : m;
    if (force_measure) CPSGPU_CUDA(cudaMemsetAsync(tmp, 0, bytes, L.stream));
    for (int k = 0; k < degree; k++) {
      ForceVecs &fv = force_vecs(d, sol[k]);
      fforce_update(D, fv, acc, dt * alpha[k], nullptr);
    }
    double f[3] = {0.0, 0.0, 0.0};
    if (force_measure) {
      mom_norms(L, tmp, f);
      mom_add(L, m, tmp);
    }
    CPSGPU_CUDA(cudaMemcpyAsync(mom, m, bytes, cudaMemcpyDeviceToHost, L.stream));
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    if (out) {
      out->L1 = f[0];
      out->L2 = f[1];
      out->Linf = f[2];
    }
    return CPSGPU_OK;
  });
}

int cpsgpu_time_fforce(cpsgpu_dirac d, int reps, double *ms_total, double *ms_kernel, double *kernel_bytes) {
  return guarded([&] {
    if (!d || reps < 1) throw Error(CPSGPU_ERR_ARG, "bad argument");
    need_gauge(d);
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    if (D.kind == KIND_MOBIUS && D.cplx) throw Error(CPSGPU_ERR_ARG, "the fermion force is built for real Mobius b, c");
    if (D.kind == KIND_MOBIUS && D.pc_type != PC_SYM2)
      throw Error(CPSGPU_ERR_UNSUPPORTED, "the fermion force is built for the SYM2 preconditioning");
    if (!d->fv) d->fv.reset(new ForceVecs());
    Field chi(PREC_DOUBLE, L.vh, D.ls, 1);
    std::vector<double> h((size_t)24 * L.vh * D.ls);
    gen_gaussian(h.data(), (long)h.size(), 20261203ull, 9);
    const double *hp = h.data();
    upload(L, chi, &hp, 1);
    const size_t bytes = (size_t)2 * L.vh * 4 * 18 * sizeof(double);
    d->mom.ensure(bytes);
    CPSGPU_CUDA(cudaMemsetAsync(d->mom.ptr, 0, bytes, L.stream));
    cudaEvent_t e[3];
    for (auto &x : e) CPSGPU_CUDA(cudaEventCreate(&x));
    float t_all = 0.f, t_k = 0.f;
    for (int k = 0; k < reps + 2; k++) {
      CPSGPU_CUDA(cudaEventRecord(e[0], L.stream));
      calc_hmd_force_vecs(D, *d->fv, chi.view());
      CPSGPU_CUDA(cudaEventRecord(e[1], L.stream));
      fforce_update(D, *d->fv, d->mom.as<double>(), 0.01, nullptr);
      CPSGPU_CUDA(cudaEventRecord(e[2], L.stream));
      CPSGPU_CUDA(cudaEventSynchronize(e[2]));
      float a = 0.f, b = 0.f;
      CPSGPU_CUDA(cudaEventElapsedTime(&a, e[0], e[2]));
      CPSGPU_CUDA(cudaEventElapsedTime(&b, e[1], e[2]));
      if (k >= 2) {
        t_all += a;
        t_k += b;
      }
    }
    for (auto &x : e) cudaEventDestroy(x);
    if (ms_total) *ms_total = t_all / reps;
    if (ms_kernel) *ms_kernel = t_k / reps;
    if (kernel_bytes) *kernel_bytes = fforce_bytes(D);
    return CPSGPU_OK;
  });
}

int cpsgpu_ritz(cpsgpu_dirac d, double *const *psi_all, int N_eig, const cpsgpu_ritz_arg *arg, double *lambda,
                int *iterations) {
  int status = CPSGPU_OK;
  const int rc = guarded([&] {
    if (!d || !psi_all || !arg) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (N_eig < 1) throw Error(CPSGPU_ERR_ARG, "N_eig must be >= 1");
    if (arg->n_renorm < 1) throw Error(CPSGPU_ERR_ARG, "n_renorm must be >= 1");
    for (int k = 0; k < N_eig; k++)
      if (!psi_all[k]) throw Error(CPSGPU_ERR_ARG, "null vector");
    need_gauge(d);
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    std::vector<Field> f(N_eig);
    for (int k = 0; k < N_eig; k++) {
      f[k].create(PREC_DOUBLE, L.vh, D.ls, 1);
      const double *h = psi_all[k];
      upload(L, f[k], &h, 1);
    }
    RitzArgs ra{arg->RsdR_a, arg->RsdR_r, arg->Rsdlam, arg->Cutl_zero, arg->Cv_fact, arg->n_renorm,
                arg->Kalk_Sim, arg->N_min, arg->N_max, arg->MaxCG, arg->ProjApsiP, arg->neg};
    double lam = 0.0;
    const int k = ritz(D, f, N_eig, ra, &lam);
    double *h = psi_all[N_eig - 1];
    download(L, f[N_eig - 1], &h, 1);
    if (lambda) *lambda = lam;
    if (iterations) *iterations = k < 0 ? arg->MaxCG : k;
    if (k < 0) status = CPSGPU_MAX_ITER;
    return CPSGPU_OK;
  });
  return rc != CPSGPU_OK ? rc : status;
}

namespace {
std::vector<Field> upload_all(cpsgpu_dirac d, double *const *v, int n) {
  Dirac &D = *d->D;
  Lattice &L = *D.lat;
  std::vector<Field> f(n);
  for (int k = 0; k < n; k++) {
    if (!v[k]) throw Error(CPSGPU_ERR_ARG, "null vector");
    f[k].create(PREC_DOUBLE, L.vh, D.ls, 1);
    const double *h = v[k];
    upload(L, f[k], &h, 1);
  }
  return f;
}
void download_all(cpsgpu_dirac d, std::vector<Field> &f, double *const *v) {
  Lattice &L = *d->D->lat;
  for (size_t k = 0; k < f.size(); k++) {
    double *h = v[k];
    download(L, f[k], &h, 1);
  }
}
}  // namespace

int cpsgpu_jacobi(cpsgpu_dirac d, double *const *psi, int N_eig, double *lambda, double *off_diag, double toler,
                  int n_max, int *sweeps) {
  int status = CPSGPU_OK;
  const int rc = guarded([&] {
    if (!d || !psi || !lambda || (N_eig > 1 && !off_diag)) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (N_eig < 1) throw Error(CPSGPU_ERR_ARG, "N_eig must be >= 1");
    need_gauge(d);
    std::vector<Field> f = upload_all(d, psi, N_eig);
    std::vector<std::complex<double>> off((size_t)N_eig * (N_eig - 1) / 2);
    for (size_t k = 0; k < off.size(); k++) off[k] = {off_diag[2 * k], off_diag[2 * k + 1]};
    const int k = jacobi(*d->D, f, N_eig, lambda, off, toler, n_max);
    download_all(d, f, psi);
    for (size_t q = 0; q < off.size(); q++) {
      off_diag[2 * q] = off[q].real();
      off_diag[2 * q + 1] = off[q].imag();
    }
    if (sweeps) *sweeps = k;
    if (k < 0) status = CPSGPU_MAX_ITER;
    return CPSGPU_OK;
  });
  return rc != CPSGPU_OK ? rc : status;
}

int cpsgpu_ritz_eig(cpsgpu_dirac d, double *const *psi, int N_eig, const cpsgpu_ritz_arg *arg, int N_KS_max,
                    double *lambda_H, int *valid_eig, int *iterations) {
  int status = CPSGPU_OK;
  const int rc = guarded([&] {
    if (!d || !psi || !arg || !lambda_H || !valid_eig) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (N_eig < 1) throw Error(CPSGPU_ERR_ARG, "N_eig must be >= 1");
    if (arg->n_renorm < 1) throw Error(CPSGPU_ERR_ARG, "n_renorm must be >= 1");
    need_gauge(d);
    std::vector<Field> f = upload_all(d, psi, N_eig);
    RitzArgs ra{arg->RsdR_a, arg->RsdR_r, arg->Rsdlam, arg->Cutl_zero, arg->Cv_fact, arg->n_renorm,
                arg->Kalk_Sim, arg->N_min, arg->N_max, arg->MaxCG, arg->ProjApsiP, arg->neg};
    const int r = ritz_eig(*d->D, f, ra, N_KS_max, lambda_H, valid_eig);
    download_all(d, f, psi);
    if (iterations) *iterations = r;
    if (r < 0) status = CPSGPU_MAX_ITER;
    return CPSGPU_OK;
  });
  return rc != CPSGPU_OK ? rc : status;
}

int cpsgpu_eigencache_load(cpsgpu_dirac d, const char *name, int neig, const float *const *evecs,
                           const double *evals) {
  return guarded([&] {
    if (!d || !name || (neig > 0 && (!evecs || !evals))) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (neig < 0 || neig > 65535) throw Error(CPSGPU_ERR_ARG, "need 0 <= neig <= 65535");
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    const size_t nreal = (size_t)24 * L.vh * D.ls;
    std::vector<Field> f(neig);
    Field f64(PREC_DOUBLE, L.vh, D.ls, 1);
    std::vector<double> h(nreal);
    for (int k = 0; k < neig; k++) {
      if (!evecs[k]) throw Error(CPSGPU_ERR_ARG, "null eigenvector");
      for (size_t q = 0; q < nreal; q++) h[q] = (double)evecs[k][q];
      const double *hp = h.data();
      upload(L, f64, &hp, 1);
      f[k].create(PREC_SINGLE, L.vh, D.ls, 1);
      launch_convert(L.stream, PREC_SINGLE, f[k].view(), PREC_DOUBLE, f64.view());
    }
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    eigencache_store(L, name, std::move(f), evals);
    return CPSGPU_OK;
  });
}

int cpsgpu_eigencache_clear(cpsgpu_lattice lat) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    eigencache_clear(*lat->L);
    return CPSGPU_OK;
  });
}

int cpsgpu_inv_lowmode_approx(cpsgpu_dirac d, double *const *out, const double *const *in, int len, const char *name,
                              int neig, int ritz_mat_oper) {
  return guarded([&] {
    if (!d || !name || (len > 0 && (!out || !in))) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (len < 0 || neig < 0 || neig > 65535) throw Error(CPSGPU_ERR_ARG, "need len >= 0, 0 <= neig <= 65535");
    if (ritz_mat_oper < 1 || ritz_mat_oper > 9)
      throw Error(CPSGPU_ERR_UNSUPPORTED, "RitzMatOper not implemented (inv_lowmode_approx.C:329-346)");
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    std::vector<Field> fin(len), fout(len);
    for (int i = 0; i < len; i++) {
      if (!in[i] || !out[i]) throw Error(CPSGPU_ERR_ARG, "null vector");
      fin[i].create(PREC_DOUBLE, L.vh, D.ls, 1);
      fout[i].create(PREC_DOUBLE, L.vh, D.ls, 1);
      upload(L, fin[i], &in[i], 1);
    }
    const bool square = (ritz_mat_oper == CPSGPU_RITZ_MAT_HERM || ritz_mat_oper == CPSGPU_RITZ_MATPC_HERM);
    std::vector<SpinorView> vo(len), vi(len);
    for (int i = 0; i < len; i++) {
      vo[i] = fout[i].view();
      vi[i] = fin[i].view();
    }
    inv_lowmode_approx(D, vo, vi, name, neig, square);
    for (int i = 0; i < len; i++) {
      double *o = out[i];
      download(L, fout[i], &o, 1);
    }
    return CPSGPU_OK;
  });
}

int cpsgpu_imp_res_lanczos(cpsgpu_dirac d, float *const *V, double *alpha, const cpsgpu_lanczos_arg *arg,
                           int *restarts) {
  int status = CPSGPU_OK;
  const int rc = guarded([&] {
    if (!d || !V || !alpha || !arg) throw Error(CPSGPU_ERR_ARG, "null argument");
    Dirac &D = *d->D;
    if (D.kind == KIND_WILSON)
      throw Error(CPSGPU_ERR_UNSUPPORTED, "RitzMat(V*,V*,MP*) is not implemented for Wilson fermions");
    const int nk = arg->nk_lanczos_vectors, nt = arg->nt_lanczos_vectors, np = arg->np_lanczos_vectors;
    if (nk < 2 || nt < 1 || nt > nk || np < 0) throw Error(CPSGPU_ERR_ARG, "need nk >= 2, 1 <= nt <= nk, np >= 0");
    if (arg->conv_check < 1 || arg->maxiters < 0) throw Error(CPSGPU_ERR_ARG, "need conv_check >= 1, maxiters >= 0");
    if (arg->Npol < 2) throw Error(CPSGPU_ERR_ARG, "the Chebyshev filter needs Npol >= 2");
    auto neg_of = [](int t) {
      if (t == CPSGPU_RITZ_MATPCDAG_MATPC) return 0;
      if (t == CPSGPU_RITZ_NEG_MATPCDAG_MATPC) return 1;
      throw Error(CPSGPU_ERR_UNSUPPORTED, "RitzMatOper not implemented (MATPCDAG_MATPC, NEG_MATPCDAG_MATPC are)");
    };
    LanczosArgs la{neg_of(arg->RitzMat_lanczos), neg_of(arg->RitzMat_convcheck), nk, nt, np, arg->maxiters,
                   arg->conv_check, arg->Npol, arg->stop_residual, arg->params[0], arg->params[1], arg->eigen_shift};
    const double aa = la.p0 * la.p0, bb = (la.p1 + std::fabs(la.eigen_shift)) * (la.p1 + std::fabs(la.eigen_shift));
    if (!(aa != bb)) throw Error(CPSGPU_ERR_ARG, "the filter interval is empty (params[0]^2 == (params[1] + |eigen_shift|)^2)");
    const int m = nk + np;
    for (int k = 0; k < m; k++)
      if (!V[k]) throw Error(CPSGPU_ERR_ARG, "null Lanczos vector");
    need_gauge(d);
    Lattice &L = *D.lat;
    const size_t nreal = (size_t)24 * L.vh * D.ls;
    std::vector<Field> fv(m);
    for (auto &f : fv) f.create(PREC_SINGLE, L.vh, D.ls, 1);
    Field f64(PREC_DOUBLE, L.vh, D.ls, 1);
    std::vector<double> h(nreal);
    for (size_t q = 0; q < nreal; q++) h[q] = (double)V[0][q];
    const double *hp = h.data();
    upload(L, f64, &hp, 1);
    launch_convert(L.stream, PREC_SINGLE, fv[0].view(), PREC_DOUBLE, f64.view());
    const int it = imp_res_lanczos(D, fv, alpha, la);
    for (int k = 0; k < m; k++) {
      launch_convert(L.stream, PREC_DOUBLE, f64.view(), PREC_SINGLE, fv[k].view());
      double *o = h.data();
      download(L, f64, &o, 1);
      for (size_t q = 0; q < nreal; q++) V[k][q] = (float)h[q];
    }
    if (restarts) *restarts = it;
    if (it < 0) status = CPSGPU_NONFINITE;
    return CPSGPU_OK;
  });
  return rc != CPSGPU_OK ? rc : status;
}

int cpsgpu_inveigcg(cpsgpu_dirac d, double *sol, const double *src, const cpsgpu_cg_arg *arg, int nev, int m,
                    double *const *V, double *M, float *const *U, const double *invH, int def_len,
                    const double *restart, int restart_len, int *iterations, double *true_res) {
  return guarded([&] {
    if (!d || !sol || !src || !arg) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (nev < 0 || def_len < 0 || restart_len < 0) throw Error(CPSGPU_ERR_ARG, "negative count");
    if (nev > 0 && m <= 2 * nev) throw Error(CPSGPU_ERR_ARG, "m should be larger than 2*nev (inv_eig_cg.C:133)");
    if (nev > 0 && (!V || !M)) throw Error(CPSGPU_ERR_ARG, "null V or M");
    if (def_len > 0 && (!U || !invH)) throw Error(CPSGPU_ERR_ARG, "null U or invH");
    if (restart_len > 0 && !restart) throw Error(CPSGPU_ERR_ARG, "null restart");
    need_gauge(d);
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    const size_t nreal = (size_t)24 * L.vh * D.ls;
    Field fsol(PREC_DOUBLE, L.vh, D.ls, 1), fsrc(PREC_DOUBLE, L.vh, D.ls, 1);
    upload(L, fsrc, &src, 1);
    std::vector<Field> fv(nev > 0 ? m : 0), fu(def_len);
    for (auto &f : fv) f.create(PREC_DOUBLE, L.vh, D.ls, 1);
    std::vector<double> h(def_len > 0 ? nreal : 0);
    for (int k = 0; k < def_len; k++) {
      if (!U[k]) throw Error(CPSGPU_ERR_ARG, "null deflation vector");
      for (size_t q = 0; q < nreal; q++) h[q] = (double)U[k][q];
      fu[k].create(PREC_DOUBLE, L.vh, D.ls, 1);
      const double *hp = h.data();
      upload(L, fu[k], &hp, 1);
    }
    std::vector<std::complex<double>> ih((size_t)def_len * def_len);
    for (size_t k = 0; k < ih.size(); k++) ih[k] = {invH[2 * k], invH[2 * k + 1]};
    double tr = 0.0;
    const int it = inveigcg(D, fsol, fsrc, arg->stop_rsd, arg->max_num_iter, nev, m, fv, M, fu, ih, restart,
                            restart_len, &tr);
    download(L, fsol, &sol, 1);
    for (int k = 0; k < (int)fv.size(); k++) {
      double *hv = V[k];
      if (hv) download(L, fv[k], &hv, 1);
    }
    if (iterations) *iterations = it;
    if (true_res) *true_res = tr;
    return CPSGPU_OK;
  });
}

int cpsgpu_minresext(cpsgpu_dirac d, double *psi, const double *phi, double *const *v, double *const *vm,
                     int degree, double *error) {
  return guarded([&] {
    if (!d || !psi || !phi || (degree > 0 && (!v || !vm))) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (degree < 0 || degree > 16) throw Error(CPSGPU_ERR_ARG, "degree must be in [0, 16]");
    for (int k = 0; k < degree; k++)
      if (!v[k] || !vm[k]) throw Error(CPSGPU_ERR_ARG, "null basis vector");
    need_gauge(d);
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    Field fpsi(PREC_DOUBLE, L.vh, D.ls, 1), fphi(PREC_DOUBLE, L.vh, D.ls, 1);
    upload(L, fphi, &phi, 1);
    std::vector<Field> fv(degree), fvm(degree);
    for (int k = 0; k < degree; k++) {
      fv[k].create(PREC_DOUBLE, L.vh, D.ls, 1);
      fvm[k].create(PREC_DOUBLE, L.vh, D.ls, 1);
      const double *h = v[k];
      upload(L, fv[k], &h, 1);
    }
    minresext(D, fpsi, fphi, fv, fvm, error);
    download(L, fpsi, &psi, 1);
    for (int k = 0; k < degree; k++) {
      double *h = v[k], *hm = vm[k];
      download(L, fv[k], &h, 1);
      download(L, fvm[k], &hm, 1);
    }
    return CPSGPU_OK;
  });
}

int cpsgpu_bicgstab(cpsgpu_dirac d, double *psi, const double *chi, double chi_norm, int n, const cpsgpu_cg_arg *arg,
                    int *iterations, double *true_res) {
  return guarded([&] {
    if (!d || !psi || !chi || !arg) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (n < 1 || n > 10) throw Error(CPSGPU_ERR_ARG, "BiCGstab(n): n in [1, 10] (bicgstab.C:67-70)");
    need_gauge(d);
    Dirac &D = *d->D;
    Lattice &L = *D.lat;
    Field fp(PREC_DOUBLE, L.vh, D.ls, 1), fc(PREC_DOUBLE, L.vh, D.ls, 1);
    const double *pp = psi;
    upload(L, fp, &pp, 1);
    upload(L, fc, &chi, 1);
    double tr = 0.0;
    const int k = bicgstab(D, fp, fc, chi_norm, n, arg->stop_rsd, arg->max_num_iter, &tr);
    download(L, fp, &psi, 1);
    if (iterations) *iterations = k;
    if (true_res) *true_res = tr;
    return CPSGPU_OK;
  });
}

int cpsgpu_minvcg(cpsgpu_dirac d, double *const *psi, const double *chi, double chi_norm, const double *shift,
                  int nshift, double *rsdcg, int type, const double *alpha, int max_num_iter, int precision,
                  int refine, int *iterations) {
  return guarded([&] {
    if (!d || !psi || !chi || !shift || !rsdcg || nshift < 1) throw Error(CPSGPU_ERR_ARG, "bad argument");
    if (type < 0 || type > 2) throw Error(CPSGPU_ERR_ARG, "bad multishift type");
    if (type == CPSGPU_MS_SINGLE && !alpha) throw Error(CPSGPU_ERR_ARG, "SINGLE needs alpha");
    check_prec(precision);
    need_gauge(d);
    int k = minvcg(*d->D, psi, chi, chi_norm, shift, nshift, rsdcg, type, alpha, max_num_iter, precision, refine);
    if (iterations) *iterations = k;
    return CPSGPU_OK;
  });
}

int cpsgpu_get_minvcg_stats(cpsgpu_dirac d, cpsgpu_minvcg_stats *stats) {
  return guarded([&] {
    if (!d || !stats) throw Error(CPSGPU_ERR_ARG, "bad argument");
    const MsWork &m = d->D->ms;
    stats->upload_s = m.upload_s;
    stats->recurrence_s = m.recurrence_s;
    stats->refine_s = m.refine_s;
    stats->download_s = m.download_s;
    stats->refine_iterations_max = m.refine_max;
    stats->refine_iterations_sum = m.refine_sum;
    return CPSGPU_OK;
  });
}

// ---- device fields
int cpsgpu_field_create(cpsgpu_dirac d, int precision, int nrhs, cpsgpu_field *f) {
  return guarded([&] {
    if (!d || !f || nrhs < 1) throw Error(CPSGPU_ERR_ARG, "bad argument");
    check_prec(precision);
    auto *o = new cpsgpu_field_s;
    o->d = d;
    try {
      o->f.create(precision, d->D->lat->vh, d->D->ls, nrhs);
    } catch (...) {
      delete o;
      throw;
    }
    *f = o;
    return CPSGPU_OK;
  });
}

int cpsgpu_field_destroy(cpsgpu_field f) {
  return guarded([&] {
    delete f;
    return CPSGPU_OK;
  });
}

int cpsgpu_field_upload(cpsgpu_field f, const double *host) {
  return guarded([&] {
    if (!f || !host) throw Error(CPSGPU_ERR_ARG, "null argument");
    Lattice &L = *f->d->D->lat;
    size_t n = (size_t)24 * f->f.vh * f->f.ls;
    std::vector<const double *> ptrs(f->f.nrhs);
    for (int k = 0; k < f->f.nrhs; k++) ptrs[k] = host + n * k;
    upload(L, f->f, ptrs.data(), f->f.nrhs);
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    return CPSGPU_OK;
  });
}

int cpsgpu_field_download(cpsgpu_field f, double *host) {
  return guarded([&] {
    if (!f || !host) throw Error(CPSGPU_ERR_ARG, "null argument");
    Lattice &L = *f->d->D->lat;
    size_t n = (size_t)24 * f->f.vh * f->f.ls;
    std::vector<double *> ptrs(f->f.nrhs);
    for (int k = 0; k < f->f.nrhs; k++) ptrs[k] = host + n * k;
    download(L, f->f, ptrs.data(), f->f.nrhs);
    return CPSGPU_OK;
  });
}

int cpsgpu_field_gaussian(cpsgpu_field f, unsigned long long seed) {
  return guarded([&] {
    if (!f) throw Error(CPSGPU_ERR_ARG, "null field");
    size_t n = (size_t)24 * f->f.vh * f->f.ls * f->f.nrhs;
    std::vector<double> h(n);
    gen_gaussian(h.data(), (long)n, seed, 0);
    Lattice &L = *f->d->D->lat;
    size_t per = n / f->f.nrhs;
    std::vector<const double *> ptrs(f->f.nrhs);
    for (int k = 0; k < f->f.nrhs; k++) ptrs[k] = h.data() + per * k;
    upload(L, f->f, ptrs.data(), f->f.nrhs);
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    return CPSGPU_OK;
  });
}

int cpsgpu_dslash_field(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in, int cb, int dag) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (out->f.prec != in->f.prec || out->f.nrhs != in->f.nrhs) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    need_gauge(d);
    op_dslash(*d->D, in->f.prec, out->f.view(), in->f.view(), cb ? 1 : 0, dag ? 1 : 0);
    return CPSGPU_OK;
  });
}

int cpsgpu_lattice_set_t_partition(cpsgpu_lattice lat, int nodes_t, int coor_t) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    if (nodes_t < 1 || coor_t < 0 || coor_t >= nodes_t) throw Error(CPSGPU_ERR_ARG, "need 0 <= coor_t < nodes_t");
    Lattice &L = *lat->L;
    L.t_nodes = nodes_t;
    L.t_coor = coor_t;
    return CPSGPU_OK;
  });
}

int cpsgpu_lattice_set_stream(cpsgpu_lattice lat, void *stream) {
  return guarded([&] {
    if (!lat) throw Error(CPSGPU_ERR_ARG, "null lattice");
    Lattice &L = *lat->L;
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));  // nothing of the old stream is left in flight
    L.stream = stream ? static_cast<cudaStream_t>(stream) : L.own_stream;
    L.caller_stream = (stream != nullptr);
    return CPSGPU_OK;
  });
}

int cpsgpu_field_dot_device(cpsgpu_field a, cpsgpu_field b, double *dev_out) {
  return guarded([&] {
    if (!a || !b || !dev_out) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (a->f.prec != PREC_DOUBLE || b->f.prec != PREC_DOUBLE) throw Error(CPSGPU_ERR_ARG, "FP64 fields required");
    if (a->f.sites() != b->f.sites()) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    field_dot_device(*a->d->D->lat, a->f.view(), b->f.view(), dev_out);
    return CPSGPU_OK;
  });
}

int cpsgpu_field_axpby_device(cpsgpu_field out, const double *dev_a, double scale, cpsgpu_field x, cpsgpu_field y) {
  return guarded([&] {
    if (!out || !x || !y || !dev_a) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (out->f.prec != PREC_DOUBLE || x->f.prec != PREC_DOUBLE || y->f.prec != PREC_DOUBLE)
      throw Error(CPSGPU_ERR_ARG, "FP64 fields required");
    if (out->f.sites() != x->f.sites() || out->f.sites() != y->f.sites()) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    Lattice &L = *out->d->D->lat;
    launch_axpby_dev(L.stream, out->f.view(), dev_a, scale, x->f.view(), y->f.view());
    return CPSGPU_OK;
  });
}

int cpsgpu_dd_face_bytes(cpsgpu_dirac d, int precision, int nrhs, size_t *bytes) {
  return guarded([&] {
    if (!d || !bytes || nrhs < 1) throw Error(CPSGPU_ERR_ARG, "bad argument");
    *bytes = dd_face_bytes(*d->D, precision, nrhs);
    return CPSGPU_OK;
  });
}

int cpsgpu_dslash_dd_pack(cpsgpu_dirac d, cpsgpu_field in, int cb, int dag, void *to_prev, void *to_next) {
  return guarded([&] {
    if (!d || !in || !to_prev || !to_next) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (!d->D->lat->have_gauge) throw Error(CPSGPU_ERR_STATE, "no gauge field imported");
    dd_pack(*d->D, in->f.prec, in->f.view(), cb ? 1 : 0, dag ? 1 : 0, to_prev, to_next);
    if (!d->D->lat->caller_stream) CPSGPU_CUDA(cudaStreamSynchronize(d->D->lat->stream));
    return CPSGPU_OK;
  });
}

int cpsgpu_dslash_dd(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in, int cb, int dag, const void *from_next,
                     const void *from_prev) {
  return guarded([&] {
    if (!d || !out || !in || !from_next || !from_prev) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (out->f.prec != in->f.prec || out->f.nrhs != in->f.nrhs) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    if (!d->D->lat->have_gauge) throw Error(CPSGPU_ERR_STATE, "no gauge field imported");
    dd_dslash(*d->D, in->f.prec, out->f.view(), in->f.view(), cb ? 1 : 0, dag ? 1 : 0, from_next, from_prev);
    if (!d->D->lat->caller_stream) CPSGPU_CUDA(cudaStreamSynchronize(d->D->lat->stream));
    return CPSGPU_OK;
  });
}

int cpsgpu_dslash_dd_interior(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in, int cb, int dag) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (out->f.prec != in->f.prec || out->f.nrhs != in->f.nrhs) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    if (!d->D->lat->have_gauge) throw Error(CPSGPU_ERR_STATE, "no gauge field imported");
    // enqueued only: the caller moves the faces meanwhile
    dd_dslash(*d->D, in->f.prec, out->f.view(), in->f.view(), cb ? 1 : 0, dag ? 1 : 0, nullptr, nullptr, SUB_INTERIOR);
    return CPSGPU_OK;
  });
}

int cpsgpu_dslash_dd_boundary(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in, int cb, int dag,
                              const void *from_next, const void *from_prev) {
  return guarded([&] {
    if (!d || !out || !in || !from_next || !from_prev) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (out->f.prec != in->f.prec || out->f.nrhs != in->f.nrhs) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    if (!d->D->lat->have_gauge) throw Error(CPSGPU_ERR_STATE, "no gauge field imported");
    dd_dslash(*d->D, in->f.prec, out->f.view(), in->f.view(), cb ? 1 : 0, dag ? 1 : 0, from_next, from_prev,
              SUB_BOUNDARY);
    if (!d->D->lat->caller_stream) CPSGPU_CUDA(cudaStreamSynchronize(d->D->lat->stream));
    return CPSGPU_OK;
  });
}

int cpsgpu_field_axpby(cpsgpu_field out, double a, cpsgpu_field x, cpsgpu_field y) {
  return guarded([&] {
    if (!out || !x || !y) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (out->f.prec != PREC_DOUBLE || x->f.prec != PREC_DOUBLE || y->f.prec != PREC_DOUBLE)
      throw Error(CPSGPU_ERR_ARG, "FP64 fields required");
    if (out->f.sites() != x->f.sites() || out->f.sites() != y->f.sites()) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    Lattice &L = *out->d->D->lat;
    launch_axpby(L.stream, out->f.view(), a, x->f.view(), y->f.view());
    if (!L.caller_stream) CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    return CPSGPU_OK;
  });
}

int cpsgpu_field_dot(cpsgpu_field a, cpsgpu_field b, double *re, double *im) {
  return guarded([&] {
    if (!a || !b || !re || !im) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (a->f.prec != PREC_DOUBLE || b->f.prec != PREC_DOUBLE) throw Error(CPSGPU_ERR_ARG, "FP64 fields required");
    if (a->f.sites() != b->f.sites()) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    field_dot(*a->d->D->lat, a->f.view(), b->f.view(), re, im);
    return CPSGPU_OK;
  });
}

int cpsgpu_mdagm_field(cpsgpu_dirac d, cpsgpu_field out, cpsgpu_field in) {
  return guarded([&] {
    if (!d || !out || !in) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (out->f.prec != in->f.prec || out->f.nrhs != in->f.nrhs) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    need_gauge(d);
    op_mdagm(*d->D, in->f.prec, out->f.view(), in->f.view(), d->w[in->f.prec], nullptr, 0);
    return CPSGPU_OK;
  });
}

int cpsgpu_invcg_field(cpsgpu_dirac d, cpsgpu_field sol, cpsgpu_field src, const cpsgpu_cg_arg *arg,
                       cpsgpu_cg_result *res) {
  return guarded([&] {
    if (!d || !sol || !src || !arg || !res) throw Error(CPSGPU_ERR_ARG, "null argument");
    if (sol->f.prec != PREC_DOUBLE || src->f.prec != PREC_DOUBLE) throw Error(CPSGPU_ERR_ARG, "FP64 fields required");
    if (sol->f.nrhs != src->f.nrhs) throw Error(CPSGPU_ERR_ARG, "field mismatch");
    check_prec(arg->precision);
    need_gauge(d);
    int nrhs = src->f.nrhs;
    CgSolver &S = solver_for(d, arg->precision, nrhs);
    Lattice &L = *d->D->lat;
    CPSGPU_CUDA(cudaMemcpyAsync(S.b64.data.ptr, src->f.data.ptr, src->f.data.bytes, cudaMemcpyDeviceToDevice, L.stream));
    CPSGPU_CUDA(cudaMemcpyAsync(S.x64.data.ptr, sol->f.data.ptr, sol->f.data.bytes, cudaMemcpyDeviceToDevice, L.stream));
    std::vector<CgResult> r;
    S.run(to_args(arg), r);
    CPSGPU_CUDA(cudaMemcpyAsync(sol->f.data.ptr, S.x64.data.ptr, sol->f.data.bytes, cudaMemcpyDeviceToDevice, L.stream));
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    for (int k = 0; k < nrhs; k++) to_result(r[k], res + k);
    return CPSGPU_OK;
  });
}

int cpsgpu_solve_batch(int n, const cpsgpu_dirac *ops, const cpsgpu_field *sol, const cpsgpu_field *src,
                       const cpsgpu_cg_arg *args, cpsgpu_cg_result *res) {
  return guarded([&] {
    if (n < 1 || !ops || !sol || !src || !args || !res) throw Error(CPSGPU_ERR_ARG, "bad argument");
    std::vector<CgSolver *> solvers;
    std::vector<CgArgs> a;
    for (int k = 0; k < n; k++) {
      cpsgpu_dirac d = ops[k];
      if (!d || !sol[k] || !src[k]) throw Error(CPSGPU_ERR_ARG, "null operator or field");
      if (sol[k]->d != d || src[k]->d != d) throw Error(CPSGPU_ERR_ARG, "fields must belong to their operator");
      if (sol[k]->f.prec != PREC_DOUBLE || src[k]->f.prec != PREC_DOUBLE) throw Error(CPSGPU_ERR_ARG, "FP64 fields required");
      if (sol[k]->f.nrhs != src[k]->f.nrhs) throw Error(CPSGPU_ERR_ARG, "field mismatch");
      if (args[k].max_num_iter < 1) throw Error(CPSGPU_ERR_ARG, "max_num_iter must be >= 1");
      check_prec(args[k].precision);
      need_gauge(d);
      for (int j = 0; j < k; j++)
        if (ops[j] == d && args[j].precision == args[k].precision)
          throw Error(CPSGPU_ERR_ARG, "an operator appears twice in one precision: put its right-hand sides in one field");
      CgSolver &S = solver_for(d, args[k].precision, src[k]->f.nrhs);
      cudaStream_t st = d->D->lat->stream;
      CPSGPU_CUDA(cudaMemcpyAsync(S.b64.data.ptr, src[k]->f.data.ptr, src[k]->f.data.bytes, cudaMemcpyDeviceToDevice, st));
      CPSGPU_CUDA(cudaMemcpyAsync(S.x64.data.ptr, sol[k]->f.data.ptr, sol[k]->f.data.bytes, cudaMemcpyDeviceToDevice, st));
      solvers.push_back(&S);
      a.push_back(to_args(&args[k]));
    }
    std::vector<std::vector<CgResult>> r;
    solve_batch(solvers, a, r);
    int o = 0;
    for (int k = 0; k < n; k++) {
      cudaStream_t st = ops[k]->D->lat->stream;
      CPSGPU_CUDA(cudaMemcpyAsync(sol[k]->f.data.ptr, solvers[k]->x64.data.ptr, sol[k]->f.data.bytes,
                                  cudaMemcpyDeviceToDevice, st));
      CPSGPU_CUDA(cudaStreamSynchronize(st));
      for (const CgResult &x : r[k]) to_result(x, res + o++);
    }
    return CPSGPU_OK;
  });
}

int cpsgpu_dirac_set_pc_type(cpsgpu_dirac d, int pc_type) {
  return guarded([&] {
    if (!d) throw Error(CPSGPU_ERR_ARG, "null operator");
    if (d->D->kind != KIND_MOBIUS) throw Error(CPSGPU_ERR_ARG, "preconditioning type: Mobius operators only");
    CPSGPU_CUDA(cudaStreamSynchronize(d->D->lat->stream));
    try {
      d->D->set_pc_type(pc_type);
    } catch (const Error &e) {
      throw Error(CPSGPU_ERR_ARG, e.what());
    }
    // captured graphs hold the launches of the old form
    drop_captured(d);
    return CPSGPU_OK;
  });
}

int cpsgpu_dirac_get_pc_type(cpsgpu_dirac d, int *pc_type) {
  return guarded([&] {
    if (!d || !pc_type) throw Error(CPSGPU_ERR_ARG, "bad argument");
    *pc_type = (d->D->kind == KIND_MOBIUS) ? d->D->pc_type : PC_SYM2;
    return CPSGPU_OK;
  });
}

int cpsgpu_set_mix_impl(cpsgpu_dirac d, int impl) {
  return guarded([&] {
    if (!d) throw Error(CPSGPU_ERR_ARG, "null operator");
    if (d->D->kind != KIND_MOBIUS) throw Error(CPSGPU_ERR_ARG, "Ls x Ls mixing: Mobius operators only");
    if (impl < 0 || impl > 3)
      throw Error(CPSGPU_ERR_ARG, "mixing kernel: 0 default, 1 tensor cores, 2 shared memory, 3 register-tiled");
    CPSGPU_CUDA(cudaStreamSynchronize(d->D->lat->stream));
    d->D->mix_tc = (impl == 1);
    d->D->mix_reg = (impl != 2);
    d->D->mix_bulk = (impl == 0 || impl == 1);
    // allocated here, never inside a graph capture
    if (d->D->mix_tc) d->D->mixTcFrag.ensure(2 * 2 * 32 * 4 * sizeof(unsigned));
    // captured graphs hold the other kernels
    drop_captured(d);
    return CPSGPU_OK;
  });
}

int cpsgpu_autotune(cpsgpu_dirac d, int prec, int nrhs, int *tuned) {
  return guarded([&] {
    if (!d || nrhs < 1) throw Error(CPSGPU_ERR_ARG, "bad argument");
    check_prec(prec);
    need_gauge(d);
    CPSGPU_CUDA(cudaStreamSynchronize(d->D->lat->stream));
    drop_captured(d);  // recaptured with the tuned shapes and link form
    int n = autotune(*d->D, prec, nrhs);
    if (tuned) *tuned = n;
    return CPSGPU_OK;
  });
}

int cpsgpu_time_m5inv(cpsgpu_dirac d, int prec, int reps, double *ms, double *bytes) {
  return guarded([&] {
    if (!d || reps < 1 || !ms) throw Error(CPSGPU_ERR_ARG, "bad argument");
    check_prec(prec);
    need_gauge(d);
    *ms = time_m5inv(*d->D, prec, reps, bytes);
    if (mix_bulk_error()) throw Error(CPSGPU_ERR_STATE, "a bounded wait of the bulk-staged mixing kernel ran out");
    return CPSGPU_OK;
  });
}

int cpsgpu_get_rhs_tile(cpsgpu_dirac d, int prec, int nrhs, int *tile) {
  return guarded([&] {
    if (!d || nrhs < 1 || !tile) throw Error(CPSGPU_ERR_ARG, "bad argument");
    check_prec(prec);
    *tile = std::max(1, std::min(d->D->rhs_tile(prec, nrhs), nrhs));
    return CPSGPU_OK;
  });
}

int cpsgpu_set_rhs_tile(cpsgpu_dirac d, int prec, int tile) {
  return guarded([&] {
    if (!d || tile < 0) throw Error(CPSGPU_ERR_ARG, "bad argument");
    check_prec(prec);
    CPSGPU_CUDA(cudaStreamSynchronize(d->D->lat->stream));
    d->D->rtile[prec] = tile;
    // captured graphs hold the launches of the old tile
    drop_captured(d);
    return CPSGPU_OK;
  });
}

static_assert(CPSGPU_ORDER_SLICES == ORDER_SLICES && CPSGPU_ORDER_SITES == ORDER_SITES,
              "public and internal hop orders");

int cpsgpu_get_hop_shape(cpsgpu_dirac d, int prec, int *sites, int *slices, int *slices_per_thread, int *order) {
  return guarded([&] {
    if (!d || !sites || !slices || !slices_per_thread || !order) throw Error(CPSGPU_ERR_ARG, "bad argument");
    check_prec(prec);
    const Dirac &D = *d->D;
    const TuneKey key{prec, D.lat->recon(prec), EP_STORE, D.kind, D.ls};
    const dim3 b = hop_block(key, false);
    *sites = (int)b.x;
    *slices = (int)b.y;
    *slices_per_thread = (b.z == 2 && D.kind == KIND_DWF && prec != PREC_DOUBLE && D.ls % (4 * (int)b.y) == 0) ? 2 : 1;
    *order = hop_order(key);
    return CPSGPU_OK;
  });
}

int cpsgpu_set_hop_shape(cpsgpu_dirac d, int prec, int sites, int slices, int slices_per_thread, int order) {
  return guarded([&] {
    if (!d || sites < 1 || slices < 1 || sites * slices > 256 || sites * slices % 32 != 0 ||
        (slices_per_thread != 1 && slices_per_thread != 2))
      throw Error(CPSGPU_ERR_ARG, "hop shape: sites x slices a multiple of 32 up to 256, 1 or 2 slices per thread");
    if (order < 0 || order >= ORDER_COUNT) throw Error(CPSGPU_ERR_ARG, "hop order: CPSGPU_ORDER_SLICES or CPSGPU_ORDER_SITES");
    check_prec(prec);
    const Dirac &D = *d->D;
    if (slices > std::max(D.ls, 1)) throw Error(CPSGPU_ERR_ARG, "hop shape: more slices per block than Ls");
    if (slices_per_thread == 2 && (D.kind != KIND_DWF || prec == PREC_DOUBLE || D.ls % (4 * slices) != 0))
      throw Error(CPSGPU_ERR_ARG, "slice pairs: DWF, FP32 or FP16 fields, Ls a multiple of 4 x slices");
    const dim3 b((unsigned)sites, (unsigned)slices, (unsigned)slices_per_thread);
    const int eps[] = {EP_STORE, EP_AXPY, EP_CG, EP_RES};
    CPSGPU_CUDA(cudaStreamSynchronize(D.lat->stream));
    for (int ep : eps) tune_set(TuneKey{prec, D.lat->recon(prec), ep, D.kind, D.ls}, b, order);
    // captured graphs hold the launches of the old shape
    drop_captured(d);
    return CPSGPU_OK;
  });
}

int cpsgpu_time_dslash(cpsgpu_dirac d, int prec, int cb, int dag, int reps, double *ms, double *bytes) {
  return guarded([&] {
    if (!d || reps < 1 || !ms) throw Error(CPSGPU_ERR_ARG, "bad argument");
    check_prec(prec);
    need_gauge(d);
    *ms = time_dslash(*d->D, prec, cb ? 1 : 0, dag ? 1 : 0, reps, bytes);
    return CPSGPU_OK;
  });
}

int cpsgpu_time_mdagm(cpsgpu_dirac d, int prec, int reps, double *ms, double *bytes) {
  return guarded([&] {
    if (!d || reps < 1 || !ms) throw Error(CPSGPU_ERR_ARG, "bad argument");
    check_prec(prec);
    need_gauge(d);
    *ms = time_mdagm(*d->D, prec, reps, bytes);
    return CPSGPU_OK;
  });
}

int cpsgpu_host_alloc(size_t bytes, void **ptr) {
  return guarded([&] {
    if (!ptr) throw Error(CPSGPU_ERR_ARG, "null pointer");
    CPSGPU_CUDA(cudaMallocHost(ptr, bytes));
    return CPSGPU_OK;
  });
}

int cpsgpu_host_free(void *ptr) {
  return guarded([&] {
    if (ptr) CPSGPU_CUDA(cudaFreeHost(ptr));
    return CPSGPU_OK;
  });
}

int cpsgpu_gen_gauge(const int node_sites[4], unsigned long long seed, double width, double *u) {
  return guarded([&] {
    if (!node_sites || !u) throw Error(CPSGPU_ERR_ARG, "null argument");
    for (int k = 0; k < 4; k++)
      if (node_sites[k] <= 0 || (node_sites[k] & 1)) throw Error(CPSGPU_ERR_ARG, "extents must be positive and even");
    gen_gauge(node_sites, seed, width, u);
    return CPSGPU_OK;
  });
}

int cpsgpu_gen_gaussian(double *out, long n, unsigned long long seed, unsigned int stream) {
  return guarded([&] {
    if (!out || n < 0) throw Error(CPSGPU_ERR_ARG, "bad argument");
    gen_gaussian(out, n, seed, stream);
    return CPSGPU_OK;
  });
}

}  // extern "C"
