// Host-driven Krylov routines with every vector on the device:
//   BiCGstab(n) on MatPc: DiracOpWilsonTypes::BiCGstab (bicgstab.C:35-229);
//   the chronological initial guess DiracOp::MinResExt (minresext.C:30-150).
// Their complex scalars (rho, alpha, omega, tau, gamma; the small Gram
// matrix) are the reference's short host computations, step for step; each
// global dot product <a, b> = sum conj(a) b (compDotProduct,
// vector_util.C:889-903) is a device reduction read back by the host.
#include <complex>
#include <vector>

#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

namespace {

constexpr int TPB = 256;

// per-block partials of <a, b> (re, im), one thread per 5D site
__global__ void cdot_kernel(SpinorView a, SpinorView b, double *partials, size_t n) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (idx < n) {
    const long sl = (long)(idx / a.vh), i = (long)(idx % a.vh);
    double x[24], y[24];
    SpinorIO<PREC_DOUBLE>::load(a, sl, i, x);
    SpinorIO<PREC_DOUBLE>::load(b, sl, i, y);
#pragma unroll
    for (int k = 0; k < 24; k += 2) {
      v[0] += x[k] * y[k] + x[k + 1] * y[k + 1];
      v[1] += x[k] * y[k + 1] - x[k + 1] * y[k];
    }
  }
  block_partial<2>(v, partials);
}

// a = f c + d, f complex (cTimesV1PlusV2, vector_util.C:912-922)
__global__ void caxpy_kernel(SpinorView a, double re, double im, SpinorView c, SpinorView d, size_t n) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const long sl = (long)(idx / a.vh), i = (long)(idx % a.vh);
  double x[24], y[24];
  SpinorIO<PREC_DOUBLE>::load(c, sl, i, x);
  SpinorIO<PREC_DOUBLE>::load(d, sl, i, y);
#pragma unroll
  for (int k = 0; k < 24; k += 2) {
    const double cr = x[k], ci = x[k + 1];
    y[k] += re * cr - im * ci;
    y[k + 1] += re * ci + im * cr;
  }
  SpinorIO<PREC_DOUBLE>::store(a, sl, i, y);
}

using cd = std::complex<double>;

struct Ctx {
  Dirac &D;
  Lattice &L;
  OpWork w;
  SolverScalars *st;
  double *partials;
  size_t sites;
  unsigned blocks() const { return (unsigned)((sites + TPB - 1) / TPB); }

  cd dot(const Field &a, const Field &b) {
    cdot_kernel<<<blocks(), TPB, 0, L.stream>>>(a.view(), b.view(), partials, sites);
    CPSGPU_CUDA(cudaGetLastError());
    launch_counter()++;
    launch_finalize(L.stream, 2, partials, st, RED_STORE, blocks(), 1, GATE_NONE);
    double s[2];
    CPSGPU_CUDA(cudaMemcpyAsync(s, st->sum, sizeof(s), cudaMemcpyDeviceToHost, L.stream));
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    return {s[0], s[1]};
  }
  double norm2(const Field &a) {
    launch_norm(L.stream, PREC_DOUBLE, a.view(), st, partials, RED_STORE, GATE_NONE);
    double s = 0.0;
    CPSGPU_CUDA(cudaMemcpyAsync(&s, st->sum, sizeof(s), cudaMemcpyDeviceToHost, L.stream));
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    return s;
  }
  // a = f c + d
  void caxpy(Field &a, cd f, const Field &c, const Field &d) {
    caxpy_kernel<<<blocks(), TPB, 0, L.stream>>>(a.view(), f.real(), f.imag(), c.view(), d.view(), sites);
    CPSGPU_CUDA(cudaGetLastError());
    launch_counter()++;
  }
  void matpc(Field &out, const Field &in) { op_matpc(D, PREC_DOUBLE, out.view(), in.view(), 0, w, nullptr, 0, 0); }
  // out = MatPcDagMatPc in; returns |MatPc in|^2
  double mdagm(Field &out, const Field &in) {
    CPSGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(SolverScalars), L.stream));
    op_mdagm(D, PREC_DOUBLE, out.view(), in.view(), w, st, RED_STORE);
    double s = 0.0;
    CPSGPU_CUDA(cudaMemcpyAsync(&s, st->sum, sizeof(s), cudaMemcpyDeviceToHost, L.stream));
    CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
    return s;
  }
};

}  // namespace

int bicgstab(Dirac &D, Field &psi, const Field &chi, double chi_norm, int nn, double stop_rsd, int max_num_iter,
             double *true_res) {
  constexpr int NMAX = 10;
  if (nn <= 0 || nn > NMAX) throw Error(-1, "BiCGstab: n must be in [1, 10]");
  Lattice &L = *D.lat;
  Ctx c{D, L, OpWork(), L.scratch_st.as<SolverScalars>(), nullptr, (size_t)L.vh * D.ls};
  L.partials.ensure((size_t)c.blocks() * 2 * sizeof(double));
  c.partials = L.partials.as<double>();
  CPSGPU_CUDA(cudaMemsetAsync(c.st, 0, sizeof(SolverScalars), L.stream));
  std::vector<Field> r(nn + 1), u(nn + 1);
  for (int i = 0; i <= nn; i++) {
    r[i].create(PREC_DOUBLE, L.vh, D.ls, 1);
    u[i].create(PREC_DOUBLE, L.vh, D.ls, 1);
  }
  Field r0(PREC_DOUBLE, L.vh, D.ls, 1);
  cd rho0 = 1.0, rho1, alpha = 0.0, omega = 1.0, beta;
  double sigma[NMAX + 1];
  cd gamma[NMAX + 1], gamma_p[NMAX + 1], gamma_pp[NMAX + 1], tau[NMAX + 1][NMAX + 1];
  int converged = 0, k;

  if (chi_norm == 0.0) chi_norm = c.norm2(chi);
  if (chi_norm == 0.0) {  // the solution of a zero source is zero
    launch_zero(L.stream, psi);
    return 0;
  }
  const double rsd_sq = chi_norm * stop_rsd * stop_rsd;
  // r[0] = chi - MatPc psi;  r0 = r[0];  u[0] = 0
  c.matpc(r[0], psi);
  c.caxpy(r[0], -1.0, r[0], chi);
  sigma[0] = c.norm2(r[0]);
  CPSGPU_CUDA(cudaMemcpyAsync(r0.data.ptr, r[0].data.ptr, r0.data.bytes, cudaMemcpyDeviceToDevice, L.stream));
  launch_zero(L.stream, u[0]);

  for (k = 1; k <= max_num_iter && !converged; k += nn) {
    rho0 *= -omega;
    for (int j = 0; j < nn; j++) {  // BiCG part
      rho1 = c.dot(r0, r[j]);
      beta = alpha * rho1 / rho0;
      rho0 = rho1;
      for (int i = 0; i <= j; i++) c.caxpy(u[i], -beta, u[i], r[i]);
      c.matpc(u[j + 1], u[j]);
      alpha = rho0 / c.dot(r0, u[j + 1]);
      for (int i = 0; i <= j; i++) c.caxpy(r[i], -alpha, u[i + 1], r[i]);
      c.matpc(r[j + 1], r[j]);
      c.caxpy(psi, alpha, u[0], psi);
    }
    for (int j = 1; j <= nn; j++) {  // MR part
      for (int i = 1; i < j; i++) {
        tau[i][j] = c.dot(r[i], r[j]) / sigma[i];
        c.caxpy(r[j], -tau[i][j], r[i], r[j]);
      }
      sigma[j] = c.norm2(r[j]);
      gamma_p[j] = c.dot(r[j], r[0]) / sigma[j];
    }
    gamma[nn] = gamma_p[nn];
    omega = gamma[nn];
    for (int j = nn - 1; j > 0; j--) {
      gamma[j] = gamma_p[j];
      for (int i = j + 1; i <= nn; i++) gamma[j] -= tau[j][i] * gamma[i];
    }
    for (int j = 1; j < nn; j++) {
      gamma_pp[j] = gamma[j + 1];
      for (int i = j + 1; i < nn; i++) gamma_pp[j] += tau[j][i] * gamma[i + 1];
    }
    c.caxpy(u[0], -gamma[nn], u[nn], u[0]);
    c.caxpy(psi, gamma[1], r[0], psi);
    c.caxpy(r[0], -gamma_p[nn], r[nn], r[0]);
    for (int j = 1; j < nn; j++) {
      c.caxpy(u[0], -gamma[j], u[j], u[0]);
      c.caxpy(psi, gamma_pp[j], r[j], psi);
      c.caxpy(r[0], -gamma_p[j], r[j], r[0]);
    }
    sigma[0] = c.norm2(r[0]);
    if (sigma[0] < rsd_sq) converged = 1;
  }
  if (converged && true_res) *true_res = std::sqrt(sigma[0]);
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
  return k;
}

void minresext(Dirac &D, Field &psi, const Field &phi, std::vector<Field> &v, std::vector<Field> &vm,
               double *error) {
  const int degree = (int)v.size();
  Lattice &L = *D.lat;
  if (degree == 0) {  // no guess requested: psi = 0
    launch_zero(L.stream, psi);
    if (error) *error = 1.0;
    return;
  }
  if (degree > 16) throw Error(-1, "MinResExt: at most 16 previous solutions");
  Ctx c{D, L, OpWork(), L.scratch_st.as<SolverScalars>(), nullptr, (size_t)L.vh * D.ls};
  L.partials.ensure((size_t)c.blocks() * 2 * sizeof(double));
  c.partials = L.partials.as<double>();
  std::vector<std::vector<cd>> G(degree, std::vector<cd>(degree));
  std::vector<cd> a(degree), b(degree);
  cd xp;
  // orthonormalise the basis
  for (int i = 0; i < degree; i++) {
    launch_scale(L.stream, 1.0 / std::sqrt(c.norm2(v[i])), v[i].view());
    for (int j = i + 1; j < degree; j++) {
      xp = c.dot(v[i], v[j]);
      c.caxpy(v[j], -xp, v[i], v[j]);
    }
  }
  for (int i = 0; i < degree; i++) {
    b[i] = c.dot(v[i], phi);
    G[i][i] = cd(c.mdagm(vm[i], v[i]), 0.0);
  }
  for (int j = 0; j < degree; j++)
    for (int k = j + 1; k < degree; k++) {
      G[j][k] = c.dot(v[j], vm[k]);
      G[k][j] = std::conj(G[j][k]);
    }
  // Gauss-Jordan elimination with the reference's (diagonal) pivoting
  for (int i = 0; i < degree; i++) {
    int k = i;
    for (int j = i + 1; j < degree; j++)
      if (std::abs(G[j][j]) > std::abs(G[k][k])) k = j;
    if (k != i) {
      std::swap(b[k], b[i]);
      std::swap(G[k], G[i]);
    }
    for (int j = i + 1; j < degree; j++) {
      xp = G[j][i] / G[i][i];
      b[j] -= xp * b[i];
      for (int kk = 0; kk < degree; kk++) G[j][kk] -= xp * G[i][kk];
    }
  }
  Field r(PREC_DOUBLE, L.vh, D.ls, 1);
  launch_zero(L.stream, psi);
  CPSGPU_CUDA(cudaMemcpyAsync(r.data.ptr, phi.data.ptr, r.data.bytes, cudaMemcpyDeviceToDevice, L.stream));
  for (int i = degree - 1; i >= 0; i--) {
    a[i] = 0.0;
    for (int j = i + 1; j < degree; j++) a[i] += G[i][j] * a[j];
    a[i] = (b[i] - a[i]) / G[i][i];
    c.caxpy(psi, a[i], v[i], psi);
    c.caxpy(r, -a[i], vm[i], r);
  }
  if (error) *error = std::sqrt(c.norm2(r) / c.norm2(phi));
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
}

}  // namespace cpsgpu
