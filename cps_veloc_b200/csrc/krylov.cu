// Host-driven Krylov routines with every vector on the device:
//   BiCGstab(n) on MatPc: DiracOpWilsonTypes::BiCGstab (bicgstab.C:35-229);
//   the chronological initial guess DiracOp::MinResExt (minresext.C:30-150).
// Their complex scalars (rho, alpha, omega, tau, gamma; the small Gram
// matrix) are the reference's short host computations, step for step; each
// global dot product <a, b> = sum conj(a) b (compDotProduct,
// vector_util.C:889-903) is a device reduction read back by the host.
#include <algorithm>
#include <cmath>
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

// out[j][k] = sum_i V[i][k] QZ[i + m j] for j < rank: the Ritz vectors of
// an eigCG restart as combinations of the m Lanczos vectors
// (eigcg_vec_mult, inv_eig_cg.C:76-126).  A thread per real, VM_R outputs
// in registers at a time; V reads are coalesced, QZ is read uniformly.
constexpr int VM_R = 16;
__global__ void __launch_bounds__(256) vec_mult_kernel(const double *const *V, int m, const double *QZ, int rank,
                                                       double *const *out, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    for (int j0 = 0; j0 < rank; j0 += VM_R) {
      double acc[VM_R];
#pragma unroll
      for (int q = 0; q < VM_R; q++) acc[q] = 0.0;
      for (int i = 0; i < m; i++) {
        const double v = V[i][k];
#pragma unroll
        for (int q = 0; q < VM_R; q++)
          if (j0 + q < rank) acc[q] = fma(v, QZ[i + m * (j0 + q)], acc[q]);
      }
#pragma unroll
      for (int q = 0; q < VM_R; q++)
        if (j0 + q < rank) out[j0 + q][k] = acc[q];
    }
}

// <a, b> of two FP32 fields, accumulated in FP64 (per-block partials)
__global__ void cdot_f_kernel(SpinorView a, SpinorView b, double *partials, size_t n) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (idx < n) {
    const long sl = (long)(idx / a.vh), i = (long)(idx % a.vh);
    float x[24], y[24];
    SpinorIO<PREC_SINGLE>::load(a, sl, i, x);
    SpinorIO<PREC_SINGLE>::load(b, sl, i, y);
#pragma unroll
    for (int k = 0; k < 24; k += 2) {
      v[0] += (double)x[k] * y[k] + (double)x[k + 1] * y[k + 1];
      v[1] += (double)x[k] * y[k + 1] - (double)x[k + 1] * y[k];
    }
  }
  block_partial<2>(v, partials);
}

// y += f x in FP32, f complex (ZAXPYfloat of lanczos_GramSchm_test)
__global__ void caxpy_f_kernel(SpinorView y, float re, float im, SpinorView x, size_t n) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const long sl = (long)(idx / y.vh), i = (long)(idx % y.vh);
  float a[24], b[24];
  SpinorIO<PREC_SINGLE>::load(x, sl, i, a);
  SpinorIO<PREC_SINGLE>::load(y, sl, i, b);
#pragma unroll
  for (int k = 0; k < 24; k += 2) {
    b[k] += re * a[k] - im * a[k + 1];
    b[k + 1] += re * a[k + 1] + im * a[k];
  }
  SpinorIO<PREC_SINGLE>::store(y, sl, i, b);
}

// out = a out + b x + c y (the Chebyshev recurrence), a thread per real
__global__ void cheb_kernel(double *out, double a, double b, const double *x, double c, const double *y, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    double o = a * out[k];
    o += b * x[k];
    if (c != 0.0) o += c * y[k];
    out[k] = o;
  }
}

// out[j][k] = sum_i V[i][k] QZ[i + m j] for j < rank with FP32 vectors and
// FP64 sums (the Lanczos restart's V Q); out must not alias V
__global__ void __launch_bounds__(256) vec_mult_f_kernel(const float *const *V, int m, const double *QZ, int rank,
                                                         float *const *out, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    for (int j0 = 0; j0 < rank; j0 += VM_R) {
      double acc[VM_R];
#pragma unroll
      for (int q = 0; q < VM_R; q++) acc[q] = 0.0;
      for (int i = 0; i < m; i++) {
        const double v = V[i][k];
#pragma unroll
        for (int q = 0; q < VM_R; q++)
          if (j0 + q < rank) acc[q] = fma(v, QZ[i + m * (j0 + q)], acc[q]);
      }
#pragma unroll
      for (int q = 0; q < VM_R; q++)
        if (j0 + q < rank) out[j0 + q][k] = (float)acc[q];
    }
}

// Real symmetric eigenproblem by cyclic Jacobi rotations (Golub and Van
// Loan, Matrix Computations, section 8.5).  ap: packed lower triangle
// (i(i+1)/2 + j); evec[k n + i] = component k of eigenvector i.  The
// reference's eigen_solver (eigen_solver.C:40) has the same layout, but its
// QL step leaves the eigenvector update commented out, so the vectors it
// returns are the Householder transform, not eigenvectors; these are.
void sym_eigen(const std::vector<double> &ap, int n, std::vector<double> &evec, std::vector<double> &eval) {
  std::vector<double> a((size_t)n * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j <= i; j++) a[(size_t)i * n + j] = a[(size_t)j * n + i] = ap[(size_t)i * (i + 1) / 2 + j];
  evec.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) evec[(size_t)i * n + i] = 1.0;
  double fro = 0.0;
  for (double x : a) fro += x * x;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) off += 2.0 * a[(size_t)p * n + q] * a[(size_t)p * n + q];
    if (off <= 1e-30 * fro) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = a[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double theta = (a[(size_t)q * n + q] - a[(size_t)p * n + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        auto rot = [&](double &x, double &y) {
          const double u = x, w = y;
          x = cs * u - sn * w;
          y = sn * u + cs * w;
        };
        for (int k = 0; k < n; k++) rot(a[(size_t)k * n + p], a[(size_t)k * n + q]);
        for (int k = 0; k < n; k++) rot(a[(size_t)p * n + k], a[(size_t)q * n + k]);
        for (int k = 0; k < n; k++) rot(evec[(size_t)k * n + p], evec[(size_t)k * n + q]);
      }
  }
  eval.resize(n);
  for (int i = 0; i < n; i++) eval[i] = a[(size_t)i * n + i];
}

// indices of the nev smallest eigenvalues, as min_eig_index (inv_eig_cg.C:37-51) picks them
void min_eig_index(std::vector<int> &index, int nev, const std::vector<double> &eig, int n) {
  index.resize(nev);
  for (int i = 0; i < nev; i++) index[i] = i;
  for (int i = nev; i < n; i++) {
    int mx = 0;
    for (int j = 1; j < nev; j++)
      if (eig[index[j]] > eig[index[mx]]) mx = j;
    if (eig[i] < eig[index[mx]]) index[mx] = i;
  }
}

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


// DiracOp::InvEigCg (inv_eig_cg.C:129-635): CG on A = MatPcDagMatPc, FP64,
// with the eigCG bookkeeping (nev > 0) and low-mode deflation (U, invH).
// The CG steps and their order are the reference's; the small matrices (T,
// Q, H and their eigenproblems) live on the host, every vector on the
// device.  V holds the m Lanczos vectors (on return: the last restart's Ritz
// vectors first, M their Ritz values).  Returns the reference's iter.
int inveigcg(Dirac &D, Field &sol, const Field &src, double stop_rsd, int max_iter, int nev, int m,
             std::vector<Field> &V, double *M, std::vector<Field> &U, const std::vector<cd> &invH,
             const double *restart, int restart_len, double *true_res) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  Ctx c{D, L, OpWork(), L.scratch_st.as<SolverScalars>(), nullptr, (size_t)L.vh * D.ls};
  L.partials.ensure((size_t)c.blocks() * 2 * sizeof(double));
  c.partials = L.partials.as<double>();
  const int def_len = (int)U.size();
  const size_t nreal = (size_t)24 * L.vh * D.ls;
  Field r(PREC_DOUBLE, L.vh, D.ls, 1), dir(PREC_DOUBLE, L.vh, D.ls, 1), mmp(PREC_DOUBLE, L.vh, D.ls, 1);
  Field mmp_prev;
  if (nev > 0) mmp_prev.create(PREC_DOUBLE, L.vh, D.ls, 1);
  const double src_norm_sq = c.norm2(src);
  const double stp = src_norm_sq * stop_rsd * stop_rsd;
  auto copy = [&](Field &dst, const Field &from) {
    CPSGPU_CUDA(cudaMemcpyAsync(dst.data.ptr, from.data.ptr, dst.data.bytes, cudaMemcpyDeviceToDevice, s));
  };
  // out = sum_ii (invH <U, rhs>)_ii U_ii
  auto deflate = [&](const Field &rhs, Field &out) {
    std::vector<cd> ub(def_len), w(def_len, 0.0);
    for (int ii = 0; ii < def_len; ii++) ub[ii] = c.dot(U[ii], rhs);
    for (int ii = 0; ii < def_len; ii++)
      for (int jj = 0; jj < def_len; jj++) w[ii] += invH[(size_t)ii * def_len + jj] * ub[jj];
    launch_zero(s, out);
    for (int ii = 0; ii < def_len; ii++) c.caxpy(out, w[ii], U[ii], out);
  };
  launch_zero(s, sol);
  if (def_len > 0) deflate(src, sol);
  c.mdagm(mmp, sol);
  launch_axpby(s, r.view(), -1.0, mmp.view(), src.view());  // r = src - A sol
  copy(dir, r);
  double res_cur = c.norm2(r), res_prv = res_cur;

  const int nev2 = 2 * nev;
  std::vector<double> T, Tt, Y, Q, QZ, H, EIG, Mv;
  std::vector<int> INDEX;
  std::vector<Field> W;
  DeviceBuffer vptr, wptr, qzbuf;
  if (nev > 0) {
    T.assign((size_t)m * (m + 1) / 2, 0.0);
    Q.assign((size_t)m * nev2, 0.0);
    QZ.assign((size_t)m * nev2, 0.0);
    H.assign((size_t)nev2 * (nev2 + 1) / 2, 0.0);
    W.resize(nev2);
    for (auto &f : W) f.create(PREC_DOUBLE, L.vh, D.ls, 1);
    std::vector<double *> vp(m), wp(nev2);
    for (int i = 0; i < m; i++) vp[i] = V[i].data.as<double>();
    for (int i = 0; i < nev2; i++) wp[i] = W[i].data.as<double>();
    vptr.alloc(sizeof(double *) * m);
    wptr.alloc(sizeof(double *) * nev2);
    qzbuf.alloc(sizeof(double) * m * nev2);
    CPSGPU_CUDA(cudaMemcpyAsync(vptr.ptr, vp.data(), sizeof(double *) * m, cudaMemcpyHostToDevice, s));
    CPSGPU_CUDA(cudaMemcpyAsync(wptr.ptr, wp.data(), sizeof(double *) * nev2, cudaMemcpyHostToDevice, s));
    CPSGPU_CUDA(cudaStreamSynchronize(s));
  }
  auto tidx = [](int i, int j) { return (size_t)i * (i + 1) / 2 + j; };  // packed lower triangle, j <= i
  int i_eig = 0, restarted = 0, iter;
  double alpha = 1.0, beta = 0.0, alpha_old = 0.0, beta_old = 0.0;
  for (iter = 0; iter < max_iter; iter++) {
    if (nev > 0 && i_eig == m) copy(mmp_prev, mmp);
    res_prv = res_cur;
    const double pAp = c.mdagm(mmp, dir);
    if (pAp == 0) break;
    if (nev > 0) {
      if (i_eig != 0) T[tidx(i_eig - 1, i_eig - 1)] = 1.0 / alpha + beta_old / alpha_old;
      if (i_eig == m) {
        // restart: the nev lowest eigenvectors of T(m) and of T(m-1) (padded)
        Tt.assign(T.begin(), T.begin() + (size_t)m * (m - 1) / 2);
        sym_eigen(Tt, m - 1, Y, EIG);
        min_eig_index(INDEX, nev, EIG, m - 1);
        for (int i = nev; i < nev2; i++) {
          for (int j = 0; j < m - 1; j++) Q[(size_t)j * nev2 + i] = Y[(size_t)j * (m - 1) + INDEX[i - nev]];
          Q[(size_t)(m - 1) * nev2 + i] = 0.0;
        }
        sym_eigen(T, m, Y, EIG);
        min_eig_index(INDEX, nev, EIG, m);
        for (int i = 0; i < nev; i++)
          for (int j = 0; j < m; j++) Q[(size_t)j * nev2 + i] = Y[(size_t)j * m + INDEX[i]];
        // Gram-Schmidt of the second set against the first, dropping dependent vectors
        int rank = nev;
        for (int i = nev; i < nev2; i++) {
          for (int j = 0; j < rank; j++) {
            double xy = 0.0;
            for (int k = 0; k < m; k++) xy += Q[(size_t)k * nev2 + i] * Q[(size_t)k * nev2 + j];
            for (int k = 0; k < m; k++) Q[(size_t)k * nev2 + i] -= xy * Q[(size_t)k * nev2 + j];
          }
          double xx = 0.0;
          for (int k = 0; k < m; k++) xx += Q[(size_t)k * nev2 + i] * Q[(size_t)k * nev2 + i];
          if (xx > 1e-16) {
            xx = 1.0 / std::sqrt(xx);
            for (int k = 0; k < m; k++) Q[(size_t)k * nev2 + rank] = xx * Q[(size_t)k * nev2 + i];
            rank++;
          }
        }
        // H = Q^T T Q, its eigenpairs: the Ritz values M and QZ = Q Z
        for (int i = 0; i < rank; i++)
          for (int j = 0; j <= i; j++) {
            double h = 0.0;
            for (int l = 0; l < m; l++)
              for (int k = 0; k < m; k++)
                h += Q[(size_t)l * nev2 + i] * (k <= l ? T[tidx(l, k)] : T[tidx(k, l)]) * Q[(size_t)k * nev2 + j];
            H[tidx(i, j)] = h;
          }
        std::vector<double> Hp(H.begin(), H.begin() + (size_t)rank * (rank + 1) / 2);
        sym_eigen(Hp, rank, Y, Mv);
        for (int i = 0; i < nev2; i++) M[i] = i < rank ? Mv[i] : 0.0;
        for (int j = 0; j < rank; j++)
          for (int i = 0; i < m; i++) {
            double z = 0.0;
            for (int k = 0; k < rank; k++) z += Q[(size_t)i * nev2 + k] * Y[(size_t)j + (size_t)k * rank];
            QZ[(size_t)i + (size_t)m * j] = z;
          }
        CPSGPU_CUDA(cudaMemcpyAsync(qzbuf.ptr, QZ.data(), sizeof(double) * m * rank, cudaMemcpyHostToDevice, s));
        const unsigned g = (unsigned)std::min<size_t>((nreal + 255) / 256, 148 * 16);
        vec_mult_kernel<<<g, 256, 0, s>>>(vptr.as<double *>(), m, qzbuf.as<double>(), rank, wptr.as<double *>(), nreal);
        CPSGPU_CUDA(cudaGetLastError());
        launch_counter()++;
        for (int j = 0; j < rank; j++) copy(V[j], W[j]);
        // T <- diag(M) plus the coupling row of A r to the Ritz vectors
        std::fill(T.begin(), T.end(), 0.0);
        for (int i = 0; i < rank; i++) T[tidx(i, i)] = M[i];
        i_eig = rank;
        launch_axpby(s, mmp_prev.view(), -beta, mmp_prev.view(), mmp.view());
        for (int ii = 0; ii < i_eig; ii++) T[tidx(i_eig, ii)] = c.dot(mmp_prev, V[ii]).real() / std::sqrt(res_cur);
      } else if (i_eig != 0) {
        T[tidx(i_eig, i_eig - 1)] = -std::sqrt(beta) / alpha;
      }
      copy(V[i_eig], r);
      launch_scale(s, 1.0 / std::sqrt(res_cur), V[i_eig].view());
      i_eig++;
    }
    alpha_old = alpha;
    alpha = -res_prv / pAp;
    launch_axpby(s, r.view(), alpha, mmp.view(), r.view());
    res_cur = c.norm2(r);
    alpha = -alpha;
    beta_old = beta;
    beta = res_cur / res_prv;
    launch_axpby(s, sol.view(), alpha, dir.view(), sol.view());
    launch_axpby(s, dir.view(), beta, dir.view(), r.view());
    if (restarted < restart_len && def_len > 0 && res_cur < restart[restarted] * restart[restarted] * src_norm_sq) {
      // deflated restart: sol += U invH U^dag r, r -= A (that), p = r
      restarted++;
      deflate(r, dir);
      launch_axpby(s, sol.view(), 1.0, dir.view(), sol.view());
      c.mdagm(mmp, dir);
      launch_axpby(s, r.view(), -1.0, mmp.view(), r.view());
      res_cur = c.norm2(r);
      copy(dir, r);
    }
    if (res_cur <= stp) break;
  }
  c.mdagm(mmp, sol);
  launch_axpby(s, r.view(), -1.0, mmp.view(), src.view());
  if (true_res) *true_res = std::sqrt(c.norm2(r) / src_norm_sq);
  CPSGPU_CUDA(cudaStreamSynchronize(s));
  return iter;
}

// DiracOp::Ritz (ritz.C:152-532): the N_eig-th lowest eigenpair of A =
// MatPcDagMatPc (or -A, RitzMatOper NEG_MATPCDAG_MATPC) by conjugate-gradient
// minimisation of the Ritz functional orthogonal to psi_all[0..N_eig-1),
// starting from psi_all[N_eig-1], which receives the eigenvector.  The
// reference's steps and scalar recurrences (the rotation angle from mu, d,
// g2, p2; the restart and renormalisation rules) run on the host; every
// vector stays on the device.  Returns k, or -1 after MaxCG iterations.
int ritz(Dirac &D, std::vector<Field> &psi_all, int N_eig, const RitzArgs &ra, double *lambda_out) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  Ctx c{D, L, OpWork(), L.scratch_st.as<SolverScalars>(), nullptr, (size_t)L.vh * D.ls};
  L.partials.ensure((size_t)c.blocks() * 2 * sizeof(double));
  c.partials = L.partials.as<double>();
  Field psi(PREC_DOUBLE, L.vh, D.ls, 1), p(PREC_DOUBLE, L.vh, D.ls, 1), Apsi(PREC_DOUBLE, L.vh, D.ls, 1),
      Ap(PREC_DOUBLE, L.vh, D.ls, 1);
  auto ritz_mat = [&](Field &out, const Field &in) {
    c.mdagm(out, in);
    if (ra.neg) launch_scale(s, -1.0, out.view());
  };
  const int nn = N_eig - 1;
  auto gram_schm = [&](Field &v, int upto) {  // v -= <psi_all[i], v> psi_all[i]
    for (int i = 0; i < upto; i++) c.caxpy(v, -c.dot(psi_all[i], v), psi_all[i], v);
  };
  auto copy = [&](Field &dst, const Field &from) {
    CPSGPU_CUDA(cudaMemcpyAsync(dst.data.ptr, from.data.ptr, dst.data.bytes, cudaMemcpyDeviceToDevice, s));
  };
  double acc = 2.0e-24;
  acc *= acc;
  double rsda_sq = ra.RsdR_a * ra.RsdR_a;
  const double rsdr_sq = ra.RsdR_r * ra.RsdR_r;
  rsda_sq = (rsda_sq > acc) ? rsda_sq : acc;
  copy(psi, psi_all[nn]);
  gram_schm(psi, nn);
  double d = std::sqrt(c.norm2(psi)), ct = 1.0 / d, st, mu, lambda, g2, p2, g2_0, del_lam, rsd, s1, s2, s3, a, b;
  launch_scale(s, ct, psi.view());
  ritz_mat(Apsi, psi);
  if (ra.ProjApsiP == 1) gram_schm(Apsi, nn);
  mu = c.dot(psi, Apsi).real();
  lambda = mu;
  launch_axpby(s, p.view(), -lambda, psi.view(), Apsi.view());
  g2 = c.norm2(p);
  p2 = g2;
  g2_0 = g2 * ra.Cv_fact;
  g2_0 = (g2_0 > acc) ? g2_0 : acc;
  rsd = rsdr_sq * lambda * lambda;
  rsd = (rsda_sq > rsd) ? rsda_sq : rsd;
  int result = -1;
  if (ra.Kalk_Sim == 0 && ra.N_min <= 0 && g2 <= rsd) {
    copy(psi_all[nn], psi);
    result = 0;
  } else {
    del_lam = mu;
    for (int k = 1; k <= ra.MaxCG; ++k) {
      ritz_mat(Ap, p);
      if (ra.ProjApsiP == 1) gram_schm(Ap, nn);
      d = c.dot(p, Ap).real() / p2;
      s1 = 0.5 * (mu + d);
      s2 = 0.5 * (mu - d);
      p2 = 1.0 / std::sqrt(p2);
      s3 = g2 * p2;
      a = (s2 > 0.0) ? s2 : -s2;
      if (a >= s3) {
        d = s3 / s2;
        d = std::sqrt(1.0 + d * d);
        a = a * d;
      } else {
        d = s2 / s3;
        d = std::sqrt(1.0 + d * d);
        a = s3 * d;
      }
      s2 /= a;  // cos(delta)
      s3 /= a;  // sin(delta)
      if (s2 > 0) {
        s2 = 0.5 * (1.0 + s2);
        d = -std::sqrt(s2);  // sin(theta)
        s2 = -0.5 * s3 / d;  // cos(theta)
      } else {
        s2 = 0.5 * (1.0 - s2);
        s2 = std::sqrt(s2);  // cos(theta)
        d = -0.5 * s3 / s2;  // sin(theta)
      }
      s1 = 2.0 * a * d * d;
      mu -= s1;
      lambda = mu;
      del_lam = s1;
      st = d * p2;
      ct = s2;
      // psi = ct psi + st p;  Apsi = ct Apsi + st Ap;  g = Ap = Apsi - lambda psi
      launch_scale(s, ct, psi.view());
      launch_axpby(s, psi.view(), st, p.view(), psi.view());
      launch_scale(s, ct, Apsi.view());
      launch_axpby(s, Apsi.view(), st, Ap.view(), Apsi.view());
      launch_axpby(s, Ap.view(), -lambda, psi.view(), Apsi.view());
      s1 = g2;
      g2 = c.norm2(Ap);
      rsd = rsdr_sq * lambda * lambda;
      rsd = (rsda_sq > rsd) ? rsda_sq : rsd;
      st = ra.Rsdlam * std::fabs(mu);
      if ((ra.Kalk_Sim == 0 && k >= ra.N_min && (std::fabs(mu) < ra.Cutl_zero || (g2 <= rsd && del_lam <= st))) ||
          (ra.Kalk_Sim == 1 &&
           (del_lam <= st || std::fabs(mu) < ra.Cutl_zero || (k >= ra.N_min && (g2 < g2_0 || k >= ra.N_max))))) {
        gram_schm(psi, nn);
        d = std::sqrt(c.norm2(psi));
        launch_scale(s, 1.0 / d, psi.view());
        ritz_mat(Apsi, psi);
        mu = c.dot(psi, Apsi).real();
        lambda = mu;
        copy(psi_all[nn], psi);
        result = k;
        break;
      }
      b = ct * g2 / s1;
      ct *= 0.05 * b;
      d = std::sqrt(g2);
      ct /= (p2 * d);
      if (ct > 1.0) {
        copy(p, Ap);  // restart: p = g
      } else {
        c.caxpy(p, -c.dot(psi, p), psi, p);  // p -= <psi, p> psi
        launch_axpby(s, p.view(), b, p.view(), Ap.view());
      }
      if (k % ra.n_renorm == 0) {
        gram_schm(psi, nn);
        d = std::sqrt(c.norm2(psi));
        launch_scale(s, 1.0 / d, psi.view());
        ritz_mat(Apsi, psi);
        if (ra.ProjApsiP == 1) gram_schm(Apsi, nn);
        mu = c.dot(psi, Apsi).real();
        lambda = mu;
        launch_axpby(s, Ap.view(), -lambda, psi.view(), Apsi.view());
        g2 = c.norm2(Ap);
        gram_schm(p, nn);
        c.caxpy(p, -c.dot(psi, p), psi, p);
        cd xp = g2 - c.dot(Ap, p);
        xp *= 1.0 / g2;
        c.caxpy(p, xp, Ap, p);
      } else if (ra.ProjApsiP == 1 && nn > 0) {
        gram_schm(psi, nn);
        gram_schm(p, nn);
      }
      p2 = c.norm2(p);
    }
    if (result < 0) copy(psi_all[nn], psi);
  }
  if (lambda_out) *lambda_out = lambda;
  CPSGPU_CUDA(cudaStreamSynchronize(s));
  return result;
}

// DiracOp::Jacobi (jacobi.C:48-268): Jacobi rotations of the vectors psi
// that zero the complex off-diagonal elements off[j(j-1)/2 + i] =
// <psi_i, A psi_j> (i < j) of the small matrix with diagonal lambda, until
// none exceeds |lambda_i lambda_j| Toler^2; then the pairs sorted by
// |lambda|.  The 2 x 2 rotations and the bookkeeping of the other elements
// are the reference's, on the host; the vectors rotate on the device.
// Returns the sweep count, -1 after N_max sweeps.
int jacobi(Dirac &D, std::vector<Field> &psi, int N_eig, double *lambda, std::vector<cd> &off, double Toler,
           int N_max) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  Ctx c{D, L, OpWork(), L.scratch_st.as<SolverScalars>(), nullptr, (size_t)L.vh * D.ls};
  L.partials.ensure((size_t)c.blocks() * 2 * sizeof(double));
  c.partials = L.partials.as<double>();
  Field t1(PREC_DOUBLE, L.vh, D.ls, 1), t2(PREC_DOUBLE, L.vh, D.ls, 1);
  auto copy = [&](Field &dst, const Field &from) {
    CPSGPU_CUDA(cudaMemcpyAsync(dst.data.ptr, from.data.ptr, dst.data.bytes, cudaMemcpyDeviceToDevice, s));
  };
  const double tol_sq = Toler * Toler;
  for (int k = 0; k <= N_max; k++) {
    int i_rot = 0, ij = 0;
    for (int j = 1; j < N_eig; j++)
      for (int i = 0; i < j; i++, ij++) {
        double dd = std::norm(off[ij]);
        double ftmp = std::fabs(lambda[i] * lambda[j] * tol_sq);
        if (dd <= ftmp) continue;
        i_rot++;
        dd = std::sqrt(dd);
        const double acc = 100.0 * dd, diff_l = lambda[j] - lambda[i];
        double t, cs, sn;
        ftmp = std::fabs(diff_l);
        if ((ftmp + acc) == ftmp) {
          t = dd / diff_l;
        } else {
          const double theta = 0.5 * diff_l / dd;
          t = 1.0 / (std::fabs(theta) + std::sqrt(1.0 + theta * theta));
          if (theta < 0.0) t = -t;
        }
        if (diff_l >= 0) {
          cs = 1.0 / std::sqrt(1.0 + t * t);
          sn = -t * cs;
        } else {
          sn = 1.0 / std::sqrt(1.0 + t * t);
          cs = t * sn;
        }
        double al1 = cs * cs * lambda[i], al2 = cs * cs * lambda[j];
        al1 += sn * sn * lambda[j];
        al2 += sn * sn * lambda[i];
        ftmp = 2.0 * dd * sn * cs;
        lambda[i] = al1 + ftmp;
        lambda[j] = al2 - ftmp;
        const double v11 = cs;
        const cd v12 = (sn / dd) * off[ij], v21 = -std::conj(v12);
        off[ij] = 0.0;
        // psi_i <- v11 psi_i - v21 psi_j;  psi_j <- v11 psi_j - v12 psi_i
        copy(t1, psi[i]);
        launch_scale(s, v11, t1.view());
        c.caxpy(t1, -v21, psi[j], t1);
        copy(t2, psi[j]);
        launch_scale(s, v11, t2.view());
        c.caxpy(t2, -v12, psi[i], t2);
        copy(psi[i], t1);
        copy(psi[j], t2);
        for (int m = 0; m < N_eig; m++) {
          if (m == i || m == j) continue;
          if (m < i) {
            const int mi = i * (i - 1) / 2 + m, mj = j * (j - 1) / 2 + m;
            const cd c1 = off[mi] * v11 - off[mj] * v21, c2 = off[mj] * v11 - off[mi] * v12;
            off[mi] = c1;
            off[mj] = c2;
          } else if (m < j) {
            const int mi = m * (m - 1) / 2 + i, mj = j * (j - 1) / 2 + m;
            const cd c1 = std::conj(off[mi]) * v11 - off[mj] * v21, c2 = off[mj] * v11 - std::conj(off[mi]) * v12;
            off[mi] = std::conj(c1);
            off[mj] = c2;
          } else {
            const int mi = m * (m - 1) / 2 + i, mj = m * (m - 1) / 2 + j;
            const cd c1 = std::conj(off[mi]) * v11 - std::conj(off[mj]) * v21;
            const cd c2 = std::conj(off[mj]) * v11 - std::conj(off[mi]) * v12;
            off[mi] = std::conj(c1);
            off[mj] = std::conj(c2);
          }
        }
      }
    if (i_rot == 0) {
      for (int j = 1; j < N_eig; j++)
        for (int i = 0; i < j; i++)
          if (std::fabs(lambda[j]) < std::fabs(lambda[i])) {
            std::swap(lambda[i], lambda[j]);
            std::swap(psi[i], psi[j]);
          }
      CPSGPU_CUDA(cudaStreamSynchronize(s));
      return k;
    }
  }
  CPSGPU_CUDA(cudaStreamSynchronize(s));
  return -1;
}

// DiracOpWilsonTypes::RitzEig (eigen_wilson.C:89-586) with RitzEigMat =
// (-)MatPcDagMatPc.  Kalkreuter-Simma sweeps (lines 187-300): Ritz on each
// vector in turn, the off-diagonal elements <psi_j, A psi_i> and Jacobi,
// until the largest relative eigenvalue change between sweeps is <= Rsdlam;
// plain successive Ritz calls when N_eig = 1 or Kalk_Sim = 0.  Then the
// projection stage (lines 354-583): rows of the matrix of A between the
// vectors whose squared norm is below 0.98 lambda_old mark those vectors
// invalid; every vector from the first invalid one on becomes
// (1 +- A / sqrt|lambda_old|) psi, normalised; a normalised Gram-Schmidt
// pass; the matrix elements again and Jacobi with tolerance 1e-5.
// lambda_H[0..N): the last Jacobi's eigenvalues, lambda_H[N..2N): lambda_old.
// Returns the total Ritz iteration count, or the reference's -1 (a Ritz call
// hit MaxCG) / -2 (the sweeps ran out, with its test n_KS >= N_KS_max after
// the loop), or -3 when a Jacobi call ran out (the reference exits).
int ritz_eig(Dirac &D, std::vector<Field> &psi, const RitzArgs &ra0, int N_KS_max, double *lambda_H,
             int *valid_eig) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  Ctx c{D, L, OpWork(), L.scratch_st.as<SolverScalars>(), nullptr, (size_t)L.vh * D.ls};
  L.partials.ensure((size_t)c.blocks() * 2 * sizeof(double));
  c.partials = L.partials.as<double>();
  const int N_eig = (int)psi.size();
  RitzArgs ra = ra0;
  ra.Cutl_zero = 0.0;
  int Kalk_Sim = ra.Kalk_Sim;
  if (N_eig == 1) Kalk_Sim = 0;
  if (Kalk_Sim == 0) N_KS_max = 0;
  double *lambda = lambda_H, *lambda_old = lambda_H + N_eig;
  std::vector<cd> off(N_eig > 1 ? (size_t)N_eig * (N_eig - 1) / 2 : 1, 0.0);
  Field tmp(PREC_DOUBLE, L.vh, D.ls, 1), tmp2(PREC_DOUBLE, L.vh, D.ls, 1);
  auto eig_mat = [&](Field &out, const Field &in) {
    c.mdagm(out, in);
    if (ra.neg) launch_scale(s, -1.0, out.view());
  };
  auto herm_elements = [&](int n_vec) {
    int ij = 0;
    for (int i = 0; i < n_vec; i++) {
      eig_mat(tmp, psi[i]);
      lambda[i] = c.dot(psi[i], tmp).real();
      for (int j = 0; j < i; j++) off[ij++] = c.dot(psi[j], tmp);
    }
  };
  auto normalise = [&](Field &x) { launch_scale(s, 1.0 / std::sqrt(c.norm2(x)), x.view()); };
  for (int k = 0; k < N_eig; k++) {
    lambda_old[k] = 1.0;
    valid_eig[k] = 0;
  }
  int ncg_tot = 0;
  double lambda_t, del_lamb = 1.0;
  if (Kalk_Sim == 1) {
    ra.Kalk_Sim = 1;
    int n_KS;
    for (n_KS = 1; n_KS <= N_KS_max && del_lamb > ra.Rsdlam; n_KS++) {
      int ij = 0;
      for (int i = 0; i < N_eig; i++) {
        // Ritz on psi[0..i]: the first i held fixed, psi[i] the start
        const int ncnt = ritz(D, psi, i + 1, ra, &lambda_t);
        if (ncnt < 0) return ncnt;
        ncg_tot += ncnt;
        lambda[i] = lambda_t;
        eig_mat(tmp, psi[i]);
        for (int j = 0; j < i; j++) off[ij++] = c.dot(psi[j], tmp);
      }
      if (jacobi(D, psi, N_eig, lambda, off, ra.RsdR_a, 50) < 0) return -3;
      if (n_KS == 1) {
        for (int i = 0; i < N_eig; i++) lambda_old[i] = lambda[i];
      } else {
        del_lamb = 0.0;
        for (int i = 0; i < N_eig; i++) {
          lambda_t = std::fabs((lambda_old[i] - lambda[i]) / lambda[i]);
          if (lambda_t > del_lamb) del_lamb = lambda_t;
          lambda_old[i] = lambda[i];
        }
      }
    }
    if (n_KS >= N_KS_max) return -2;
  } else {
    ra.Kalk_Sim = 0;
    ra.N_min = 0;
    ra.N_max = 0;
    for (int i = 0; i < N_eig; i++) {
      ncg_tot += ritz(D, psi, i + 1, ra, &lambda_t);
      lambda_old[i] = lambda_t;
    }
  }
  // projection onto the eigenvectors of RitzEigMat itself
  herm_elements(N_eig);
  for (int i = 0; i < N_eig; i++) valid_eig[i] = 1;
  for (bool looping = true; looping;) {
    looping = false;
    for (int i = 0; i < N_eig; i++) {
      if (!valid_eig[i]) continue;
      const double rEig2 = 1.0 / lambda_old[i];
      double sum = lambda[i] * lambda[i] * rEig2;
      int xy = 0;
      for (int x = 0; x < N_eig; x++)
        for (int y = 0; y < x; y++) {
          if ((x == i && valid_eig[y]) || (y == i && valid_eig[x])) sum += std::norm(off[xy]) * rEig2;
          xy++;
        }
      if (sum < 0.98) {
        valid_eig[i] = 0;
        looping = true;
      }
    }
  }
  int N_dp = 0, i;
  for (i = 0; i < N_eig; i++) {
    if (valid_eig[i] == 1) N_dp++;
    else break;
  }
  for (i++; i < N_eig; i++) valid_eig[i] = 0;
  for (; N_dp < N_eig; N_dp++) {
    valid_eig[N_dp] = 1;
    const double lam = std::sqrt(std::fabs(lambda_old[N_dp]));
    eig_mat(tmp, psi[N_dp]);
    const double sign = c.dot(tmp, psi[N_dp]).real() < 0 ? -1.0 : 1.0;
    launch_axpby(s, tmp2.view(), sign / lam, tmp.view(), psi[N_dp].view());
    cd snorm = 0.0, onorm = 0.0;
    for (int k = 0; k < N_dp; k++) snorm += c.dot(tmp2, psi[k]);
    launch_axpby(s, tmp.view(), -sign / lam, tmp.view(), psi[N_dp].view());
    for (int k = 0; k < N_dp; k++) onorm += c.dot(tmp, psi[k]);
    const Field &pick = std::norm(onorm) > std::norm(snorm) ? tmp2 : tmp;
    CPSGPU_CUDA(cudaMemcpyAsync(psi[N_dp].data.ptr, pick.data.ptr, pick.data.bytes, cudaMemcpyDeviceToDevice, s));
    normalise(psi[N_dp]);
  }
  // GramSchmNorm(psi[b], psi[a]) (eigen_wilson.C:78-85) for every a < b
  for (int a = 0; a < N_eig; a++)
    for (int b = a + 1; b < N_eig; b++) {
      c.caxpy(psi[b], -c.dot(psi[a], psi[b]), psi[a], psi[b]);
      normalise(psi[b]);
    }
  int min_dim = 0;
  for (int k = 0; k < N_eig; k++)
    if (valid_eig[k]) min_dim++;
  herm_elements(min_dim);
  if (jacobi(D, psi, min_dim, lambda, off, 1.0e-5, 50) < 0) return -3;
  return ncg_tot;
}

// ------------------------------------------------- implicitly restarted Lanczos

namespace {

// tqri / QRtrf / eigsrt (eigen_solver.C:206-305, 1442-1498) on the host:
// the symmetric tridiagonal (d, e) and its rotations Q (row-major, ld)
double lz_pythag(double a, double b) {
  const double aa = std::fabs(a), ab = std::fabs(b);
  if (aa > ab) return aa * std::sqrt(1.0 + (ab / aa) * (ab / aa));
  return ab == 0.0 ? 0.0 : ab * std::sqrt(1.0 + (aa / ab) * (aa / ab));
}

void lz_qrtrf(double *d, double *e, int nk, double *Q, int ld, double dsh, int kmin, int kmax) {
  auto rot = [&](int k, double c, double s) {
    for (int i = 0; i < nk; i++) {
      const double q1 = Q[i * ld + k], q2 = Q[i * ld + k + 1];
      Q[i * ld + k] = c * q1 - s * q2;
      Q[i * ld + k + 1] = s * q1 + c * q2;
    }
  };
  auto step = [&](int k, double c, double s) {
    const double t1 = d[k], t2 = d[k + 1], tb = e[k];
    d[k] = c * c * t1 + s * s * t2 - 2.0 * c * s * tb;
    d[k + 1] = s * s * t1 + c * c * t2 + 2.0 * c * s * tb;
    e[k] = c * s * (t1 - t2) + (c * c - s * s) * tb;
  };
  int k = kmin;
  double den = 1.0 / lz_pythag(d[k] - dsh, e[k]);
  double c = (d[k] - dsh) * den, s = -e[k] * den;
  step(k, c, s);
  double x = -s * e[k + 1];
  e[k + 1] *= c;
  rot(k, c, s);
  for (k = kmin + 1; k < kmax; k++) {
    den = 1.0 / lz_pythag(x, e[k - 1]);
    c = e[k - 1] * den;
    s = -x * den;
    step(k, c, s);
    e[k - 1] = c * e[k - 1] - s * x;
    if (k != kmax - 1) {
      x = -s * e[k + 1];
      e[k + 1] *= c;
    }
    rot(k, c, s);
  }
}

int lz_tqri(double *d, double *e, int nk, int n, double *Q, int ld) {
  int kmin = 0, kmax = nk - 1, iter = 0;
  while (iter < n * 100) {
    const double dsub = d[kmax] - d[kmax - 1];
    double dd = lz_pythag(dsub, 2.0 * e[kmax - 1]);
    lz_qrtrf(d, e, nk, Q, ld, 0.5 * (d[kmax - 1] + d[kmax] + (dsub < 0 ? -std::fabs(dd) : std::fabs(dd))), kmin,
             kmax);
    int j;
    for (j = kmax; j >= kmin + 1; j--) {
      dd = std::fabs(d[j - 1]) + std::fabs(d[j]);
      if (std::fabs(e[j - 1]) + dd > dd) {
        kmax = j;
        break;
      }
    }
    if (j == kmin) return iter;
    for (j = 0; j < kmax; j++) {
      dd = std::fabs(d[j]) + std::fabs(d[j + 1]);
      if (std::fabs(e[j]) + dd > dd) {
        kmin = j;
        break;
      }
    }
    iter++;
  }
  return iter;
}

// descending selection sort; with Q its columns follow (the vector-free
// form keeps the last of equal values, as the reference's >= does)
void lz_eigsrt(double *d, double *Q, int ld, int n) {
  for (int i = 0; i < n - 1; i++) {
    int k = i;
    double p = d[i];
    for (int j = i + 1; j < n; j++)
      if (Q ? d[j] > p : d[j] >= p) {
        p = d[j];
        k = j;
      }
    if (k != i) {
      d[k] = d[i];
      d[i] = p;
      if (Q)
        for (int j = 0; j < n; j++) std::swap(Q[j * ld + i], Q[j * ld + k]);
    }
  }
}

struct LzDev {
  Ctx &c;
  const LanczosArgs &a;
  cudaStream_t s;
  double c0, c1;
  Field tmp1, tmp2, vtmp, vtmp2, rf;
  size_t nreal() const { return (size_t)24 * c.sites; }
  unsigned grid() const { return (unsigned)std::min<size_t>((nreal() + 255) / 256, 148 * 16); }
  void ritz(Field &out, const Field &in, int neg) {
    c.mdagm(out, in);
    if (neg) launch_scale(s, -1.0, out.view());
  }
  void cheb(Field &out, double a_, double b_, const Field &x, double c_, const Field &y) {
    cheb_kernel<<<grid(), 256, 0, s>>>((double *)out.data.ptr, a_, b_, (const double *)x.data.ptr, c_,
                                       (const double *)y.data.ptr, nreal());
    CPSGPU_CUDA(cudaGetLastError());
    launch_counter()++;
  }
  // out = T_Npol(Q) in (DiracOpDwf::RitzMat(out, in, cheby_arg), d_op_dwf.C:852-960)
  void filter(Field &out, const Field &in) {
    Field *t = &tmp1, *t2 = &tmp2;
    CPSGPU_CUDA(cudaMemcpyAsync(t2->data.ptr, in.data.ptr, in.data.bytes, cudaMemcpyDeviceToDevice, s));
    ritz(*t, in, a.neg_lanczos);
    cheb(*t, 0.5 * c1 * c0, -0.5 * c1, in, 0.0, in);
    for (int i = 2; i <= a.Npol; i++) {
      ritz(out, *t, a.neg_lanczos);
      cheb(out, c1 * c0, -c1, *t, -1.0, *t2);
      if (i != a.Npol) {
        std::swap(t, t2);
        CPSGPU_CUDA(cudaMemcpyAsync(t->data.ptr, out.data.ptr, out.data.bytes, cudaMemcpyDeviceToDevice, s));
      }
    }
  }
  double ddot(const Field &x, const Field &y) { return c.dot(x, y).real(); }
  void to_f(Field &dst, const Field &src) { launch_convert(s, PREC_SINGLE, dst.view(), PREC_DOUBLE, src.view()); }
  void to_d(Field &dst, const Field &src) { launch_convert(s, PREC_DOUBLE, dst.view(), PREC_SINGLE, src.view()); }
  // lanczos_GramSchm_test (eigen_solver.C:1341-1390): r against V[0..nvec) in FP32
  void gram_schm_f(Field &r, std::vector<Field> &V, int nvec) {
    to_f(rf, r);
    for (int i = 0; i < nvec; i++) {
      cdot_f_kernel<<<c.blocks(), TPB, 0, s>>>(V[i].view(), rf.view(), c.partials, c.sites);
      CPSGPU_CUDA(cudaGetLastError());
      launch_counter()++;
      launch_finalize(s, 2, c.partials, c.st, RED_STORE, c.blocks(), 1, GATE_NONE);
      double xp[2];
      CPSGPU_CUDA(cudaMemcpyAsync(xp, c.st->sum, sizeof(xp), cudaMemcpyDeviceToHost, s));
      CPSGPU_CUDA(cudaStreamSynchronize(s));
      caxpy_f_kernel<<<c.blocks(), TPB, 0, s>>>(rf.view(), -(float)xp[0], -(float)xp[1], V[i].view(), c.sites);
      CPSGPU_CUDA(cudaGetLastError());
      launch_counter()++;
    }
    to_d(r, rf);
  }
  // DiracOp::lanczos (lanczos.C:756-883): steps k0..m-1
  void steps(int k0, int m, Field &r, std::vector<Field> &V, double *alpha, double *beta) {
    const double ff = std::sqrt(c.norm2(r));
    launch_axpby(s, vtmp.view(), 1.0 / ff, r.view(), zero_view());
    to_f(V[k0], vtmp);
    for (int k = k0; k < m; k++) {
      to_d(vtmp, V[k]);
      filter(r, vtmp);
      if (k > 0) {
        to_d(vtmp2, V[k - 1]);
        launch_axpby(s, r.view(), -beta[k - 1], vtmp2.view(), r.view());
      }
      alpha[k] = ddot(vtmp, r);
      launch_axpby(s, r.view(), -alpha[k], vtmp.view(), r.view());
      beta[k] = std::sqrt(c.norm2(r));
      if (k > 0) gram_schm_f(r, V, k + 1);
      if (k == 0 || k + 1 < m) {
        launch_axpby(s, vtmp.view(), 1.0 / beta[k], r.view(), zero_view());
        to_f(V[k + 1], vtmp);
      }
    }
  }
  Field zero;
  SpinorView zero_view() { return zero.view(); }
};

}  // namespace

// DiracOp::ImpResLanczos (d_op_base/comsrc/lanczos.C:193-745) for the DWF /
// Mobius Chebyshev-filtered RitzMat: the reference's steps (its oracle
// restatement is orc_lanczos) with the float Lanczos vectors V, every
// vector operation and the filter's MatPcDagMatPc applications on the
// device, the m x m tridiagonal's QR algebra on the host.  Returns the
// restart count; -1 on a NaN residual (the reference exits).
int imp_res_lanczos(Dirac &D, std::vector<Field> &V, double *alpha, const LanczosArgs &a) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  Ctx c{D, L, OpWork(), L.scratch_st.as<SolverScalars>(), nullptr, (size_t)L.vh * D.ls};
  L.partials.ensure((size_t)c.blocks() * 2 * sizeof(double));
  c.partials = L.partials.as<double>();
  const int nk = a.nk, nt = a.nt, np = a.np, m = nk + np;
  LzDev z{c, a, s};
  const double aa = a.p0 * a.p0, bb = (a.p1 + std::fabs(a.eigen_shift)) * (a.p1 + std::fabs(a.eigen_shift));
  z.c1 = 2.0 * (aa + bb) / (aa - bb);
  z.c0 = 2.0 / (aa + bb);
  for (Field *f : {&z.tmp1, &z.tmp2, &z.vtmp, &z.vtmp2, &z.zero}) f->create(PREC_DOUBLE, L.vh, D.ls, 1);
  z.rf.create(PREC_SINGLE, L.vh, D.ls, 1);
  launch_zero(s, z.zero);
  Field r(PREC_DOUBLE, L.vh, D.ls, 1), Apsi(PREC_DOUBLE, L.vh, D.ls, 1);
  std::vector<Field> Vn(m);
  for (auto &f : Vn) f.create(PREC_SINGLE, L.vh, D.ls, 1);
  std::vector<double> beta(m, 0.0), ttbeta(m), shifts(m), Q((size_t)m * m), QZ((size_t)m * m);
  DeviceBuffer vptr, wptr, qzbuf;
  vptr.alloc(sizeof(float *) * m);
  wptr.alloc(sizeof(float *) * m);
  qzbuf.alloc(sizeof(double) * m * m);
  // Vnew[k] = sum_j V[j] Q[j][k]; entries |Q| <= qmin left out (qmin < 0: none)
  auto rotate = [&](double qmin) {
    for (int j = 0; j < m; j++)
      for (int k = 0; k < m; k++) {
        const double w = Q[(size_t)j * m + k];
        QZ[(size_t)j + (size_t)m * k] = (qmin >= 0.0 && !(std::fabs(w) > qmin)) ? 0.0 : w;
      }
    std::vector<float *> vp(m), wp(m);
    for (int j = 0; j < m; j++) {
      vp[j] = (float *)V[j].data.ptr;
      wp[j] = (float *)Vn[j].data.ptr;
    }
    CPSGPU_CUDA(cudaMemcpyAsync(vptr.ptr, vp.data(), sizeof(float *) * m, cudaMemcpyHostToDevice, s));
    CPSGPU_CUDA(cudaMemcpyAsync(wptr.ptr, wp.data(), sizeof(float *) * m, cudaMemcpyHostToDevice, s));
    CPSGPU_CUDA(cudaMemcpyAsync(qzbuf.ptr, QZ.data(), sizeof(double) * m * m, cudaMemcpyHostToDevice, s));
    vec_mult_f_kernel<<<z.grid(), 256, 0, s>>>(vptr.as<float *>(), m, qzbuf.as<double>(), m, wptr.as<float *>(),
                                                z.nreal());
    CPSGPU_CUDA(cudaGetLastError());
    launch_counter()++;
    CPSGPU_CUDA(cudaStreamSynchronize(s));
    for (int j = 0; j < m; j++) std::swap(V[j], Vn[j]);
  };
  auto identity = [&]() {
    std::fill(Q.begin(), Q.end(), 0.0);
    for (int j = 0; j < m; j++) Q[(size_t)j * m + j] = 1.0;
  };
  z.to_d(r, V[0]);
  for (int j = 0; j < m; j++) alpha[j] = 0.0;
  z.steps(0, m, r, V, alpha, beta.data());
  int it = 1;
  while (it <= a.maxiters) {
    shifts.assign(alpha, alpha + m);
    ttbeta = beta;
    identity();
    lz_tqri(shifts.data(), ttbeta.data(), m, m, Q.data(), m);
    lz_eigsrt(shifts.data(), nullptr, m, m);
    identity();
    for (int i = 0; i < np; i++) lz_qrtrf(alpha, beta.data(), m, Q.data(), m, shifts[nk + i], 0, m - 1);
    rotate(-1.0);
    launch_scale(s, Q[(size_t)(m - 1) * m + nk - 1], r.view());
    if (nk < m) {
      z.to_d(Apsi, V[nk]);
      launch_axpby(s, r.view(), beta[nk - 1], Apsi.view(), r.view());
    }
    beta[nk - 1] = std::sqrt(c.norm2(r));
    if (it % a.conv_check == 0) {
      int Ndone = 0;
      shifts.assign(alpha, alpha + m);
      ttbeta = beta;
      identity();
      lz_tqri(shifts.data(), ttbeta.data(), nk, m, Q.data(), m);
      lz_eigsrt(shifts.data(), Q.data(), m, m);
      for (int k = 0; k < nk; k++) {
        launch_zero(s, z.vtmp);
        for (int j = 0; j < nk; j++) {
          z.to_d(z.vtmp2, V[j]);
          launch_axpby(s, z.vtmp.view(), Q[(size_t)j * m + k], z.vtmp2.view(), z.vtmp.view());
        }
        z.ritz(Apsi, z.vtmp, a.neg_conv);
        const double bt = std::sqrt(c.norm2(z.vtmp));
        const double alp = z.ddot(Apsi, z.vtmp) / bt;
        launch_axpby(s, Apsi.view(), -alp, z.vtmp.view(), Apsi.view());
        const double rnorm = std::sqrt(c.norm2(Apsi)) / bt;
        if (rnorm < a.stop_res && k < nt) Ndone++;
        if (std::isnan(rnorm)) return -1;
      }
      if (Ndone == nt) break;
    }
    z.steps(nk, m, r, V, alpha, beta.data());
    it++;
  }
  if (it == a.maxiters + 1) it--;
  shifts.assign(alpha, alpha + m);
  ttbeta = beta;
  identity();
  lz_tqri(shifts.data(), ttbeta.data(), nk, m, Q.data(), m);
  lz_eigsrt(shifts.data(), Q.data(), m, m);
  rotate(1e-16);
  for (int i = 0; i < nt; i++) {
    z.to_d(z.vtmp, V[i]);
    z.ritz(Apsi, z.vtmp, a.neg_conv);
    alpha[i] = z.ddot(Apsi, z.vtmp);
  }
  return it;
}

}  // namespace cpsgpu
