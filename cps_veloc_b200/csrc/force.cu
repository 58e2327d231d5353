// HMC fermion force of the Wilson and Shamir-DWF actions:
// Fwilson::EvolveMomFforce (f_wilson.C:470-687) and FdwfBase::EvolveMomFforce
// (f_dwf_base_force.C:41-300), with DiracOp*::CalcHmdForceVecs
// (d_op_wilson.C:466-507, d_op_dwf.C:682-733) in front of them.
//
//   v1 = (chi, D chi),  v2 = (psi, D^dag psi),  psi = -kappa^2 MatPc chi
//
// are built on the device from the library's own operators.  The force loop
// is one kernel, a thread per (checkerboard site, parity, mu, slice group), that reads
// the four fields where the reference reads them after converting them to
// CANONICAL order (no conversion here: the kernel indexes the device layout
// of each half directly) and, per link,
//
//   T   = sum_s sprojTr(1 - g_mu)[v1(x+mu, s), v2(x, s)]
//             + sprojTr(1 + g_mu)[v2(x+mu, s), v1(x, s)]
//   F   = U_mu(x) T;  F <- 1/2 (F - F^dag) - 1/3 i Im tr(...);  F *= coeff
//   mom(x, mu) += F,  with coeff = -2 dt (negated where x+mu wraps an
//   antiperiodic direction), and L1, L2, Linf of Matrix::norm() = -2 Re tr F^2.
//
// sprojTr(1 + k g)[a, w] = Tr_spin[(1 + k g) a w^dag] is evaluated on the two
// projected spins: (1 + k g) is hermitian with (1 + k g)^2 = 2 (1 + k g), so
// the trace equals sum over s = 0, 1 of h_a(s) h_w(s)^dag with h = the first
// two spin rows of (1 + k g) applied to a and to w (the reference sums all
// four spins; the value is the same up to rounding).
//
// mom is the reference's CANONICAL Matrix field, [lexicographic site][mu]
// [row][col][re, im], kept as is on the device.
#include <cmath>

#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

namespace {

constexpr int FORCE_TPB = 128;

struct ForceParams {
  int L[4];
  int hx;
  long vh;
  int ls;
  double bc[4];
  double scale;    // mom += scale TrLessAntiHerm(U T), negated where x+mu wraps an antiperiodic direction
  int mobius;      // halves hold one 4D parity in every slice (Mobius) instead of the 5D parity (DWF)
};

struct ForceViews {
  SpinorView v1o, v1e, v2o, v2e;  // odd / even parts of v1 and v2 (WILSON order halves)
  GaugeView U;                    // FP64 18-real links, WILSON parity order
  double *mom;                    // CANONICAL [site][mu][18]
};

// the half of a full field that holds 4D parity p in slice s: for Wilson
// and DWF the odd part holds parity (s + 1) % 2 (convert.C:704-760; ls = 1:
// the odd sites); for Mobius each half holds one 4D parity in every slice
// (convert.C:797-851)
__device__ __forceinline__ const SpinorView &part(const SpinorView &o, const SpinorView &e, int p, int s,
                                                  int mobius) {
  return (mobius ? p : ((p + s) & 1)) ? o : e;
}

// T += sum over the two projected spins of h_a (x) conj(h_w)
__device__ __forceinline__ void outer_acc(cplx<double> (&T)[3][3], const half_spinor<double> &ha,
                                          const half_spinor<double> &hw) {
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const cplx<double> a = ha.h[s][i], w = hw.h[s][j];
        T[i][j].re = fma(a.re, w.re, fma(a.im, w.im, T[i][j].re));
        T[i][j].im = fma(a.im, w.re, fma(-a.re, w.im, T[i][j].im));
      }
}

// T = the spin-traced outer products of one link, summed over the slices
// s = s0, s0 + ds, ... of this thread
template <int MU>
__device__ __forceinline__ void force_trace(const ForceParams &fp, const ForceViews &v, int i, int j, int p, int s0,
                                            int ds, cplx<double> (&T)[3][3]) {
  const int q = 1 - p;  // parity of x + mu
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) T[a][b] = {0.0, 0.0};
  for (int s = s0; s < fp.ls; s += ds) {
    double a[24], w[24];
    // sprojTr(1 - g_mu)[v1(x+mu), v2(x)]
    SpinorIO<PREC_DOUBLE>::load(part(v.v1o, v.v1e, q, s, fp.mobius), s, j, a);
    SpinorIO<PREC_DOUBLE>::load(part(v.v2o, v.v2e, p, s, fp.mobius), s, i, w);
    outer_acc(T, project(a, MU, -1.0), project(w, MU, -1.0));
    // sprojTr(1 + g_mu)[v2(x+mu), v1(x)]
    SpinorIO<PREC_DOUBLE>::load(part(v.v2o, v.v2e, q, s, fp.mobius), s, j, a);
    SpinorIO<PREC_DOUBLE>::load(part(v.v1o, v.v1e, p, s, fp.mobius), s, i, w);
    outer_acc(T, project(a, MU, 1.0), project(w, MU, 1.0));
  }
}

// Block = blockDim.x sites x 4 directions x blockDim.z slice groups of one
// parity: the four links of a site sit in neighbouring warps of one block,
// so the spinors at x that all four read come from L1; thread (tx, mu, g)
// sums the slices g, g + blockDim.z, ...; the groups' sums are added in a
// fixed order through shared memory and group 0 finishes the link.  The two
// parities of a site block are consecutive blocks (blockIdx.x = 2 site block
// + parity), so a half field read as v(x) by one is still in L2 when the
// other reads it as v(x+mu): with all blocks of one parity first, every
// half came from DRAM twice.
__global__ void __launch_bounds__(FORCE_TPB, 3) fforce_kernel(const ForceParams fp, const ForceViews v,
                                                                 double *partials) {
  const int i = (blockIdx.x >> 1) * blockDim.x + threadIdx.x;
  const int p = blockIdx.x & 1, mu = threadIdx.y;
  const bool active = i < fp.vh;
  double red[3] = {0.0, 0.0, 0.0};  // L1, L2 and Linf of this thread
  int x = 0, y = 0, z = 0, t = 0, j = 0;
  bool wrap = false;
  cplx<double> T[3][3];
  if (active) {
    const int hx = fp.hx;
    int r = i / hx;
    const int xh = i - r * hx;
    y = r % fp.L[1];
    r /= fp.L[1];
    z = r % fp.L[2];
    t = r / fp.L[2];
    x = 2 * xh + ((y + z + t + p) & 1);
    // the forward neighbour x + mu (its checkerboard index j) and whether it wraps
    const int cmu = mu == 0 ? x : mu == 1 ? y : mu == 2 ? z : t;
    const int Lmu = mu == 0 ? fp.L[0] : mu == 1 ? fp.L[1] : mu == 2 ? fp.L[2] : fp.L[3];
    const int smu = mu == 1 ? hx : mu == 2 ? hx * fp.L[1] : hx * fp.L[1] * fp.L[2];
    wrap = (cmu == Lmu - 1);
    if (mu == 0) j = i - xh + ((wrap ? 0 : x + 1) >> 1);
    else j = wrap ? i - (Lmu - 1) * smu : i + smu;
    switch (mu) {
      case 0: force_trace<0>(fp, v, i, j, p, threadIdx.z, blockDim.z, T); break;
      case 1: force_trace<1>(fp, v, i, j, p, threadIdx.z, blockDim.z, T); break;
      case 2: force_trace<2>(fp, v, i, j, p, threadIdx.z, blockDim.z, T); break;
      default: force_trace<3>(fp, v, i, j, p, threadIdx.z, blockDim.z, T); break;
    }
  }
  if (blockDim.z > 1) {
    extern __shared__ double tsm[];  // [group][18][mu][tx]
    const int bx = blockDim.x * 4, col = threadIdx.x + blockDim.x * mu;
    if (active && threadIdx.z > 0) {
      double *d = tsm + (size_t)threadIdx.z * 18 * bx + col;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        d[(2 * k) * bx] = T[k / 3][k % 3].re;
        d[(2 * k + 1) * bx] = T[k / 3][k % 3].im;
      }
    }
    __syncthreads();
    if (active && threadIdx.z == 0)
      for (int g = 1; g < (int)blockDim.z; g++) {
        const double *d = tsm + (size_t)g * 18 * bx + col;
#pragma unroll
        for (int k = 0; k < 9; k++) {
          T[k / 3][k % 3].re += d[(2 * k) * bx];
          T[k / 3][k % 3].im += d[(2 * k + 1) * bx];
        }
      }
  }
  if (active && threadIdx.z == 0) {
    // F = U T  (Matrix::DotMEqual)
    su3<double> u;
    LinkIO<PREC_DOUBLE, 18>::load(v.U, p, mu, i, u);
    cplx<double> F[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const cplx<double> m = u.m[a][k], n = T[k][b];
          re = fma(m.re, n.re, fma(-m.im, n.im, re));
          im = fma(m.re, n.im, fma(m.im, n.re, im));
        }
        F[a][b] = {re, im};
      }
    // 1/2 (F - F^dag), traceless, times coeff (Matrix::TrLessAntiHermMatrix)
    const double bcmu = mu == 0 ? fp.bc[0] : mu == 1 ? fp.bc[1] : mu == 2 ? fp.bc[2] : fp.bc[3];
    const double coeff = (wrap && bcmu < 0) ? -fp.scale : fp.scale;
    cplx<double> A[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) A[a][b] = {0.5 * (F[a][b].re - F[b][a].re), 0.5 * (F[a][b].im + F[b][a].im)};
    const double tri = (A[0][0].im + A[1][1].im + A[2][2].im) * (1.0 / 3.0);
#pragma unroll
    for (int a = 0; a < 3; a++) A[a][a].im -= tri;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) {
        A[a][b].re *= coeff;
        A[a][b].im *= coeff;
      }
    double tr = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) tr += A[a][b].re * A[b][a].re - A[a][b].im * A[b][a].im;
    const long lex = x + (long)fp.L[0] * (y + (long)fp.L[1] * (z + (long)fp.L[2] * t));
    double2 *m = reinterpret_cast<double2 *>(v.mom + 18 * (4 * lex + mu));
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 o = m[k];
      o.x += A[k / 3][k % 3].re;
      o.y += A[k / 3][k % 3].im;
      m[k] = o;
    }
    const double n = -2.0 * tr;
    red[0] = sqrt(fmax(n, 0.0));
    red[1] = n;
    red[2] = red[0];
  }
  // per-block L1, L2 sums and Linf max, in a fixed order
  __shared__ double sm[FORCE_TPB / 32][3];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = tid & 31, warp = tid >> 5, nwarp = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    red[0] += __shfl_down_sync(0xffffffffu, red[0], o);
    red[1] += __shfl_down_sync(0xffffffffu, red[1], o);
    red[2] = fmax(red[2], __shfl_down_sync(0xffffffffu, red[2], o));
  }
  if (lane == 0) {
    sm[warp][0] = red[0];
    sm[warp][1] = red[1];
    sm[warp][2] = red[2];
  }
  __syncthreads();
  if (tid == 0) {
    double s0 = 0.0, s1 = 0.0, mx = 0.0;
    for (int k = 0; k < nwarp; k++) {
      s0 += sm[k][0];
      s1 += sm[k][1];
      mx = fmax(mx, sm[k][2]);
    }
    double *out = partials + 3 * (blockIdx.x + (size_t)gridDim.x * blockIdx.y);
    out[0] = s0;
    out[1] = s1;
    out[2] = mx;
  }
}

// one block: the partials in block order -> out[0..2] = L1, L2, Linf sums
__global__ void __launch_bounds__(1024) force_finalize_kernel(const double *partials, unsigned nblk, double *out) {
  __shared__ double sm[32][3];
  double a = 0.0, b = 0.0, c = 0.0;
  for (unsigned k = threadIdx.x; k < nblk; k += blockDim.x) {
    a += partials[3 * k];
    b += partials[3 * k + 1];
    c = fmax(c, partials[3 * k + 2]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
    c = fmax(c, __shfl_down_sync(0xffffffffu, c, o));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sm[warp][0] = a;
    sm[warp][1] = b;
    sm[warp][2] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0, mx = 0.0;
    for (int k = 0; k < (int)(blockDim.x + 31) / 32; k++) {
      s0 += sm[k][0];
      s1 += sm[k][1];
      mx = fmax(mx, sm[k][2]);
    }
    out[0] = s0;
    out[1] = s1;
    out[2] = mx;
  }
}

// per-link Matrix::norm() = -2 Re tr M^2 of a CANONICAL Matrix field: block
// partials of sum |M|, sum |M|^2 and max |M| (as fforce_kernel writes them)
__global__ void __launch_bounds__(256) mom_norm_kernel(const double *mom, long nlink, double *partials) {
  const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double red[3] = {0.0, 0.0, 0.0};
  if (l < nlink) {
    const double2 *m = reinterpret_cast<const double2 *>(mom + 18 * l);
    cplx<double> A[3][3];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const double2 q = m[k];
      A[k / 3][k % 3] = {q.x, q.y};
    }
    double tr = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) tr += A[a][b].re * A[b][a].re - A[a][b].im * A[b][a].im;
    const double n = -2.0 * tr;
    red[0] = sqrt(fmax(n, 0.0));
    red[1] = n;
    red[2] = red[0];
  }
  __shared__ double sm[8][3];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    red[0] += __shfl_down_sync(0xffffffffu, red[0], o);
    red[1] += __shfl_down_sync(0xffffffffu, red[1], o);
    red[2] = fmax(red[2], __shfl_down_sync(0xffffffffu, red[2], o));
  }
  if (lane == 0) {
    sm[warp][0] = red[0];
    sm[warp][1] = red[1];
    sm[warp][2] = red[2];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0, mx = 0.0;
    for (int k = 0; k < (int)(blockDim.x + 31) / 32; k++) {
      s0 += sm[k][0];
      s1 += sm[k][1];
      mx = fmax(mx, sm[k][2]);
    }
    partials[3 * blockIdx.x] = s0;
    partials[3 * blockIdx.x + 1] = s1;
    partials[3 * blockIdx.x + 2] = mx;
  }
}

__global__ void add_kernel(double *y, const double *x, long n) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) y[k] += x[k];
}

// the reduced sums of the last reduction -> the reference's ForceArg
void force_arg_of(Lattice &L, const double *res, double out[3]) {
  double h[3];
  CPSGPU_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, L.stream));
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
  const double links = 4.0 * 2.0 * (double)L.vh;
  out[0] = h[0] / links;
  out[1] = std::sqrt(h[1] / links);
  out[2] = h[2];
}

}  // namespace

void calc_hmd_force_vecs(const Dirac &D, ForceVecs &fv, const SpinorView &chi) {
  if (D.kind == KIND_MOBIUS && D.cplx) throw Error(-1, "the fermion force is built for real Mobius b, c");
  const Lattice &L = *D.lat;
  for (Field *f : {&fv.v1o, &fv.v1e, &fv.v2o, &fv.v2e, &fv.t1, &fv.t2})
    if (f->data.ptr == nullptr || f->vh != L.vh || f->ls != D.ls) f->create(PREC_DOUBLE, L.vh, D.ls, 1);
  if (D.kind == KIND_MOBIUS) {
    // Fmobius::EvolveMomFforce(mom, frm, mass, step) (f_mobius.C:847-887):
    // phi1 = MatPc frm, phi2 = frm, then DiracOpMobius::CalcHmdForceVecs(v1,
    // v2, phi1, phi2) for SYM2 (d_op_mobius.C:1015-1100):
    //   phi2 <- M5^-1 phi2;  v1 = (M5^-dag Dslash4^dag phi1, phi1);
    //   v2 = (Booee M5^-1 Dslash4 phi2, Booee phi2)   [even half, odd half]
    // (the reference overwrites the caller's frm with M5^-1 frm; t2 holds it here)
    op_matpc(D, PREC_DOUBLE, fv.v1o.view(), chi, 0, fv.w, nullptr, 0, 0);  // phi1
    op_mobius_m5inv(D, PREC_DOUBLE, fv.t2.view(), chi, 0);                 // phi2
    op_mobius_dslash4(D, PREC_DOUBLE, fv.t1.view(), fv.t2.view(), 1, 0, fv.w);
    op_mobius_m5inv(D, PREC_DOUBLE, fv.v1e.view(), fv.t1.view(), 0);
    launch_mix(D, PREC_DOUBLE, D.mixB.as<double>(), fv.v1e.view(), fv.v2e.view());
    launch_mix(D, PREC_DOUBLE, D.mixB.as<double>(), fv.t2.view(), fv.v2o.view());
    op_mobius_dslash4(D, PREC_DOUBLE, fv.t1.view(), fv.v1o.view(), 1, 1, fv.w);
    op_mobius_m5inv(D, PREC_DOUBLE, fv.v1e.view(), fv.t1.view(), 1);
    return;
  }
  // f_out = (chi, D chi)
  CPSGPU_CUDA(cudaMemcpyAsync(fv.v1o.data.ptr, chi.data, fv.v1o.data.bytes, cudaMemcpyDeviceToDevice, L.stream));
  op_dslash(D, PREC_DOUBLE, fv.v1e.view(), fv.v1o.view(), 1, 0);
  // f_in = (-kappa^2 MatPc chi, D^dag of it)
  op_matpc(D, PREC_DOUBLE, fv.v2o.view(), fv.v1o.view(), 0, fv.w, nullptr, 0, 0);
  launch_scale(L.stream, -D.kappa * D.kappa, fv.v2o.view());
  op_dslash(D, PREC_DOUBLE, fv.v2e.view(), fv.v2o.view(), 1, 1);
}

void fforce_update(const Dirac &D, const ForceVecs &fv, double *mom, double dt, double out[3]) {
  const bool mob = D.kind == KIND_MOBIUS;
  Lattice &L = *D.lat;
  ForceParams fp;
  for (int k = 0; k < 4; k++) {
    fp.L[k] = L.L[k];
    fp.bc[k] = L.bc[k];
  }
  fp.hx = L.L[0] / 2;
  fp.vh = L.vh;
  fp.ls = D.ls;
  // Fwilson / FdwfBase: coeff = -2 dt.  Fmobius: FforceWilsonType with
  // coef = -step adds -coef TrLessAntiHerm(U T) with the roles of v1 and v2
  // exchanged in T (fforce_wilson_type.C do_site_force)
  fp.scale = mob ? dt : -2.0 * dt;
  fp.mobius = mob ? 1 : 0;
  ForceViews v;
  v.v1o = (mob ? fv.v2o : fv.v1o).view();
  v.v1e = (mob ? fv.v2e : fv.v1e).view();
  v.v2o = (mob ? fv.v1o : fv.v2o).view();
  v.v2e = (mob ? fv.v1e : fv.v2e).view();
  v.U.data = L.gD18.ptr;
  v.U.vh = L.vh;
  v.mom = mom;
  // one slice group: each warp then has a single mu (no divergence in the
  // projections) and the four directions of a site share L1
  const int sg = 1;
  const dim3 block(FORCE_TPB / (4 * sg), 4, sg);
  const dim3 grid(2 * (unsigned)((L.vh + block.x - 1) / block.x));
  const size_t smem = sg > 1 ? (size_t)sg * 18 * 4 * block.x * sizeof(double) : 0;
  const unsigned nblk = grid.x * grid.y;
  L.partials.ensure((size_t)nblk * 3 * sizeof(double) + 3 * sizeof(double));
  double *part = L.partials.as<double>();
  double *res = part + (size_t)nblk * 3;
  fforce_kernel<<<grid, block, smem, L.stream>>>(fp, v, part);
  CPSGPU_CUDA(cudaGetLastError());
  force_finalize_kernel<<<1, 1024, 0, L.stream>>>(part, nblk, res);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter() += 2;
  if (out) force_arg_of(L, res, out);
}

void mom_norms(Lattice &L, const double *mom, double out[3]) {
  const long nlink = 4 * 2 * L.vh;
  const unsigned nblk = (unsigned)((nlink + 255) / 256);
  L.partials.ensure((size_t)nblk * 3 * sizeof(double) + 3 * sizeof(double));
  double *part = L.partials.as<double>();
  double *res = part + (size_t)nblk * 3;
  mom_norm_kernel<<<nblk, 256, 0, L.stream>>>(mom, nlink, part);
  CPSGPU_CUDA(cudaGetLastError());
  force_finalize_kernel<<<1, 1024, 0, L.stream>>>(part, nblk, res);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter() += 2;
  force_arg_of(L, res, out);
}

void mom_add(Lattice &L, double *mom, const double *x) {
  const long n = 4 * 2 * L.vh * 18;
  add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, L.stream>>>(mom, x, n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

// algorithmic bytes of one force-kernel launch: v1, v2 read once (both
// parities, all slices), the FP64 links read once, mom read and written
double fforce_bytes(const Dirac &D) {
  const double v4 = 2.0 * (double)D.lat->vh;
  return 2.0 * 2.0 * (double)D.lat->vh * D.ls * 192.0 + v4 * 4 * 144.0 + 2.0 * v4 * 4 * 144.0;
}

}  // namespace cpsgpu
