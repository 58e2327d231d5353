// The unpreconditioned operators on both checkerboards and the shifted
// Mobius MatPcDagMatPc.
//
//   Mat     Wilson, DWF (d_op_wilson.C:362-392, d_op_dwf.C:541-583):
//             out_0 = in_0 - kappa D(in_1, CHKB_EVEN)
//             out_1 = in_1 - kappa D(in_0, CHKB_ODD)
//           Mobius (d_op_mobius.C:735-795):
//             out_0 = (1 + a5inv K D5) in_0 - kappa_b Dslash_4(in_1, CHKB_ODD)
//             out_1 = (1 + a5inv K D5) in_1 - kappa_b Dslash_4(in_0, CHKB_EVEN)
//   MatDag  the same with D^dagger (Wilson, DWF: d_op_wilson.C:394-424,
//           d_op_dwf.C:585-627; the reference's Mobius MatDag stops with an
//           error, d_op_mobius.C:879, and is refused here)
//   MatHerm gamma_5 Mat (Wilson, d_op_wilson.C:426-443); gamma_5 R Mat with
//           R the reflection s -> Ls-1-s as FdwfBase::Freflex stores it
//           (f_dwf_base.C:1693-1790: for even Ls slice s of one half comes
//           from the other half) (DWF, Mobius: d_op_dwf.C:629-660,
//           d_op_mobius.C:915-942)
//   MatPcDagMatPcShift (Mobius, d_op_mobius.C:235; zmobius_mdagm.C:79-135):
//           out = M^+ M in - 2 mu R g5 M in + mu^2 in, R g5 within the
//           checkerboard (ReflectAndMultGamma5, d_op_mobius.C:1401-1418)
//
// Half 0 / half 1 are the two checkerboards in the reference's full-vector
// order: [odd][even] for Wilson and DWF, [even][odd] for Mobius.  The hops
// are the fused hop kernel with its AXPY epilogue; the gamma_5 / reflection
// combinations are one streaming kernel.
#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

namespace {

// out(s, i) = a g5 x(r(s), i) + b y(s, i) + c z(s, i), r(s) = Ls-1-s when
// reflect, else s; y and z optional (null data).  One thread per 5D site.
template <int P>
__global__ void g5r_kernel(SpinorView out, SpinorView x, double a, int reflect, SpinorView y, double b,
                           SpinorView z, double c) {
  using R = typename PrecTraits<P>::real;
  const long n = x.vh * x.ls * x.nrhs;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const long sl = idx / x.vh, i = idx % x.vh;
  const long rhs = sl / x.ls, s = sl % x.ls;
  const long sr = rhs * x.ls + (reflect ? x.ls - 1 - s : s);
  R v[24], w[24];
  SpinorIO<P>::load(x, sr, i, v);
#pragma unroll
  for (int k = 0; k < 24; k++) v[k] = (k < 12 ? R(a) : R(-a)) * v[k];
  if (y.data) {
    SpinorIO<P>::load(y, sl, i, w);
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] += R(b) * w[k];
  }
  if (z.data) {
    SpinorIO<P>::load(z, sl, i, w);
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] += R(c) * w[k];
  }
  SpinorIO<P>::store(out, sl, i, v);
}

void launch_g5r(cudaStream_t st, int prec, const SpinorView &out, const SpinorView &x, double a, int reflect,
                const SpinorView &y = SpinorView(), double b = 0.0, const SpinorView &z = SpinorView(),
                double c = 0.0) {
  const long n = x.vh * x.ls * x.nrhs;
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (prec == PREC_DOUBLE) g5r_kernel<PREC_DOUBLE><<<grid, 256, 0, st>>>(out, x, a, reflect, y, b, z, c);
  else if (prec == PREC_SINGLE) g5r_kernel<PREC_SINGLE><<<grid, 256, 0, st>>>(out, x, a, reflect, y, b, z, c);
  else g5r_kernel<PREC_HALF><<<grid, 256, 0, st>>>(out, x, a, reflect, y, b, z, c);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

SpinorView none() { return SpinorView(); }

// out = x + coef hop(in) (the AXPY epilogue), hop reading checkerboard cb
void hop_axpy(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, const SpinorView &x, int cb,
              int dag, double coef) {
  HopLaunch L;
  L.prec = prec;
  L.ep = EP_AXPY;
  L.cb = cb;
  L.dag = dag;
  L.coef.assign(D.ls, coef);
  launch_hop(D, L, in, out, x, none(), none(), none(), none(), nullptr);
}

}  // namespace

void op_mat(const Dirac &D, int prec, const SpinorView &out0, const SpinorView &out1, const SpinorView &in0,
            const SpinorView &in1, int dag, OpWork &w) {
  if (D.kind != KIND_MOBIUS) {
    hop_axpy(D, prec, out0, in1, in0, 0, dag, -D.kappa);
    hop_axpy(D, prec, out1, in0, in1, 1, dag, -D.kappa);
    return;
  }
  if (dag) throw Error(-1, "Mobius MatDag: the reference's DiracOpMobius::MatDag stops with an error");
  if (D.cplx) throw Error(-1, "Mobius Mat: real b, c only (DiracOpMobius)");
  const Lattice &lat = *D.lat;
  ensure_field(w.t0, prec, lat.vh, D.ls, in0.nrhs);
  const SpinorView t = w.t0.view();
  // out_0 = M5a in_0 - kappa_b W(B in_1) with W reading the odd half
  launch_mix(D, prec, D.mixB.as<double>(), in1, t);
  launch_mix(D, prec, D.mixM5a.as<double>(), in0, out0);
  hop_axpy(D, prec, out0, t, out0, 1, 0, -D.kappa);
  launch_mix(D, prec, D.mixB.as<double>(), in0, t);
  launch_mix(D, prec, D.mixM5a.as<double>(), in1, out1);
  hop_axpy(D, prec, out1, t, out1, 0, 0, -D.kappa);
}

void op_mat_herm(const Dirac &D, int prec, const SpinorView &out0, const SpinorView &out1, const SpinorView &in0,
                 const SpinorView &in1, OpWork &w) {
  const Lattice &lat = *D.lat;
  ensure_field(w.t1, prec, lat.vh, D.ls, in0.nrhs);
  ensure_field(w.t2, prec, lat.vh, D.ls, in0.nrhs);
  op_mat(D, prec, w.t1.view(), w.t2.view(), in0, in1, 0, w);
  if (D.kind == KIND_WILSON) {
    launch_g5r(lat.stream, prec, out0, w.t1.view(), 1.0, 0);
    launch_g5r(lat.stream, prec, out1, w.t2.view(), 1.0, 0);
    return;
  }
  // Freflex: even Ls swaps the halves, odd Ls keeps them
  const bool swap = (D.ls % 2) == 0;
  launch_g5r(lat.stream, prec, out0, swap ? w.t2.view() : w.t1.view(), 1.0, 1);
  launch_g5r(lat.stream, prec, out1, swap ? w.t1.view() : w.t2.view(), 1.0, 1);
}

void op_mdagm_shift(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, double mu, OpWork &w,
                    SolverScalars *st) {
  if (D.kind != KIND_MOBIUS) throw Error(-1, "MatPcDagMatPcShift: Mobius operators (DiracOpMobius)");
  ensure_field(w.t2, prec, D.lat->vh, D.ls, in.nrhs);
  op_matpc(D, prec, w.t2.view(), in, 0, w, st, st ? 1 : 0, RED_STORE);
  op_matpc(D, prec, out, w.t2.view(), 1, w, st, 0, 0);
  // out += -2 mu R g5 (M in) + mu^2 in
  launch_g5r(D.lat->stream, prec, out, w.t2.view(), -2.0 * mu, 1, out, 1.0, in, mu * mu);
}

}  // namespace cpsgpu
