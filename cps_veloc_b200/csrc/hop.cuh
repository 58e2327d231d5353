// The even-odd hopping kernel shared by the Wilson, Shamir-DWF and Mobius
// operators, with fused epilogues.
//
// One thread computes one output site (checkerboard site i, slice s, rhs).
// A block is BX consecutive sites x BS slices, so the BS threads that share
// a site share its eight links through L1, and each warp's spinor and link
// loads are fully coalesced (see fields.cuh).  Neighbour indices are computed
// in-kernel from the site coordinates, with the lattice wrapped in every
// direction and the boundary sign bc[mu] applied to each wrapping hop.
//
// What the reference spreads over several passes is fused here:
//   * DWF: the 4D hop of every slice (dwf_dslash_4.C:68-154, slice s hops
//     from 4D parity (s+cb)%2) and the fifth-direction hop
//     (dwf_dslash_5_plus_omp.C:115-271) are one kernel;
//   * axpby + norm of MatPc (wilson_m.C:83-91, dwf_m.C:60, the |M p|^2 of
//     wilson_mdagm.C:124-137 / dwf_mdagm.C:49-55) is the AXPY epilogue;
//   * the CG updates after MatPcDagMatPc (inv_cg.C:333-349) are the CG
//     epilogue: the operator output is never written to memory;
//   * Mobius: the s-local chains M5^-1 / b,c mixing / kappa_b scaling that
//     sit between two hops (zmobius_m-sym2.h, zmobius_mdag-sym2.h) are one
//     dense Ls x Ls matrix per chirality applied in the MIX epilogue from
//     shared memory (a block then holds all Ls slices of its sites).
#pragma once
#include "fields.cuh"
#include "reduce.cuh"

namespace cpsgpu {

constexpr int MAX_LS = 32;

enum Epilogue {
  EP_STORE = 0,     // out = hop
  EP_AXPY = 1,      // out = x + coef[s] * hop                 (+ |out|^2, |x|^2)
  EP_MIX = 2,       // out = Mix hop
  EP_MIX_AXPY = 3,  // out = x + Mix hop                       (+ |out|^2, |x|^2)
  EP_CG = 4,        // q = x + coef[s] hop + shift p; r -= alpha q; sol += alpha p; |r|^2
  EP_MIX_CG = 5,    // q = x + Mix hop + shift p; as EP_CG
  EP_RES = 6,       // q = x + coef[s] hop + shift sol; r = b - q (stored in r's precision); |r|^2
  EP_MIX_RES = 7,   // q = x + Mix hop + shift sol; as EP_RES
};

__host__ __device__ constexpr bool ep_mix(int e) { return e == EP_MIX || e == EP_MIX_AXPY || e == EP_MIX_CG || e == EP_MIX_RES; }
__host__ __device__ constexpr bool ep_cg(int e) { return e == EP_CG || e == EP_MIX_CG; }
__host__ __device__ constexpr bool ep_res(int e) { return e == EP_RES || e == EP_MIX_RES; }
__host__ __device__ constexpr bool ep_axpy(int e) { return e == EP_AXPY || e == EP_MIX_AXPY; }

// Gating of a launch on the solver state.
enum Gate { GATE_NONE = 0, GATE_RUNNING = 1, GATE_RELIABLE = 2 };

struct HopParams {
  int L[4];
  int hx;           // L[0] / 2
  long vh;          // checkerboard volume
  int ls;
  double bc[4];     // boundary sign per direction
  int cb;           // input checkerboard (as the reference's cb argument)
  int dag;
  int dwf;          // 1: 5D even-odd (parity (s+cb)%2, fifth-dir hop)
  double h5;        // DWF fifth-dir weight 2/a5
  double h5wall;    // DWF wall weight -2 m_f / a5
  double coef[MAX_LS];  // per-slice coefficient of the AXPY/CG/RES epilogues
  const double *mix;    // [2][ls][ls] row-major, upper then lower chirality
  int norm;         // AXPY: accumulate reductions
  int red_op;       // ReduceOp for the finalize
  int gate;         // Gate
};

struct HopViews {
  GaugeView U;
  SpinorView in, out, x;  // hop input, output, axpby source
  SpinorView r, sol, p;   // CG / RES epilogue fields
  SpinorView b;           // RES: right-hand side (double)
};

__device__ __forceinline__ long site_cb(int x, int hx, int y, int z, int t, const int *L) {
  return (long)(x >> 1) + (long)hx * (y + (long)L[1] * (z + (long)L[2] * t));
}

// acc = sum over mu of the forward and backward hops into output site i,
// slice sl, whose 4D parity is pout (input parity pin = 1 - pout).
template <int P, int RECON>
__device__ __forceinline__ void hop_site(const HopParams &hp, const HopViews &v, long i, long sl,
                                         int pout, typename PrecTraits<P>::real *acc) {
  using R = typename PrecTraits<P>::real;
  const int pin = 1 - pout;
  const int hx = hp.hx;
  const long xh = i % hx;
  long rem = i / hx;
  const int y = (int)(rem % hp.L[1]);
  rem /= hp.L[1];
  const int z = (int)(rem % hp.L[2]);
  const int t = (int)(rem / hp.L[2]);
  const int x = 2 * (int)xh + ((y + z + t + pout) & 1);
  const int c[4] = {x, y, z, t};
  const R sdag = hp.dag ? R(-1) : R(1);
#pragma unroll
  for (int k = 0; k < 24; k++) acc[k] = R(0);
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    // forward: U_mu(x) (1 - sdag g_mu) psi(x + mu)
    {
      int cn[4] = {c[0], c[1], c[2], c[3]};
      bool wrap = (c[mu] == hp.L[mu] - 1);
      cn[mu] = wrap ? 0 : c[mu] + 1;
      long j = site_cb(cn[0], hx, cn[1], cn[2], cn[3], hp.L);
      R psi[24];
      SpinorIO<P>::load(v.in, sl, j, psi);
      su3<R> u;
      LinkIO<P, RECON>::load(v.U, pout, mu, i, u);
      half_spinor<R> h = project(psi, mu, -sdag);
      half_spinor<R> g = link_mul(u, h, false);
      R w = wrap ? R(hp.bc[mu]) : R(1);
      reconstruct_acc(acc, g, mu, -sdag, w);
    }
    // backward: U_mu(x - mu)^dagger (1 + sdag g_mu) psi(x - mu)
    {
      int cn[4] = {c[0], c[1], c[2], c[3]};
      bool wrap = (c[mu] == 0);
      cn[mu] = wrap ? hp.L[mu] - 1 : c[mu] - 1;
      long j = site_cb(cn[0], hx, cn[1], cn[2], cn[3], hp.L);
      R psi[24];
      SpinorIO<P>::load(v.in, sl, j, psi);
      su3<R> u;
      LinkIO<P, RECON>::load(v.U, pin, mu, j, u);
      half_spinor<R> h = project(psi, mu, sdag);
      half_spinor<R> g = link_mul(u, h, true);
      R w = wrap ? R(hp.bc[mu]) : R(1);
      reconstruct_acc(acc, g, mu, sdag, w);
    }
  }
}

// Fifth-direction hop of the Shamir DWF operator, accumulated into acc.
template <int P>
__device__ __forceinline__ void hop5_dwf(const HopParams &hp, const HopViews &v, long i, int s, long rhs,
                                         typename PrecTraits<P>::real *acc) {
  using R = typename PrecTraits<P>::real;
  const int ls = hp.ls;
  // the half fed from s-1 is the upper one for D, the lower one for D^dagger
  const int hb = hp.dag ? 1 : 0, ha = 1 - hb;
  const int sb = (s == 0) ? ls - 1 : s - 1, sa = (s == ls - 1) ? 0 : s + 1;
  const R wb = R((s == 0) ? hp.h5wall : hp.h5), wa = R((s == ls - 1) ? hp.h5wall : hp.h5);
  R q[12];
  SpinorIO<P>::load_half(v.in, rhs * ls + sb, i, hb, q);
#pragma unroll
  for (int k = 0; k < 12; k++) acc[12 * hb + k] += wb * q[k];
  SpinorIO<P>::load_half(v.in, rhs * ls + sa, i, ha, q);
#pragma unroll
  for (int k = 0; k < 12; k++) acc[12 * ha + k] += wa * q[k];
}

template <typename R>
__device__ __forceinline__ double norm2_24(const R *a) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 24; k++) s += double(a[k]) * double(a[k]);
  return s;
}

// PR: precision of r and p (CG/RES epilogues); PX: precision of sol.
template <int P, int RECON, int EP, int PR, int PX>
__global__ void __launch_bounds__(256) hop_kernel(const HopParams hp, const HopViews v, SolverScalars *st,
                                                  double *partials) {
  using R = typename PrecTraits<P>::real;
  const long rhs = blockIdx.z;
  if (hp.gate == GATE_RUNNING && st[rhs].done) return;
  if (hp.gate == GATE_RELIABLE && (st[rhs].done || !st[rhs].reliable)) return;

  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y * blockDim.y + threadIdx.y;
  const bool active = (i < hp.vh) && (s < hp.ls);
  const long sl = rhs * hp.ls + s;
  const int pin = hp.dwf ? ((s + hp.cb) & 1) : hp.cb;
  const int pout = 1 - pin;

  R acc[24];
  if (active) {
    hop_site<P, RECON>(hp, v, i, sl, pout, acc);
    if (hp.dwf) hop5_dwf<P>(hp, v, i, s, rhs, acc);
  }

  if constexpr (ep_mix(EP)) {
    // all Ls slices of this block's sites: out(s) = sum_t Mix_chi[s][t] acc(t)
    extern __shared__ unsigned char smraw[];
    R *sm = reinterpret_cast<R *>(smraw);  // [ls][BX][24]
    double *mx = reinterpret_cast<double *>(sm + (size_t)hp.ls * blockDim.x * 24);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    for (int k = tid; k < 2 * hp.ls * hp.ls; k += blockDim.x * blockDim.y) mx[k] = hp.mix[k];
    if (s < hp.ls) {
      R *mine = sm + ((size_t)s * blockDim.x + threadIdx.x) * 24;
#pragma unroll
      for (int k = 0; k < 24; k++) mine[k] = active ? acc[k] : R(0);
    }
    __syncthreads();
    if (active) {
#pragma unroll
      for (int k = 0; k < 24; k++) acc[k] = R(0);
      for (int t2 = 0; t2 < hp.ls; t2++) {
        const R mu_ = R(mx[s * hp.ls + t2]);
        const R md_ = R(mx[hp.ls * hp.ls + s * hp.ls + t2]);
        const R *src = sm + ((size_t)t2 * blockDim.x + threadIdx.x) * 24;
#pragma unroll
        for (int k = 0; k < 12; k++) acc[k] += mu_ * src[k];
#pragma unroll
        for (int k = 12; k < 24; k++) acc[k] += md_ * src[k];
      }
    }
  }

  if constexpr (EP == EP_STORE || EP == EP_MIX) {
    if (active) SpinorIO<P>::store(v.out, sl, i, acc);
  } else if constexpr (ep_axpy(EP)) {
    double red[2] = {0.0, 0.0};
    if (active) {
      R xv[24];
      SpinorIO<P>::load(v.x, sl, i, xv);
      const R cf = ep_mix(EP) ? R(1) : R(hp.coef[s]);
#pragma unroll
      for (int k = 0; k < 24; k++) acc[k] = xv[k] + cf * acc[k];
      SpinorIO<P>::store(v.out, sl, i, acc);
      if (hp.norm) {
        red[0] = norm2_24(acc);
        red[1] = norm2_24(xv);
      }
    }
    if (hp.norm) grid_reduce_finalize<2>(red, partials, st, hp.red_op);
  } else if constexpr (ep_cg(EP)) {
    using RR = typename PrecTraits<PR>::real;
    using RX = typename PrecTraits<PX>::real;
    double red[1] = {0.0};
    if (active) {
      R xv[24];
      SpinorIO<P>::load(v.x, sl, i, xv);
      RR pv[24], rv[24];
      RX sv[24];
      SpinorIO<PR>::load(v.p, sl, i, pv);
      SpinorIO<PR>::load(v.r, sl, i, rv);
      if (v.sol.data) SpinorIO<PX>::load(v.sol, sl, i, sv);
      else
#pragma unroll
        for (int k = 0; k < 24; k++) sv[k] = RX(0);
      const double alpha = st[rhs].alpha;
      const R cf = ep_mix(EP) ? R(1) : R(hp.coef[s]);
      const R sh = R(st[rhs].shift);
      const RR a = RR(alpha);
      const RX ax = RX(alpha);
#pragma unroll
      for (int k = 0; k < 24; k++) {
        R q = xv[k] + cf * acc[k] + sh * R(pv[k]);
        rv[k] = rv[k] - a * RR(q);
        sv[k] = sv[k] + ax * RX(pv[k]);
      }
      SpinorIO<PR>::store(v.r, sl, i, rv);
      // the multishift solver updates its solutions itself (no sol view)
      if (v.sol.data) SpinorIO<PX>::store(v.sol, sl, i, sv);
      red[0] = norm2_24(rv);
    }
    grid_reduce_finalize<1>(red, partials, st, hp.red_op);
  } else if constexpr (ep_res(EP)) {
    double red[1] = {0.0};
    if (active) {
      R xv[24], bv[24], sv[24];
      SpinorIO<P>::load(v.x, sl, i, xv);
      SpinorIO<P>::load(v.b, sl, i, bv);
      SpinorIO<P>::load(v.sol, sl, i, sv);
      const R cf = ep_mix(EP) ? R(1) : R(hp.coef[s]);
      const R sh = R(st[rhs].shift);
#pragma unroll
      for (int k = 0; k < 24; k++) acc[k] = bv[k] - (xv[k] + cf * acc[k] + sh * sv[k]);
      red[0] = norm2_24(acc);
      using RR = typename PrecTraits<PR>::real;
      RR rv[24];
#pragma unroll
      for (int k = 0; k < 24; k++) rv[k] = RR(acc[k]);
      SpinorIO<PR>::store(v.r, sl, i, rv);
    }
    grid_reduce_finalize<1>(red, partials, st, hp.red_op);
  }
}

}  // namespace cpsgpu
