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
#include <type_traits>

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

// n / d for 0 <= n < 2^31 by multiply-high (Granlund and Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994): with
// s = ceil(log2 d) and m = floor(2^32 (2^s - d) / d) + 1, q = (mulhi(n,m) + n) >> s.
struct FastDiv {
  unsigned m;
  int s;
  int d;
  __host__ void init(int d_) {
    d = d_;
    s = 0;
    while ((1u << s) < (unsigned)d) s++;
    unsigned long long num = ((1ull << 32) * ((1ull << s) - (unsigned)d));
    m = (unsigned)(num / (unsigned)d + 1);
    if (d == 1) { m = 0; s = 0; }
  }
  __device__ __forceinline__ int div(int n) const {
    return (int)((__umulhi((unsigned)n, m) + (unsigned)n) >> s);
  }
};

enum HopSub { SUB_ALL = 0, SUB_INTERIOR = 1, SUB_BOUNDARY = 2 };

struct HopParams {
  int L[4];
  int hx;           // L[0] / 2
  long vh;          // checkerboard volume
  int ls;
  FastDiv dhx, dly, dlz;  // divisions by L[0]/2, L[1], L[2]
  int nsg;          // slice groups in the launch
  int rtile;        // right-hand sides per tile: consecutive blocks take the same sites of rtile solves
  int nrhs;         // right-hand sides in the launch
  double bc[4];     // boundary sign per direction
  int cb;           // input checkerboard (as the reference's cb argument)
  int dag;
  int dwf;          // 1: 5D even-odd (parity (s+cb)%2, fifth-dir hop)
  double h5;        // DWF fifth-dir weight 2/a5
  double h5wall;    // DWF wall weight -2 m_f / a5
  double coef[MAX_LS];  // per-slice coefficient of the AXPY/CG/RES epilogues
  const double *mix;    // [2][ls][ls] row-major, upper then lower chirality ([..][re, im] if mix_cplx)
  int mix_cplx;         // complex mixing matrices (zMobius)
  int norm;         // AXPY: accumulate reductions
  int red_op;       // ReduceOp for the finalize
  int gate;         // Gate
  // t-slab domain decomposition (the HALO kernels): face = sites of one
  // t-slice of a checkerboard;
  // tb_fwd / tb_bwd: this slab's forward / backward t end is the lattice's
  // own boundary, where bc[3] applies (both 1 without decomposition)
  int face, tb_fwd, tb_bwd;
  // DWF slice groups of one 4D parity: group g holds slices
  // (g / 2) * 2 BS + (g % 2) + 2 k, so the BS threads of a site read the same
  // eight links (the parity of slice s alternates with s)
  int spar;
  // HopSub: SUB_ALL every site; SUB_INTERIOR the t-slices 1 .. L[3]-2 of a
  // slab (their hops need no halo); SUB_BOUNDARY its first and last
  // t-slices, subn site blocks each
  int sub, subn;
  int i0, iend, jump;  // first site, end of the (first) site range, the boundary subset's jump
};

struct HopViews {
  GaugeView U;
  SpinorView in, out, x;  // hop input, output, axpby source
  SpinorView r, sol, p;   // CG / RES epilogue fields
  SpinorView b;           // RES: right-hand side (double)
  // t halos, [slice][12 reals][face] in the hop's precision: hf from the
  // next slab, (1 - sdag g_t) psi of its first t-slice; hb from the previous
  // slab, U_t^dagger (1 + sdag g_t) psi of its last t-slice
  const void *hf, *hb;
};

// one half spinor of a t halo ([slice][12 reals][face])
template <typename R>
__device__ __forceinline__ half_spinor<R> load_halo(const void *p, int face, long sl, int f) {
  const R *q = reinterpret_cast<const R *>(p) + (size_t)sl * 12 * face + f;
  half_spinor<R> r;
#pragma unroll
  for (int sp = 0; sp < 2; sp++)
#pragma unroll
    for (int col = 0; col < 3; col++) {
      const int k = 2 * (col + 3 * sp);
      r.h[sp][col] = {__ldg(q + (size_t)k * face), __ldg(q + (size_t)(k + 1) * face)};
    }
  return r;
}

// acc = sum over mu of the forward and backward hops into output site i,
// slice sl, whose 4D parity is pout (input parity pin = 1 - pout).
// All site arithmetic is 32-bit; the coordinates come from three
// multiply-high divisions and each neighbour index from i by a stride.
// HALO: the t hops across a slab's ends read the halos (t-slab decomposition);
// a separate instantiation, so the undecomposed kernels carry none of it.
template <int P, int RECON, bool DAG, bool HALO>
__device__ __forceinline__ void hop_site(const HopParams &hp, const HopViews &v, int i, long sl,
                                         int pout, typename PrecTraits<P>::real *acc) {
  using R = typename PrecTraits<P>::real;
  const int pin = 1 - pout;
  const int hx = hp.hx, Ly = hp.L[1], Lz = hp.L[2];
  const int q1 = hp.dhx.div(i);
  const int xh = i - q1 * hx;
  const int q2 = hp.dly.div(q1);
  const int y = q1 - q2 * Ly;
  const int t = hp.dlz.div(q2);
  const int z = q2 - t * Lz;
  const int x = 2 * xh + ((y + z + t + pout) & 1);
  const int c[4] = {x, y, z, t};
  const int stride[4] = {0, hx, hx * Ly, hx * Ly * Lz};
  const Slice<P> in(v.in, sl);
  // sdag is a compile-time +-1, so every (1 -+ gamma) sign folds into adds
  constexpr R sdag = DAG ? R(-1) : R(1);
  HopAcc<R> A;
  A.zero();
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    // forward: U_mu(x) (1 - sdag g_mu) psi(x + mu)
    {
      const bool wrap = (c[mu] == hp.L[mu] - 1);
      int j;
      if (mu == 0) j = i - xh + ((wrap ? 0 : x + 1) >> 1);
      else j = wrap ? i - (hp.L[mu] - 1) * stride[mu] : i + stride[mu];
      if (HALO && mu == 3 && wrap) {
        // x + t lives on the next slab, which sent its projected half spinor
        su3<R> u;
        LinkIO<P, RECON>::load(v.U, pout, mu, i, u);
        A.hop(u, load_halo<R>(v.hf, hp.face, sl, j), false, mu, -sdag, (hp.tb_fwd && hp.bc[mu] < 0) ? R(-1) : R(1));
      } else {
        R psi[24], sc;
        in.load_raw(j, psi, sc);
        su3<R> u;
        LinkIO<P, RECON>::load(v.U, pout, mu, i, u);
        // the storage scale and the boundary sign ride on the accumulating FMAs
        A.hop(u, project(psi, mu, -sdag), false, mu, -sdag,
              (wrap && hp.bc[mu] < 0 && (!HALO || mu != 3 || hp.tb_fwd)) ? -sc : sc);
      }
    }
    // backward: U_mu(x - mu)^dagger (1 + sdag g_mu) psi(x - mu)
    {
      const bool wrap = (c[mu] == 0);
      int j;
      if (mu == 0) j = i - xh + ((wrap ? hp.L[0] - 1 : x - 1) >> 1);
      else j = wrap ? i + (hp.L[mu] - 1) * stride[mu] : i - stride[mu];
      if (HALO && mu == 3 && wrap) {
        // x - t and its link live on the previous slab, which sent U^dagger (1 + sdag g_t) psi
        A.add(load_halo<R>(v.hb, hp.face, sl, i), mu, sdag, (hp.tb_bwd && hp.bc[mu] < 0) ? R(-1) : R(1));
      } else {
        R psi[24], sc;
        in.load_raw(j, psi, sc);
        su3<R> u;
        LinkIO<P, RECON>::load(v.U, pin, mu, j, u);
        A.hop(u, project(psi, mu, sdag), true, mu, sdag,
              (wrap && hp.bc[mu] < 0 && (!HALO || mu != 3 || hp.tb_bwd)) ? -sc : sc);
      }
    }
  }
  A.store(acc);
}

// hop_site for two slices of the same 4D parity at once (DWF): each link is
// loaded (and, for 12 reals, rebuilt) once and applied to both slices, and
// the neighbour indices and boundary signs are computed once.  No halos.
template <int P, int RECON, bool DAG>
__device__ __forceinline__ void hop_site2(const HopParams &hp, const HopViews &v, int i, long sl0, long sl1,
                                          int pout, typename PrecTraits<P>::real *acc0,
                                          typename PrecTraits<P>::real *acc1) {
  using R = typename PrecTraits<P>::real;
  const int pin = 1 - pout;
  const int hx = hp.hx, Ly = hp.L[1], Lz = hp.L[2];
  const int q1 = hp.dhx.div(i);
  const int xh = i - q1 * hx;
  const int q2 = hp.dly.div(q1);
  const int y = q1 - q2 * Ly;
  const int t = hp.dlz.div(q2);
  const int z = q2 - t * Lz;
  const int x = 2 * xh + ((y + z + t + pout) & 1);
  const int c[4] = {x, y, z, t};
  const int stride[4] = {0, hx, hx * Ly, hx * Ly * Lz};
  const Slice<P> in0(v.in, sl0), in1(v.in, sl1);
  constexpr R sdag = DAG ? R(-1) : R(1);
  HopAcc<R> A0, A1;
  A0.zero();
  A1.zero();
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    {
      const bool wrap = (c[mu] == hp.L[mu] - 1);
      int j;
      if (mu == 0) j = i - xh + ((wrap ? 0 : x + 1) >> 1);
      else j = wrap ? i - (hp.L[mu] - 1) * stride[mu] : i + stride[mu];
      const R sgn = (wrap && hp.bc[mu] < 0) ? R(-1) : R(1);
      R psi0[24], psi1[24], sc0, sc1;
      in0.load_raw(j, psi0, sc0);
      in1.load_raw(j, psi1, sc1);
      su3<R> u;
      LinkIO<P, RECON>::load(v.U, pout, mu, i, u);
      A0.hop(u, project(psi0, mu, -sdag), false, mu, -sdag, sgn * sc0);
      A1.hop(u, project(psi1, mu, -sdag), false, mu, -sdag, sgn * sc1);
    }
    {
      const bool wrap = (c[mu] == 0);
      int j;
      if (mu == 0) j = i - xh + ((wrap ? hp.L[0] - 1 : x - 1) >> 1);
      else j = wrap ? i + (hp.L[mu] - 1) * stride[mu] : i - stride[mu];
      const R sgn = (wrap && hp.bc[mu] < 0) ? R(-1) : R(1);
      R psi0[24], psi1[24], sc0, sc1;
      in0.load_raw(j, psi0, sc0);
      in1.load_raw(j, psi1, sc1);
      su3<R> u;
      LinkIO<P, RECON>::load(v.U, pin, mu, j, u);
      A0.hop(u, project(psi0, mu, sdag), true, mu, sdag, sgn * sc0);
      A1.hop(u, project(psi1, mu, sdag), true, mu, sdag, sgn * sc1);
    }
  }
  A0.store(acc0);
  A1.store(acc1);
}

// Fifth-direction hop of the Shamir DWF operator, accumulated into acc.
template <int P, bool DAG>
__device__ __forceinline__ void hop5_dwf(const HopParams &hp, const HopViews &v, int i, int s, long rhs,
                                         typename PrecTraits<P>::real *acc) {
  using R = typename PrecTraits<P>::real;
  const int ls = hp.ls;
  // the half fed from s-1 is the upper one for D, the lower one for D^dagger
  // (register arrays are only ever indexed with compile-time offsets)
  const int sb = (s == 0) ? ls - 1 : s - 1, sa = (s == ls - 1) ? 0 : s + 1;
  const R wb = R((s == 0) ? hp.h5wall : hp.h5), wa = R((s == ls - 1) ? hp.h5wall : hp.h5);
  R q[12], w[12], sq_, sw_;
  if constexpr (!DAG) {
    Slice<P>(v.in, rhs * ls + sb).load_half_raw(i, 0, q, sq_);
    Slice<P>(v.in, rhs * ls + sa).load_half_raw(i, 1, w, sw_);
  } else {
    Slice<P>(v.in, rhs * ls + sa).load_half_raw(i, 0, q, sq_);
    Slice<P>(v.in, rhs * ls + sb).load_half_raw(i, 1, w, sw_);
  }
  const R wq = (DAG ? wa : wb) * sq_, ww = (DAG ? wb : wa) * sw_;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    acc[k] += wq * q[k];
    acc[12 + k] += ww * w[k];
  }
}

template <typename R>
__device__ __forceinline__ double norm2_24(const R *a) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 24; k++) s += double(a[k]) * double(a[k]);
  return s;
}

// The non-mixing epilogues of one output (slice sl = rhs * Ls + s, site i),
// acc = the hop.  Reductions are added to red: AXPY |out|^2, |x|^2; CG |r|^2;
// RES |r|^2.  PR: precision of r and p (CG/RES); PX: precision of sol.
template <int P, int EP, int PR, int PX>
__device__ __forceinline__ void hop_epilogue(const HopParams &hp, const HopViews &v, const SolverScalars *st,
                                             long rhs, long sl, int s, int i, bool active,
                                             typename PrecTraits<P>::real *acc, double *red) {
  using R = typename PrecTraits<P>::real;
  if constexpr (EP == EP_STORE || EP == EP_MIX) {
    if (active) SpinorIO<P>::store(v.out, sl, i, acc);
  } else if constexpr (ep_axpy(EP)) {
    // out = x + c hop, streamed 4 reals at a time (few live registers).
    // A thread sums its own 24 squares in the arithmetic precision (FP32 for
    // the sloppy operators: no FP64 conversions per value); everything from
    // the per-thread partial sums on is FP64.
    using RA = typename std::conditional<P == PREC_DOUBLE, double, float>::type;
    RA n_out = RA(0), n_x = RA(0);
    if (active) {
      const R cf = ep_mix(EP) ? R(1) : R(hp.coef[s]);
      ChunkReader<P> xr(v.x, sl, i);
#pragma unroll
      for (int c = 0; c < 6; c++) {
        R xv[4];
        xr.get(c, xv);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          if (hp.norm) n_x += xv[k] * xv[k];
          acc[4 * c + k] = xv[k] + cf * acc[4 * c + k];
          if (hp.norm) n_out += acc[4 * c + k] * acc[4 * c + k];
        }
        if constexpr (P != PREC_HALF) Chunk4<P>::store(v.out, sl, i, c, acc + 4 * c);
      }
      if constexpr (P == PREC_HALF) SpinorIO<P>::store(v.out, sl, i, acc);
    }
    red[0] += double(n_out);
    red[1] += double(n_x);
  } else if constexpr (ep_cg(EP)) {
    // q = x + c hop + shift p;  r -= alpha q;  sol += alpha p;  |r|^2
    using RR = typename PrecTraits<PR>::real;
    using RX = typename PrecTraits<PX>::real;
    RR n_r = RR(0);  // this thread's |r|^2 in r's arithmetic precision
    if (active) {
      const double alpha = st[rhs].alpha;
      const R cf = ep_mix(EP) ? R(1) : R(hp.coef[s]);
      const R sh = R(st[rhs].shift);
      const RR a = RR(alpha);
      const RX ax = RX(alpha);
      const bool with_sol = (v.sol.data != nullptr);  // the multishift solver keeps its own solutions
      RR rfull[PR == PREC_HALF ? 24 : 1];
      ChunkReader<P> xr(v.x, sl, i);
      ChunkReader<PR> pr(v.p, sl, i), rr(v.r, sl, i);
#pragma unroll
      for (int c = 0; c < 6; c++) {
        R xv[4];
        RR pv[4], rv[4];
        xr.get(c, xv);
        pr.get(c, pv);
        rr.get(c, rv);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          R q = xv[k] + cf * acc[4 * c + k] + sh * R(pv[k]);
          rv[k] = rv[k] - a * RR(q);
          n_r += rv[k] * rv[k];
        }
        if constexpr (PR == PREC_HALF) {
#pragma unroll
          for (int k = 0; k < 4; k++) rfull[4 * c + k] = rv[k];
        } else {
          Chunk4<PR>::store(v.r, sl, i, c, rv);
        }
        if (with_sol) {
          RX sv[4];
          Chunk4<PX>::load(v.sol, sl, i, c, sv);
#pragma unroll
          for (int k = 0; k < 4; k++) sv[k] = sv[k] + ax * RX(pv[k]);
          if constexpr (PX != PREC_HALF) Chunk4<PX>::store(v.sol, sl, i, c, sv);
        }
      }
      if constexpr (PR == PREC_HALF) SpinorIO<PR>::store(v.r, sl, i, rfull);
    }
    red[0] += double(n_r);
  } else if constexpr (ep_res(EP)) {
    // r = b - (x + c hop + shift sol), stored in r's precision;  |r|^2
    using RR = typename PrecTraits<PR>::real;
    if (active) {
      const R cf = ep_mix(EP) ? R(1) : R(hp.coef[s]);
      const R sh = R(st[rhs].shift);
      RR rfull[PR == PREC_HALF ? 24 : 1];
      ChunkReader<P> xr(v.x, sl, i), br(v.b, sl, i), sr(v.sol, sl, i);
#pragma unroll
      for (int c = 0; c < 6; c++) {
        R xv[4], bv[4], sv[4];
        xr.get(c, xv);
        br.get(c, bv);
        sr.get(c, sv);
        RR rv[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          R q = bv[k] - (xv[k] + cf * acc[4 * c + k] + sh * sv[k]);
          red[0] += double(q) * double(q);
          rv[k] = RR(q);
        }
        if constexpr (PR == PREC_HALF) {
#pragma unroll
          for (int k = 0; k < 4; k++) rfull[4 * c + k] = rv[k];
        } else {
          Chunk4<PR>::store(v.r, sl, i, c, rv);
        }
      }
      if constexpr (PR == PREC_HALF) SpinorIO<PR>::store(v.r, sl, i, rfull);
    }
  }
}

// reductions of an epilogue: AXPY with norms 2, CG and RES 1, else none
template <int EP> __host__ __device__ constexpr int ep_nred() {
  return ep_axpy(EP) ? 2 : (ep_cg(EP) || ep_res(EP)) ? 1 : 0;
}

// Minimum resident 256-thread blocks per SM the register allocator must
// allow (2 = at most 128 registers per thread, 3 = at most 85).
#ifndef CPSGPU_HOP_MINB_DOUBLE
#define CPSGPU_HOP_MINB_DOUBLE 2
#endif
#ifndef CPSGPU_HOP_MINB_SLOPPY
#define CPSGPU_HOP_MINB_SLOPPY 3
#endif
#ifndef CPSGPU_HOP_MINB_PAIR
#define CPSGPU_HOP_MINB_PAIR 2
#endif

template <int P, int NS> __host__ __device__ constexpr int hop_min_blocks() {
  return P == PREC_DOUBLE ? CPSGPU_HOP_MINB_DOUBLE : NS == 2 ? CPSGPU_HOP_MINB_PAIR : CPSGPU_HOP_MINB_SLOPPY;
}

// NS = 2 (DWF, no mixing, no halos): every thread computes two slices of the
// same 4D parity, s and s + 2, sharing their links (hop_site2); slice group g
// of a block with BS threads in y covers the parity-(g % 2) slices of the run
// [(g / 2) 4 BS, (g / 2 + 1) 4 BS), and Ls is a multiple of 4 BS.
template <int P, int RECON, int EP, int PR, int PX, bool DAG, bool HALO = false, int NS = 1>
__global__ void __launch_bounds__(256, (hop_min_blocks<P, NS>())) hop_kernel(const HopParams hp, const HopViews v,
                                                                           SolverScalars *st, double *partials) {
  using R = typename PrecTraits<P>::real;
  static_assert(NS == 1 || (!HALO && !ep_mix(EP)), "slice pairs: DWF hops without halos or mixing");
  // blockIdx.x = (site block, slice group, rhs within the tile), rhs fastest:
  // consecutive blocks read the same links (for rtile solves) and the same
  // fifth-direction neighbourhoods, which are then still in L1 / L2
  // ORDER_SLICES: blockIdx.x = (site block, slice group, rhs within the
  // tile), rhs fastest; ORDER_SITES: blockIdx.x = (site block, rhs),
  // blockIdx.y = slice group.  Either way consecutive blocks read the same
  // links (rtile solves) and sb numbers the blocks of one solve.
  const int rin = blockIdx.x % hp.rtile, sbx = blockIdx.x / hp.rtile;
  const long rhs = (long)blockIdx.z * hp.rtile + rin;
  if (rhs >= hp.nrhs) return;  // the last tile may be partial
  if (hp.gate == GATE_RUNNING && st[rhs].done) return;
  if (hp.gate == GATE_RELIABLE && (st[rhs].done || !st[rhs].reliable)) return;
  const unsigned nbx = gridDim.x / hp.rtile;
  const unsigned nblk = nbx * gridDim.y;  // blocks of one solve
  const int sb = (int)(blockIdx.y * nbx) + sbx;
  int sgrp, sblk;
  if (gridDim.y > 1) {
    sgrp = blockIdx.y;
    sblk = sbx;
  } else {
    sgrp = sbx % hp.nsg;
    sblk = sbx / hp.nsg;
  }
  int i = sblk * blockDim.x + threadIdx.x;
  bool in_range;
  if constexpr (HALO) {
    // a slab's sites, or its first and last t-slices (the second half of
    // the blocks jumps to the last t-slice)
    i += hp.i0;
    in_range = i < hp.iend;
    if (hp.sub == SUB_BOUNDARY && sblk >= hp.subn) {
      i += hp.jump;
      in_range = i < hp.vh;
    }
  } else {
    // every site (i0 = 0), or a slab's interior (i0 = one t-slice)
    i += hp.i0;
    in_range = i < hp.vh - hp.i0;
  }
  const int s = NS == 2 ? (sgrp >> 1) * 4 * (int)blockDim.y + (sgrp & 1) + 4 * (int)threadIdx.y
                : hp.spar ? (sgrp >> 1) * 2 * (int)blockDim.y + (sgrp & 1) + 2 * (int)threadIdx.y
                          : sgrp * (int)blockDim.y + (int)threadIdx.y;
  const bool active = in_range && (s + 2 * (NS - 1) < hp.ls);
  const long sl = rhs * hp.ls + s;
  const int pin = hp.dwf ? ((s + hp.cb) & 1) : hp.cb;
  const int pout = 1 - pin;
  constexpr int NV = ep_nred<EP>();

  R acc[24];
  if constexpr (NS == 2) {
    R acc1[24];
    if (active) {
      hop_site2<P, RECON, DAG>(hp, v, i, sl, sl + 2, pout, acc, acc1);
      hop5_dwf<P, DAG>(hp, v, i, s, rhs, acc);
      hop5_dwf<P, DAG>(hp, v, i, s + 2, rhs, acc1);
    }
    double red[NV > 0 ? NV : 1] = {};
    hop_epilogue<P, EP, PR, PX>(hp, v, st, rhs, sl, s, i, active, acc, red);
    hop_epilogue<P, EP, PR, PX>(hp, v, st, rhs, sl + 2, s + 2, i, active, acc1, red);
    if constexpr (NV > 0) {
      if (!ep_axpy(EP) || hp.norm) block_partial<NV>(reinterpret_cast<double(&)[NV]>(red), partials, (unsigned)rhs, (unsigned)sb, nblk);
    }
    return;
  } else {
    if (active) {
      hop_site<P, RECON, DAG, HALO>(hp, v, i, sl, pout, acc);
      if (hp.dwf) hop5_dwf<P, DAG>(hp, v, i, s, rhs, acc);
    }
  }

  if constexpr (ep_mix(EP)) {
    // all Ls slices of this block's sites: out(s) = sum_t Mix_chi[s][t] acc(t)
    extern __shared__ unsigned char smraw[];
    R *sm = reinterpret_cast<R *>(smraw);  // [ls][24][BX]: a warp's accesses are consecutive words
    double *mx = reinterpret_cast<double *>(sm + (size_t)hp.ls * blockDim.x * 24);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nmx = 2 * hp.ls * hp.ls * (hp.mix_cplx ? 2 : 1);
    for (int k = tid; k < nmx; k += blockDim.x * blockDim.y) mx[k] = hp.mix[k];
    // FP32 arithmetic with real matrices: the staging is [ls][12][BX] pairs
    // of reals, one 8-byte load and one packed multiply-add per pair (each
    // lane the fused multiply-add of the scalar form)
    constexpr bool PAIRS = std::is_same<R, float>::value;
    const bool pairs = PAIRS && !hp.mix_cplx;
    if (s < hp.ls) {
      if (pairs) {
        float2 *mine2 = reinterpret_cast<float2 *>(sm) + (size_t)s * 12 * blockDim.x + threadIdx.x;
#pragma unroll
        for (int k = 0; k < 12; k++)
          mine2[k * blockDim.x] = active ? make_float2(float(acc[2 * k]), float(acc[2 * k + 1])) : make_float2(0.f, 0.f);
      } else {
        R *mine = sm + (size_t)s * 24 * blockDim.x + threadIdx.x;
#pragma unroll
        for (int k = 0; k < 24; k++) mine[k * blockDim.x] = active ? acc[k] : R(0);
      }
    }
    __syncthreads();
    if (active) {
#pragma unroll
      for (int k = 0; k < 24; k++) acc[k] = R(0);
      if (pairs) {
        if constexpr (PAIRS) {
          float2 a2[12];
#pragma unroll
          for (int k = 0; k < 12; k++) a2[k] = make_float2(0.f, 0.f);
          for (int t2 = 0; t2 < hp.ls; t2++) {
            const float mu_ = float(mx[s * hp.ls + t2]);
            const float md_ = float(mx[hp.ls * hp.ls + s * hp.ls + t2]);
            const float2 *src2 = reinterpret_cast<const float2 *>(sm) + (size_t)t2 * 12 * blockDim.x + threadIdx.x;
#pragma unroll
            for (int k = 0; k < 6; k++) a2[k] = __ffma2_rn(make_float2(mu_, mu_), src2[k * blockDim.x], a2[k]);
#pragma unroll
            for (int k = 6; k < 12; k++) a2[k] = __ffma2_rn(make_float2(md_, md_), src2[k * blockDim.x], a2[k]);
          }
#pragma unroll
          for (int k = 0; k < 12; k++) {
            acc[2 * k] = a2[k].x;
            acc[2 * k + 1] = a2[k].y;
          }
        }
      } else if (!hp.mix_cplx) {
        for (int t2 = 0; t2 < hp.ls; t2++) {
          const R mu_ = R(mx[s * hp.ls + t2]);
          const R md_ = R(mx[hp.ls * hp.ls + s * hp.ls + t2]);
          const R *src = sm + (size_t)t2 * 24 * blockDim.x + threadIdx.x;
#pragma unroll
          for (int k = 0; k < 12; k++) acc[k] += mu_ * src[k * blockDim.x];
#pragma unroll
          for (int k = 12; k < 24; k++) acc[k] += md_ * src[k * blockDim.x];
        }
      } else {
        // complex entries on (re, im) pairs
        for (int t2 = 0; t2 < hp.ls; t2++) {
          const double *pu = mx + 2 * (s * hp.ls + t2), *pd = mx + 2 * (hp.ls * hp.ls + s * hp.ls + t2);
          const R ur = R(pu[0]), ui = R(pu[1]), dr = R(pd[0]), di = R(pd[1]);
          const R *src = sm + (size_t)t2 * 24 * blockDim.x + threadIdx.x;
#pragma unroll
          for (int k = 0; k < 12; k += 2) {
            const R xr = src[k * blockDim.x], xi = src[(k + 1) * blockDim.x];
            acc[k] += ur * xr - ui * xi;
            acc[k + 1] += ur * xi + ui * xr;
          }
#pragma unroll
          for (int k = 12; k < 24; k += 2) {
            const R xr = src[k * blockDim.x], xi = src[(k + 1) * blockDim.x];
            acc[k] += dr * xr - di * xi;
            acc[k + 1] += dr * xi + di * xr;
          }
        }
      }
    }
  }

  double red[NV > 0 ? NV : 1] = {};
  hop_epilogue<P, EP, PR, PX>(hp, v, st, rhs, sl, s, i, active, acc, red);
  if constexpr (NV > 0) {
    if (!ep_axpy(EP) || hp.norm) block_partial<NV>(reinterpret_cast<double(&)[NV]>(red), partials, (unsigned)rhs, (unsigned)sb, nblk);
  }
}

}  // namespace cpsgpu
