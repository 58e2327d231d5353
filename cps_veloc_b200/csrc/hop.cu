// Launch configuration and template dispatch of the hop kernel (hop.cuh).
#include <algorithm>
#include <cstring>

#include "cpsgpu_impl.h"
#include "hop.cuh"
#include "tune.h"

namespace cpsgpu {

namespace {

using HopFn = void (*)(const HopParams, const HopViews, SolverScalars *, double *);

bool g_dag = false;  // set by launch_hop before pick()
int g_ns = 1;        // slices per thread (2: DWF slice pairs)

template <int P, int RECON, int EP, int PR, int PX>
HopFn get() {
  // FP32 arithmetic only: the FP64 pair kernel spills kilobytes
  if constexpr (!ep_mix(EP) && P != PREC_DOUBLE) {
    if (g_ns == 2)
      return g_dag ? hop_kernel<P, RECON, EP, PR, PX, true, false, 2> : hop_kernel<P, RECON, EP, PR, PX, false, false, 2>;
  }
  return g_dag ? hop_kernel<P, RECON, EP, PR, PX, true> : hop_kernel<P, RECON, EP, PR, PX, false>;
}

template <int P, int RECON>
HopFn pick_ep(int ep, int pr, int px) {
  constexpr int PXS = (P == PREC_DOUBLE) ? PREC_DOUBLE : PREC_SINGLE;
  switch (ep) {
    case EP_STORE: return get<P, RECON, EP_STORE, P, P>();
    case EP_AXPY: return get<P, RECON, EP_AXPY, P, P>();
    case EP_MIX: return get<P, RECON, EP_MIX, P, P>();
    case EP_MIX_AXPY: return get<P, RECON, EP_MIX_AXPY, P, P>();
    case EP_CG:
      if (pr == P && px == PXS) return get<P, RECON, EP_CG, P, PXS>();
      break;
    case EP_MIX_CG:
      if (pr == P && px == PXS) return get<P, RECON, EP_MIX_CG, P, PXS>();
      break;
    case EP_RES:
    case EP_MIX_RES:
      if constexpr (P == PREC_DOUBLE) {
        if (ep == EP_RES) {
          if (pr == PREC_DOUBLE) return get<P, RECON, EP_RES, PREC_DOUBLE, P>();
          if (pr == PREC_SINGLE) return get<P, RECON, EP_RES, PREC_SINGLE, P>();
          if (pr == PREC_HALF) return get<P, RECON, EP_RES, PREC_HALF, P>();
        } else {
          if (pr == PREC_DOUBLE) return get<P, RECON, EP_MIX_RES, PREC_DOUBLE, P>();
          if (pr == PREC_SINGLE) return get<P, RECON, EP_MIX_RES, PREC_SINGLE, P>();
          if (pr == PREC_HALF) return get<P, RECON, EP_MIX_RES, PREC_HALF, P>();
        }
      }
      break;
  }
  throw Error(-2, "hop: unsupported epilogue/precision combination");
}

HopFn pick(int prec, int recon, int ep, int pr, int px) {
  if (prec == PREC_DOUBLE) return recon == 18 ? pick_ep<PREC_DOUBLE, 18>(ep, pr, px) : pick_ep<PREC_DOUBLE, 12>(ep, pr, px);
  if (prec == PREC_SINGLE) return recon == 18 ? pick_ep<PREC_SINGLE, 18>(ep, pr, px) : pick_ep<PREC_SINGLE, 12>(ep, pr, px);
  if (recon == LINK_F32_18) return pick_ep<PREC_HALF, LINK_F32_18>(ep, pr, px);
  if (recon == LINK_F32_12) return pick_ep<PREC_HALF, LINK_F32_12>(ep, pr, px);
  return recon == 18 ? pick_ep<PREC_HALF, 18>(ep, pr, px) : pick_ep<PREC_HALF, 12>(ep, pr, px);
}

// the t-slab decomposition's hops (store epilogue, FP64 / FP32)
HopFn pick_halo(int prec, int recon) {
  if (recon != 12 && recon != 18) throw Error(-2, "decomposed hop: 12- or 18-real links");
  if (prec == PREC_DOUBLE)
    return recon == 12 ? (g_dag ? hop_kernel<PREC_DOUBLE, 12, EP_STORE, PREC_DOUBLE, PREC_DOUBLE, true, true>
                                : hop_kernel<PREC_DOUBLE, 12, EP_STORE, PREC_DOUBLE, PREC_DOUBLE, false, true>)
                       : (g_dag ? hop_kernel<PREC_DOUBLE, 18, EP_STORE, PREC_DOUBLE, PREC_DOUBLE, true, true>
                                : hop_kernel<PREC_DOUBLE, 18, EP_STORE, PREC_DOUBLE, PREC_DOUBLE, false, true>);
  return recon == 12 ? (g_dag ? hop_kernel<PREC_SINGLE, 12, EP_STORE, PREC_SINGLE, PREC_SINGLE, true, true>
                              : hop_kernel<PREC_SINGLE, 12, EP_STORE, PREC_SINGLE, PREC_SINGLE, false, true>)
                     : (g_dag ? hop_kernel<PREC_SINGLE, 18, EP_STORE, PREC_SINGLE, PREC_SINGLE, true, true>
                              : hop_kernel<PREC_SINGLE, 18, EP_STORE, PREC_SINGLE, PREC_SINGLE, false, true>);
}

size_t real_size(int prec) { return prec == PREC_DOUBLE ? 8 : 4; }

}  // namespace

void launch_hop(const Dirac &D, const HopLaunch &L, const SpinorView &in, const SpinorView &out,
                const SpinorView &x, const SpinorView &r, const SpinorView &sol, const SpinorView &p,
                const SpinorView &b, SolverScalars *st) {
  const Lattice &lat = *D.lat;
  HopParams hp;
  memset(&hp, 0, sizeof(hp));
  for (int k = 0; k < 4; k++) {
    hp.L[k] = lat.L[k];
    hp.bc[k] = lat.bc[k];
  }
  hp.hx = lat.L[0] / 2;
  hp.dhx.init(hp.hx);
  hp.dly.init(lat.L[1]);
  hp.dlz.init(lat.L[2]);
  hp.vh = lat.vh;
  hp.ls = D.ls;
  hp.cb = L.cb;
  hp.dag = L.dag;
  hp.dwf = (D.kind == KIND_DWF);
  hp.h5 = 2.0 * D.a5inv;              // 2 / a5 (dwf_dslash_5_plus_omp.C:137)
  hp.h5wall = -2.0 * D.mass * D.a5inv; // -2 m_f / a5 (:138)
  for (int s = 0; s < D.ls && s < MAX_LS; s++) hp.coef[s] = L.coef.empty() ? 0.0 : L.coef[(size_t)s < L.coef.size() ? s : 0];
  hp.mix = L.mix;
  hp.mix_cplx = (L.mix != nullptr && D.cplx) ? 1 : 0;
  hp.norm = L.norm;
  hp.red_op = L.red_op;
  hp.gate = L.gate;
  hp.face = (int)(lat.vh / lat.L[3]);
  hp.tb_fwd = (lat.t_coor == lat.t_nodes - 1) ? 1 : 0;
  hp.tb_bwd = (lat.t_coor == 0) ? 1 : 0;
  const bool split = (lat.t_nodes > 1);
  if (!split && L.sub != SUB_ALL) throw Error(-4, "interior / boundary hops: a t-partitioned lattice");
  // the interior of a slab reads no halo: the undecomposed kernel serves it
  const bool halo = split && L.sub != SUB_INTERIOR;
  if (halo && (!L.halo_fwd || !L.halo_bwd))
    throw Error(-1, "t-partitioned lattice: only the decomposed dslash (with its halos) applies the operator");
  if (split && (L.ep != EP_STORE || (L.prec != PREC_DOUBLE && L.prec != PREC_SINGLE)))
    throw Error(-2, "decomposed hop: store epilogue, FP64 or FP32");
  hp.sub = L.sub;

  HopViews v;
  v.U = lat.gauge(L.prec);
  v.in = in;
  v.out = out;
  v.x = x;
  v.r = r;
  v.sol = sol;
  v.p = p;
  v.b = b;
  v.hf = L.halo_fwd;
  v.hb = L.halo_bwd;

  const int recon = lat.recon(L.prec);
  const bool mix = ep_mix(L.ep);
  TuneKey key{L.prec, recon, L.ep, D.kind, D.ls};
  dim3 block = hop_block(key, mix);
  // block.z of a tuned shape: slices per thread (2: DWF slice pairs)
  g_ns = (block.z == 2 && hp.dwf && !mix && !halo && L.prec != PREC_DOUBLE && D.ls % (4 * (int)block.y) == 0) ? 2 : 1;
  block.z = 1;
  g_dag = (L.dag != 0);
  HopFn fn = halo ? pick_halo(L.prec, recon) : pick(L.prec, recon, L.ep, L.pr, L.px);
  unsigned nsb;
  if (L.sub == SUB_BOUNDARY) {
    hp.subn = (hp.face + (int)block.x - 1) / (int)block.x;
    nsb = 2u * (unsigned)hp.subn;
    hp.i0 = 0;
    hp.iend = hp.face;
    hp.jump = (int)lat.vh - hp.face - hp.subn * (int)block.x;
  } else {
    const long nsites = (L.sub == SUB_INTERIOR) ? lat.vh - 2L * hp.face : lat.vh;
    if (nsites <= 0) return;  // a slab of two t-slices has no interior
    nsb = (unsigned)((nsites + block.x - 1) / block.x);
    hp.i0 = (L.sub == SUB_INTERIOR) ? hp.face : 0;
    hp.iend = hp.i0 + (int)nsites;
  }
  hp.nsg = g_ns == 2 ? D.ls / (2 * (int)block.y) : (D.ls + block.y - 1) / block.y;
  // ORDER_SITES: the slice groups on the grid's y (blocks run x fastest)
  const bool sites_first = (hop_order(key) == ORDER_SITES && hp.nsg > 1);
  hp.spar = (hp.dwf && !mix && block.y > 1 && D.ls % (2 * block.y) == 0) ? 1 : 0;
  hp.nrhs = in.nrhs;
  hp.rtile = std::max(1, std::min(D.rhs_tile(L.prec, in.nrhs), in.nrhs));
  const unsigned ntile = (unsigned)((in.nrhs + hp.rtile - 1) / hp.rtile);
  dim3 grid = sites_first ? dim3(nsb * hp.rtile, hp.nsg, ntile) : dim3(nsb * hp.nsg * hp.rtile, 1, ntile);
  size_t smem = 0;
  if (mix) {
    smem = (size_t)D.ls * block.x * 24 * real_size(L.prec) + 2 * (size_t)D.ls * D.ls * sizeof(double) * (D.cplx ? 2 : 1);
    // the attribute belongs to the kernel on one device: raised once per (device, kernel, size)
    struct Raised {
      int dev;
      HopFn fn;
      size_t smem;
    };
    static thread_local std::vector<Raised> raised;
    bool done = false;
    for (auto &e : raised)
      if (e.dev == lat.device && e.fn == fn && e.smem >= smem) done = true;
    if (!done) {
      CPSGPU_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      raised.push_back({lat.device, fn, smem});
    }
  }
  double *part = L.partials ? L.partials : lat.partials.as<double>();
  fn<<<grid, block, smem, lat.stream>>>(hp, v, st, part);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
  // the epilogue's reduction: per-block partials, summed and applied here
  const int nv = (ep_axpy(L.ep) && L.norm) ? 2 : (ep_cg(L.ep) || ep_res(L.ep)) ? 1 : 0;
  if (nv && st) launch_finalize(lat.stream, nv, part, st, L.red_op, nsb * hp.nsg, in.nrhs, L.gate);
}

}  // namespace cpsgpu
