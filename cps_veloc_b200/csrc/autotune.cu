// Autotuner: times candidate block shapes of the hop kernels on the live
// lattice and records the fastest in the launch table (tune.cpp).  A shape
// is (sites per block) x (slices per block) x (slices per thread, DWF) and
// the block traversal order (HopOrder): every shape is timed on the plain
// hop, and the four fastest in each order on a whole MatPcDagMatPc, whose
// epilogue kernels take the same shape; the mixing epilogue of the Mobius
// operator needs all slices of a site in one block, so only its site count
// varies.
#include <algorithm>
#include <vector>

#include "cpsgpu_impl.h"
#include "hop.cuh"
#include "tune.h"
#include "solver.h"

namespace cpsgpu {

namespace {
SpinorView none() { return SpinorView(); }

float time_launch(const Dirac &D, HopLaunch &Lh, const Field &in, const Field &out, const Field &x,
                  SolverScalars *st, cudaEvent_t e0, cudaEvent_t e1) {
  cudaStream_t s = D.lat->stream;
  for (int k = 0; k < 2; k++) launch_hop(D, Lh, in.view(), out.view(), x.view(), none(), none(), none(), none(), st);
  CPSGPU_CUDA(cudaEventRecord(e0, s));
  const int reps = 5;
  for (int k = 0; k < reps; k++) launch_hop(D, Lh, in.view(), out.view(), x.view(), none(), none(), none(), none(), st);
  CPSGPU_CUDA(cudaEventRecord(e1, s));
  CPSGPU_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  CPSGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  return ms / reps;
}
}  // namespace

int autotune(Dirac &D, int prec, int nrhs) {
  Lattice &L = *D.lat;
  Field in(prec, L.vh, D.ls, nrhs), out(prec, L.vh, D.ls, nrhs), x(prec, L.vh, D.ls, nrhs);
  Field cg_r, cg_sol;  // the CG epilogue's residual and solution
  launch_zero(L.stream, in);
  launch_zero(L.stream, x);
  size_t nblk = (size_t)((L.vh + 15) / 16) * D.ls + 1024;
  L.partials.ensure(nblk * 2 * nrhs * sizeof(double));
  cudaEvent_t e0, e1;
  CPSGPU_CUDA(cudaEventCreate(&e0));
  CPSGPU_CUDA(cudaEventCreate(&e1));
  int tuned = 0;
  // plain hop shapes (also used by the AXPY / CG / RES epilogues); for FP32
  // and FP16 also the stored link form (12 reals rebuilt, or all 18)
  std::vector<int> recons;
  if (prec == PREC_DOUBLE) recons.push_back(L.recon(prec));
  else if (prec == PREC_HALF) recons = {12, 18, LINK_F32_12, LINK_F32_18};
  else recons = {12, 18};
  float best_recon_t = 1e30f;
  int best_recon = recons[0];
  for (int recon : recons) {
    if (prec != PREC_DOUBLE) L.sloppy_recon[prec] = recon;
    HopLaunch Lh;
    Lh.prec = prec;
    Lh.ep = EP_STORE;
    Lh.cb = 1;
    std::vector<dim3> cand;
    // 8 or 16 sites per block: a warp spans 4 or 2 same-parity slices of
    // the same sites, whose lanes then read the same link addresses
    const int bxs[] = {8, 16, 32, 64, 128, 256};
    const int bss[] = {1, 2, 4, 8, 16};
    for (int bx : bxs)
      for (int bs : bss)
        if (bx * bs <= 256 && bx * bs >= (bx == 8 ? 32 : 64) && bs <= (D.ls > 1 ? D.ls : 1)) {
          cand.push_back(dim3(bx, bs));
          // DWF slice pairs: two same-parity slices per thread sharing links
          if (D.kind == KIND_DWF && prec != PREC_DOUBLE && D.ls % (4 * bs) == 0) cand.push_back(dim3(bx, bs, 2));
        }
    TuneKey key{prec, recon, EP_STORE, D.kind, D.ls};
    std::vector<std::pair<float, dim3>> timed;
    for (auto b : cand) {
      tune_set(key, b);
      timed.push_back({time_launch(D, Lh, in, out, x, nullptr, e0, e1), b});
    }
    std::stable_sort(timed.begin(), timed.end(),
                     [](const std::pair<float, dim3> &a, const std::pair<float, dim3> &b) { return a.first < b.first; });
    const int eps[] = {EP_STORE, EP_AXPY, EP_CG, EP_RES};
    auto set_all = [&](dim3 b, int o) {
      for (int ep : eps) tune_set(TuneKey{prec, recon, ep, D.kind, D.ls}, b, o);
    };
    // a whole MatPcDagMatPc and, for Wilson and DWF, the solver's last hop
    // with its CG epilogue (r -= alpha q, sol += alpha p, |r|^2: the
    // DRAM-bound kernel of an iteration): the epilogue kernels take the same
    // shape and re-read what the plain hop does not
    OpWork w;
    SolverScalars *st = L.scratch_st.as<SolverScalars>();
    if (D.kind != KIND_MOBIUS) {
      ensure_field(cg_r, prec, L.vh, D.ls, nrhs);
      ensure_field(cg_sol, px_of(prec), L.vh, D.ls, nrhs);
      launch_zero(L.stream, cg_r);
      launch_zero(L.stream, cg_sol);
    }
    auto one = [&]() {
      op_mdagm(D, prec, out.view(), in.view(), w, st, RED_STORE);
      if (D.kind == KIND_MOBIUS) return;
      HopLaunch Lc;
      Lc.prec = prec;
      Lc.ep = EP_CG;
      Lc.cb = 0;
      Lc.dag = 1;
      Lc.pr = prec;
      Lc.px = px_of(prec);
      Lc.red_op = RED_STORE;
      Lc.coef.assign(D.ls, -D.kappa * D.kappa);
      launch_hop(D, Lc, out.view(), SpinorView(), x.view(), cg_r.view(), cg_sol.view(), in.view(), SpinorView(), st);
    };
    auto mdagm_ms = [&]() -> float {
      CPSGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(SolverScalars), L.stream));
      for (int k = 0; k < 2; k++) one();
      CPSGPU_CUDA(cudaEventRecord(e0, L.stream));
      for (int k = 0; k < 5; k++) one();
      CPSGPU_CUDA(cudaEventRecord(e1, L.stream));
      CPSGPU_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      CPSGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      return ms;
    };
    dim3 bestb = timed.empty() ? hop_block(key, false) : timed[0].second;
    int besto = ORDER_SLICES;
    if (L.t_nodes > 1) {
      // a slab of a decomposed lattice applies no whole operator: the plain hop decides, in site order
      float best = timed.empty() ? 1e30f : timed[0].first;
      for (int o = ORDER_SITES; o < ORDER_COUNT; o++) {
        tune_set(key, bestb, o);
        float t = time_launch(D, Lh, in, out, x, nullptr, e0, e1);
        if (t < best) { best = t; besto = o; }
      }
    } else {
      // the few fastest shapes of the plain hop, in every site order, on
      // the whole operator.  With several slices, only shapes whose blocks
      // share each link between slices (several slices per block, or slice
      // pairs): with one slice per block every slice's block re-reads the
      // links, which the operator alone hides in L2 but a solve, whose
      // vector kernels evict them, pays for in DRAM
      std::vector<dim3> pick;
      for (auto &tb : timed)
        if (D.ls == 1 || tb.second.y > 1 || tb.second.z > 1) pick.push_back(tb.second);
      if (pick.empty())
        for (auto &tb : timed) pick.push_back(tb.second);
      if (pick.size() > 4) pick.resize(4);
      float best = 1e30f;
      for (auto b : pick)
        for (int o = ORDER_SLICES; o < ORDER_COUNT; o++) {
          set_all(b, o);
          const float t = mdagm_ms();
          if (t < best) { best = t; bestb = b; besto = o; }
        }
      // the link form on the whole operator too (its epilogue kernels need
      // more registers than the plain hop)
      if (prec != PREC_DOUBLE && best < best_recon_t) {
        best_recon_t = best;
        best_recon = recon;
      }
    }
    set_all(bestb, besto);
    tuned += 4;
  }
  if (prec != PREC_DOUBLE) L.sloppy_recon[prec] = best_recon;
  const int recon = L.recon(prec);
  if (nrhs > 1) {
    // right-hand-side tile: how many solves' blocks of the same sites run
    // back to back (link reuse across right-hand sides)
    HopLaunch Lh;
    Lh.prec = prec;
    Lh.ep = D.kind == KIND_MOBIUS ? EP_MIX : EP_STORE;
    Lh.mix = D.kind == KIND_MOBIUS ? D.mixQ.as<double>() : nullptr;
    Lh.cb = 1;
    float best = 1e30f;
    int bestr = 1;
    const int tiles[] = {1, 2, 4, 8, 12, 16};
    for (int r : tiles) {
      if (r > nrhs) break;
      D.rtile[prec] = r;
      float t = time_launch(D, Lh, in, out, x, nullptr, e0, e1);
      if (t < best) { best = t; bestr = r; }
    }
    D.rtile[prec] = bestr;
    tuned++;
  }
  if (D.kind == KIND_MOBIUS) {
    HopLaunch Lh;
    Lh.prec = prec;
    Lh.ep = EP_MIX;
    Lh.cb = 1;
    Lh.mix = D.mixQ.as<double>();
    TuneKey key{prec, recon, EP_MIX, D.kind, D.ls};
    float best = 1e30f;
    dim3 bestb = hop_block(key, true);
    for (int bx = 1; bx * D.ls <= 256; bx *= 2) {
      dim3 b(bx, D.ls);
      tune_set(key, b);
      float t = time_launch(D, Lh, in, out, x, nullptr, e0, e1);
      if (t < best) { best = t; bestb = b; }
    }
    const int eps[] = {EP_MIX, EP_MIX_AXPY, EP_MIX_CG, EP_MIX_RES};
    for (int ep : eps) {
      tune_set(TuneKey{prec, recon, ep, D.kind, D.ls}, bestb);
      tuned++;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return tuned;
}

}  // namespace cpsgpu
