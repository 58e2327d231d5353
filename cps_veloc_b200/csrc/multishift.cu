// Multishift CG (DiracOp::MInvCG, minvcg.C:47-353), device resident.
//
// One iteration is: the M half of MatPcDagMatPc on p_0 (reducing <p,(A+m_0)p>,
// whose last block runs the shifted z / beta recurrences for every shift),
// the M^dagger half with the residual update r += b A p_0 and |r|^2 fused in
// (last block: per-shift convergence), then one kernel that updates psi_s
// and p_s of every shift still running (a thread per site and shift; a thread
// per site summing over the shifts when only the weighted sum is kept).  The
// scalars never leave the device.
//
// precision CPSGPU_SINGLE runs the recurrences on FP32 vectors, the
// solutions included (the per-shift update then moves half the bytes of the
// FP64 one), and then refines every shift with the reliable-update CG on
// MatPcDagMatPc + shift_s, from its FP32 solution, to its own residual.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/cpsgpu.h"
#include "cpsgpu_impl.h"
#include "hop.cuh"
#include "solver.h"

namespace cpsgpu {

namespace {

template <int P> using RealT = typename PrecTraits<P>::real;

// psi_s += w_s (-bs_s) p_s for shifts running at the start of the iteration,
// then p_0 = r + a p_0, p_s = z_s r + as_s p_s for shifts still running.
template <int P>
__global__ void ms_update_kernel(SpinorView r, const SpinorView *pv, const SpinorView *psiv, SpinorView chi,
                                 const MsScalars *ms, const SolverScalars *st, int use_chi) {
  if (ms->upd_done_iter == ms->k) return;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const long per = r.vh * r.ls;
  if (idx >= (size_t)per) return;
  const long sl = (long)(idx / r.vh), i = (long)(idx % r.vh);
  const int n = ms->nshift;
  const bool single = (ms->type == 0);
  const bool more = (st->done == 0);
  RealT<P> rv[24];
  SpinorIO<P>::load(r, sl, i, rv);
  double acc0[24];
  if (single) SpinorIO<PREC_DOUBLE>::load(psiv[0], sl, i, acc0);
  double c[24];
  if (use_chi) SpinorIO<PREC_DOUBLE>::load(chi, sl, i, c);
  for (int s = 0; s < n; s++) {
    const bool upd = !ms->conv_prev[s];
    const bool adv = more && !ms->conv[s];
    if (!upd && !adv) continue;
    RealT<P> pp[24];
    SpinorIO<P>::load(pv[s], sl, i, pp);
    if (upd) {
      const double f = -ms->bs[s] * ms->weight[s];
      if (single) {
#pragma unroll
        for (int k = 0; k < 24; k++) acc0[k] += f * (use_chi ? c[k] : double(pp[k]));
      } else {
        double y[24];
        SpinorIO<PREC_DOUBLE>::load(psiv[s], sl, i, y);
#pragma unroll
        for (int k = 0; k < 24; k++) y[k] += f * (use_chi ? c[k] : double(pp[k]));
        SpinorIO<PREC_DOUBLE>::store(psiv[s], sl, i, y);
      }
    }
    if (adv) {
      const RealT<P> zr = (s == 0) ? RealT<P>(1) : RealT<P>(ms->z[ms->iz][s]);
      const RealT<P> ap = (s == 0) ? RealT<P>(ms->a) : RealT<P>(ms->as[s]);
#pragma unroll
      for (int k = 0; k < 24; k++) pp[k] = zr * rv[k] + ap * pp[k];
      SpinorIO<P>::store(pv[s], sl, i, pp);
    }
  }
  if (single) SpinorIO<PREC_DOUBLE>::store(psiv[0], sl, i, acc0);
}

// The same update with one thread per (site, shift), for solutions kept
// per shift (types MULTI and GENERAL): blockIdx.x = site block x nshift +
// shift, so the blocks of one site block are consecutive and r is read from
// L2 by all but the first shift.
template <int P, int PS>
__global__ void __launch_bounds__(128) ms_update_shift_kernel(SpinorView r, const SpinorView *pv,
                                                              const SpinorView *psiv, SpinorView chi,
                                                              const MsScalars *ms, const SolverScalars *st,
                                                              int use_chi) {
  if (ms->upd_done_iter == ms->k) return;
  const int n = ms->nshift;
  const int s = blockIdx.x % n;
  const size_t idx = (size_t)(blockIdx.x / n) * blockDim.x + threadIdx.x;
  const long per = r.vh * r.ls;
  if (idx >= (size_t)per) return;
  const long sl = (long)(idx / r.vh), i = (long)(idx % r.vh);
  const bool upd = !ms->conv_prev[s];
  const bool adv = (st->done == 0) && !ms->conv[s];
  if (!upd && !adv) return;
  RealT<P> pp[24];
  SpinorIO<P>::load(pv[s], sl, i, pp);
  if (upd) {
    // solutions in PS (FP64, or FP32 in the sloppy phase), updated in FP64
    const double f = -ms->bs[s] * ms->weight[s];
    RealT<PS> y[24];
    double c[24];
    SpinorIO<PS>::load(psiv[s], sl, i, y);
    if (use_chi) SpinorIO<PREC_DOUBLE>::load(chi, sl, i, c);
#pragma unroll
    for (int k = 0; k < 24; k++) y[k] = RealT<PS>(double(y[k]) + f * (use_chi ? c[k] : double(pp[k])));
    SpinorIO<PS>::store(psiv[s], sl, i, y);
  }
  if (adv) {
    RealT<P> rv[24];
    SpinorIO<P>::load(r, sl, i, rv);
    const RealT<P> zr = (s == 0) ? RealT<P>(1) : RealT<P>(ms->z[ms->iz][s]);
    const RealT<P> ap = (s == 0) ? RealT<P>(ms->a) : RealT<P>(ms->as[s]);
#pragma unroll
    for (int k = 0; k < 24; k++) pp[k] = zr * rv[k] + ap * pp[k];
    SpinorIO<P>::store(pv[s], sl, i, pp);
  }
}

__global__ void ms_mark_kernel(MsScalars *ms) { ms->upd_done_iter = ms->k; }

// the condition of the recurrences' WHILE node, after each chunk: another
// chunk while the solve runs, never more than ctl[1] chunks (ctl[0] counts)
__global__ void ms_loop_cond_kernel(cudaGraphConditionalHandle h, const SolverScalars *st, int *ctl) {
  if (threadIdx.x != 0) return;
  const int bodies = ++ctl[0];
  cudaGraphSetConditional(h, (st->done == 0 && bodies < ctl[1]) ? 1u : 0u);
}

}  // namespace

int minvcg(Dirac &D, double *const *psi_h, const double *chi_h, double chi_norm, const double *shift, int nshift,
           double *rsdcg, int type, const double *alpha, int max_num_iter, int precision, int refine) {
  if (nshift > MS_MAX) throw Error(-1, "at most 64 shifts");
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  using clk = std::chrono::steady_clock;
  auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
  const clk::time_point t_start = clk::now();
  const int P = (precision == PREC_DOUBLE) ? PREC_DOUBLE : PREC_SINGLE;
  if (P != PREC_DOUBLE && L.recon_err > 1e-5) throw Error(-1, "sloppy multishift needs SU(3) links");
  const long vh = L.vh;
  const int ls = D.ls;
  const size_t nreal = (size_t)24 * vh * ls;
  // the sloppy path refines every shift, so it keeps individual solutions
  const int dev_type = (P != PREC_DOUBLE && type == 0) ? 1 : type;
  const int npsi = (dev_type == 0) ? 1 : nshift;

  // workspace kept on the operator across calls (allocated on first use)
  MsWork &mw = D.ms;
  Field &chi64 = mw.chi, &r = mw.r, &tmp64 = mw.tmp;
  ensure_field(chi64, PREC_DOUBLE, vh, ls, 1);
  ensure_field(r, P, vh, ls, 1);
  ensure_field(tmp64, PREC_DOUBLE, vh, ls, 1);
  if (mw.p.size() < (size_t)nshift) mw.p.resize(nshift);
  if (mw.psi.size() < (size_t)npsi) mw.psi.resize(npsi);
  std::vector<Field> &p = mw.p, &psi = mw.psi;
  for (int k = 0; k < nshift; k++) ensure_field(p[k], P, vh, ls, 1);
  const int PS = P;  // precision of the solutions during the recurrences
  for (int k = 0; k < npsi; k++) ensure_field(psi[k], PS, vh, ls, 1);
  OpWork &w = mw.w;
  ensure_field(w.t1, P, vh, ls, 1);
  ensure_field(w.t2, P, vh, ls, 1);
  if (D.kind == KIND_MOBIUS) ensure_field(w.t0, P, vh, ls, 1);
  if (D.kind == KIND_MOBIUS && (D.plan[0].xmix || D.plan[1].xmix)) ensure_field(w.t3, P, vh, ls, 1);
  size_t nblk = (size_t)((vh + 31) / 32) * ls + 1024;
  L.partials.ensure(nblk * 2 * sizeof(double));

  L.staging.ensure(nreal * sizeof(double));
  CPSGPU_CUDA(cudaMemcpyAsync(L.staging.ptr, chi_h, nreal * sizeof(double), cudaMemcpyHostToDevice, s));
  launch_import_fermion(s, PREC_DOUBLE, chi64.view(), L.staging.as<double>());
  Field psi0_64;  // GENERAL: the FP64 guess of shift 0 for the initial residual
  if (dev_type == 2) {
    // GENERAL accumulates into the given solutions (only MULTI zeroes them)
    for (int k = 0; k < npsi; k++) {
      CPSGPU_CUDA(cudaMemcpyAsync(L.staging.ptr, psi_h[k], nreal * sizeof(double), cudaMemcpyHostToDevice, s));
      if (PS == PREC_DOUBLE) {
        launch_import_fermion(s, PREC_DOUBLE, psi[k].view(), L.staging.as<double>());
      } else {
        Field &g = (k == 0) ? psi0_64 : tmp64;
        if (k == 0) g.create(PREC_DOUBLE, vh, ls, 1);
        launch_import_fermion(s, PREC_DOUBLE, g.view(), L.staging.as<double>());
        launch_convert(s, PS, psi[k].view(), PREC_DOUBLE, g.view());
      }
    }
  } else {
    for (int k = 0; k < npsi; k++) launch_zero(s, psi[k]);
    if (type == 0 && dev_type == 0) {
      CPSGPU_CUDA(cudaMemcpyAsync(L.staging.ptr, psi_h[0], nreal * sizeof(double), cudaMemcpyHostToDevice, s));
      launch_import_fermion(s, PREC_DOUBLE, psi[0].view(), L.staging.as<double>());
    }
  }

  mw.st.ensure(sizeof(SolverScalars));
  mw.ms.ensure(sizeof(MsScalars));
  SolverScalars *st = mw.st.as<SolverScalars>();
  MsScalars *msd = mw.ms.as<MsScalars>();
  SolverScalars st0;
  memset(&st0, 0, sizeof(st0));
  st0.shift = shift[0];
  st0.ext = msd;

  // r = chi (SINGLE / MULTI) or chi - A psi_0 (GENERAL); cp = |r|^2
  double cp = chi_norm;
  CPSGPU_CUDA(cudaMemcpyAsync(st, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
  if (dev_type == 2) {
    CgSolver tmp(D, PREC_DOUBLE);
    tmp.setup(1);
    CPSGPU_CUDA(cudaMemcpyAsync(tmp.b64.data.ptr, chi64.data.ptr, chi64.data.bytes, cudaMemcpyDeviceToDevice, s));
    // A psi_0 without shift: residual chi - A psi_0 through the RES epilogue
    SolverScalars z0 = st0;
    z0.shift = 0.0;
    SolverScalars *tst = tmp.st.as<SolverScalars>();
    CPSGPU_CUDA(cudaMemcpyAsync(tst, &z0, sizeof(z0), cudaMemcpyHostToDevice, s));
    tmp.emit_mdagm(PREC_DOUBLE, PS == PREC_DOUBLE ? psi[0].view() : psi0_64.view(), tmp.wd, EP_RES, 0, RED_STORE,
                   GATE_NONE, tmp64.view(), PREC_DOUBLE, SpinorView(), PREC_DOUBLE);
    SolverScalars h;
    CPSGPU_CUDA(cudaMemcpyAsync(&h, tst, sizeof(h), cudaMemcpyDeviceToHost, s));
    CPSGPU_CUDA(cudaStreamSynchronize(s));
    cp = h.sum[0];
    launch_convert(s, P, r.view(), PREC_DOUBLE, tmp64.view());
  } else {
    launch_convert(s, P, r.view(), PREC_DOUBLE, chi64.view());
  }
  for (int k = 0; k < nshift; k++) launch_convert(s, P, p[k].view(), P, r.view());

  MsScalars ms0;
  memset(&ms0, 0, sizeof(ms0));
  ms0.nshift = nshift;
  ms0.first = 1;
  ms0.type = dev_type;
  ms0.max_iter = max_num_iter;
  ms0.cp = cp;
  ms0.c = cp;
  ms0.upd_done_iter = -1;
  for (int k = 0; k < nshift; k++) {
    ms0.mass[k] = shift[k];
    ms0.rsd_sq[k] = cp * rsdcg[k] * rsdcg[k];  // minvcg.C:134-137
    ms0.weight[k] = (dev_type == 0) ? alpha[k] : 1.0;
  }
  CPSGPU_CUDA(cudaMemcpyAsync(msd, &ms0, sizeof(ms0), cudaMemcpyHostToDevice, s));

  std::vector<SpinorView> pv(nshift), psiv(npsi);
  for (int k = 0; k < nshift; k++) pv[k] = p[k].view();
  for (int k = 0; k < npsi; k++) psiv[k] = psi[k].view();
  mw.pv.ensure(sizeof(SpinorView) * MS_MAX);
  mw.psiv.ensure(sizeof(SpinorView) * MS_MAX);
  DeviceBuffer &pvd = mw.pv, &psivd = mw.psiv;
  CPSGPU_CUDA(cudaMemcpyAsync(pvd.ptr, pv.data(), sizeof(SpinorView) * nshift, cudaMemcpyHostToDevice, s));
  CPSGPU_CUDA(cudaMemcpyAsync(psivd.ptr, psiv.data(), sizeof(SpinorView) * npsi, cudaMemcpyHostToDevice, s));

  // one iteration: M half (reduce <p,(A+m0)p>), M^dagger half with the
  // residual update, then the per-shift vector updates.
  auto iteration = [&](int use_chi) {
    const bool mob = (D.kind == KIND_MOBIUS);
    HopLaunch Lh;
    Lh.prec = P;
    Lh.gate = GATE_RUNNING;
    Lh.dag = 0;
    const SpinorView in = p[0].view();
    SpinorView hop_in = w.t1.view(), x = in;
    if (mob) {
      // the preconditioning's plan up to its last hop (mobius_head)
      const MobiusTail t = mobius_head(D, P, 0, in, w, Lh, st);
      hop_in = t.hop_in;
      x = t.x;
      Lh.mix = t.mix;
      Lh.coef.assign(ls, t.coef);
      Lh.ep = t.mix ? EP_MIX_AXPY : EP_AXPY;
    } else {
      Lh.ep = EP_STORE;
      Lh.cb = 1;
      launch_hop(D, Lh, in, w.t1.view(), SpinorView(), SpinorView(), SpinorView(), SpinorView(), SpinorView(), st);
      Lh.coef.assign(ls, -D.kappa * D.kappa);
      Lh.ep = EP_AXPY;
    }
    Lh.cb = 0;
    Lh.norm = 1;
    Lh.red_op = RED_MS_PAP;
    launch_hop(D, Lh, hop_in, w.t2.view(), x, SpinorView(), SpinorView(), SpinorView(), SpinorView(), st);
    Lh.mix = nullptr;
    Lh.norm = 0;
    Lh.dag = 1;
    bool mix_last = false;
    x = w.t2.view();
    if (mob) {
      const MobiusTail t = mobius_head(D, P, 1, w.t2.view(), w, Lh, st);
      hop_in = t.hop_in;
      x = t.x;
      Lh.mix = t.mix;
      Lh.coef.assign(ls, t.coef);
      mix_last = (t.mix != nullptr);
    } else {
      Lh.ep = EP_STORE;
      Lh.cb = 1;
      launch_hop(D, Lh, w.t2.view(), w.t1.view(), SpinorView(), SpinorView(), SpinorView(), SpinorView(),
                 SpinorView(), st);
      hop_in = w.t1.view();
    }
    Lh.cb = 0;
    Lh.red_op = RED_MS_RR;
    Lh.pr = P;
    Lh.px = px_of(P);
    Lh.ep = mix_last ? EP_MIX_CG : EP_CG;
    launch_hop(D, Lh, hop_in, SpinorView(), x, r.view(), SpinorView(), in, SpinorView(), st);
    size_t per = (size_t)vh * ls;
    if (dev_type != 0) {
      const unsigned g = (unsigned)((per + 127) / 128) * (unsigned)nshift;
      if (P == PREC_DOUBLE)
        ms_update_shift_kernel<PREC_DOUBLE, PREC_DOUBLE><<<g, 128, 0, s>>>(
            r.view(), pvd.as<SpinorView>(), psivd.as<SpinorView>(), chi64.view(), msd, st, use_chi);
      else
        ms_update_shift_kernel<PREC_SINGLE, PREC_SINGLE><<<g, 128, 0, s>>>(
            r.view(), pvd.as<SpinorView>(), psivd.as<SpinorView>(), chi64.view(), msd, st, use_chi);
    } else if (P == PREC_DOUBLE) {
      ms_update_kernel<PREC_DOUBLE><<<(unsigned)((per + 255) / 256), 256, 0, s>>>(
          r.view(), pvd.as<SpinorView>(), psivd.as<SpinorView>(), chi64.view(), msd, st, use_chi);
    } else {
      throw Error(-2, "multishift: one summed solution only at FP64");
    }
    CPSGPU_CUDA(cudaGetLastError());
    ms_mark_kernel<<<1, 1, 0, s>>>(msd);
    CPSGPU_CUDA(cudaGetLastError());
  };

  CPSGPU_CUDA(cudaStreamSynchronize(s));
  const clk::time_point t_rec = clk::now();
  const int chunk = 8;
  mw.ctl.ensure(2 * sizeof(int));
  const int hctl[2] = {0, (int)std::min<long>((long)max_num_iter / chunk + 4, 1L << 30)};
  const std::vector<long long> key = {P, nshift, dev_type, L.recon(P), D.pc_type, D.cplx ? 1 : 0,
                                      (long long)(size_t)r.data.ptr, (long long)(size_t)w.t1.data.ptr,
                                      (long long)(size_t)p[0].data.ptr, (long long)(size_t)psi[0].data.ptr};
  // the recurrences as a WHILE node of graph g (after deps): chunks of
  // iterations until the solve is done, no host polling; returns the node
  // and the kernels of one body
  auto add_recurrence_loop = [&](cudaGraph_t g, const cudaGraphNode_t *deps, size_t ndeps,
                                 long long *kernels) -> cudaGraphNode_t {
    cudaGraphConditionalHandle hw;
    CPSGPU_CUDA(cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp_ = {cudaGraphNodeTypeConditional};
    cp_.conditional.handle = hw;
    cp_.conditional.type = cudaGraphCondTypeWhile;
    cp_.conditional.size = 1;
    cudaGraphNode_t wn;
    CPSGPU_CUDA(cudaGraphAddNode(&wn, g, deps, ndeps, &cp_));
    cudaGraph_t body = cp_.conditional.phGraph_out[0];
    const long long c0 = launch_counter();
    CPSGPU_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    try {
      for (int k = 0; k < chunk; k++) iteration(0);
      ms_loop_cond_kernel<<<1, 32, 0, s>>>(hw, st, mw.ctl.as<int>());
      CPSGPU_CUDA(cudaGetLastError());
      launch_counter()++;
    } catch (...) {
      cudaGraph_t junk;
      cudaStreamEndCapture(s, &junk);
      launch_counter() = c0;
      throw;
    }
    cudaGraph_t captured;
    CPSGPU_CUDA(cudaStreamEndCapture(s, &captured));
    *kernels = launch_counter() - c0;
    launch_counter() = c0;
    return wn;
  };
  // capture what fn enqueues into graph g after deps; returns the captured
  // part's last nodes (in sinks) and its kernels
  auto capture_segment = [&](cudaGraph_t g, const cudaGraphNode_t *deps, size_t ndeps,
                             std::vector<cudaGraphNode_t> &sinks, auto &&fn) -> long long {
    const long long c0 = launch_counter();
    CPSGPU_CUDA(cudaStreamBeginCaptureToGraph(s, g, deps, nullptr, ndeps, cudaStreamCaptureModeRelaxed));
    try {
      fn();
      cudaStreamCaptureStatus cs;
      const cudaGraphNode_t *tail = nullptr;
      size_t ntail = 0;
      CPSGPU_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &tail, &ntail));
      sinks.assign(tail, tail + ntail);
    } catch (...) {
      cudaGraph_t junk;
      cudaStreamEndCapture(s, &junk);
      launch_counter() = c0;
      throw;
    }
    cudaGraph_t captured;
    CPSGPU_CUDA(cudaStreamEndCapture(s, &captured));
    const long long n = launch_counter() - c0;
    launch_counter() = c0;
    return n;
  };

  MsScalars mh;
  int bodies = 0;
  CgSolver *cg = nullptr;
  const size_t one = (size_t)chi64.data.bytes;
  auto x64_of = [&](int k) {
    SpinorView v = cg->x64.view();
    v.data = (char *)v.data + k * one;
    v.nrhs = 1;
    return v;
  };
  mw.refine_max = mw.refine_sum = 0;
  const bool one_graph = (P != PREC_DOUBLE && refine);
  clk::time_point t_ref;
  if (!one_graph) {
    iteration(1);  // the initial step of minvcg.C:140-188 (psi update from chi)
    // the iterations: one graph launch, the instantiated graph kept on the
    // operator while the configuration is the same
    CachedGraph &lg = mw.loop;
    if (lg.ge && lg.key != key) lg.drop();
    if (!lg.ge) {
      CPSGPU_CUDA(cudaGraphCreate(&lg.g, 0));
      try {
        add_recurrence_loop(lg.g, nullptr, 0, &lg.body_kernels);
      } catch (...) {
        lg.drop();
        throw;
      }
      CPSGPU_CUDA(cudaGraphInstantiate(&lg.ge, lg.g, 0));
      lg.key = key;
    }
    CPSGPU_CUDA(cudaMemcpyAsync(mw.ctl.ptr, hctl, sizeof(hctl), cudaMemcpyHostToDevice, s));
    CPSGPU_CUDA(cudaGraphLaunch(lg.ge, s));
    CPSGPU_CUDA(cudaMemcpyAsync(&mh, msd, sizeof(mh), cudaMemcpyDeviceToHost, s));
    CPSGPU_CUDA(cudaMemcpyAsync(&bodies, mw.ctl.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    CPSGPU_CUDA(cudaStreamSynchronize(s));
    launch_counter() += (long long)bodies * lg.body_kernels;
    // achieved residuals (minvcg.C:315-327)
    for (int k = nshift - 1; k >= 0; k--) {
      if (mh.conv[k])
        rsdcg[k] = std::sqrt(mh.rsd_out[k]);
      else
        rsdcg[k] = std::sqrt(mh.c * mh.z[mh.iz][k] * mh.z[mh.iz][k]);
    }
    t_ref = clk::now();
  } else {
    // FP32 recurrences, then the FP64 refinement of every shift with the
    // reliable-update CG, all shifts as one batched solve (right-hand side
    // k: MatPcDagMatPc + shift_k from the sloppy solution psi_k, to its own
    // residual), as ONE graph launch: the initial step, the recurrences'
    // WHILE node, the refinement's set-up (sources, FP64 starting points,
    // scalars from |b|^2 on the device, the initial residual) and its WHILE
    // node, in that order, with no host round trip between the phases
    if (!mw.refine || mw.refine_n != nshift) {
      mw.full.drop();
      mw.refine = std::make_shared<CgSolver>(D, PREC_SINGLE);
      mw.refine->setup(nshift);
      mw.refine_n = nshift;
    }
    cg = mw.refine.get();
    CgArgs a;
    a.max_num_iter = max_num_iter;
    a.src_norm_sq = 0.0;
    a.delta = 0.01;
    for (int k = 0; k < nshift; k++) {
      a.shifts.push_back(shift[k]);
      a.stop_rsds.push_back(ms0.rsd_sq[k] > 0 ? std::sqrt(ms0.rsd_sq[k] / cp) : 1e-10);
    }
    cg->begin_params(a);
    cg->set_loop_limit();
    CachedGraph &fg = mw.full;
    std::vector<long long> key2 = key;
    key2.push_back((long long)cg->id);
    if (fg.ge && fg.key != key2) fg.drop();
    if (!fg.ge) {
      CPSGPU_CUDA(cudaGraphCreate(&fg.g, 0));
      try {
        std::vector<cudaGraphNode_t> sinks;
        const long long n0 = capture_segment(fg.g, nullptr, 0, sinks, [&] { iteration(1); });
        long long kr = 0;
        const cudaGraphNode_t w1 = add_recurrence_loop(fg.g, sinks.data(), sinks.size(), &kr);
        cudaGraphNode_t e1;
        CPSGPU_CUDA(cudaGraphAddEventRecordNode(&e1, fg.g, &w1, 1, cg->tev0));
        const long long n1 = capture_segment(fg.g, &e1, 1, sinks, [&] {
          for (int k = 0; k < nshift; k++) {
            CPSGPU_CUDA(cudaMemcpyAsync((char *)cg->b64.data.ptr + k * one, chi64.data.ptr, one,
                                        cudaMemcpyDeviceToDevice, s));
            launch_convert(s, PREC_DOUBLE, x64_of(k), PS, psi[k].view());
          }
          cg->begin_device();
        });
        const long long kc = cg->add_loop(fg.g, chunk, sinks.data(), sinks.size());
        fg.body_kernels = kr;
        fg.counts = {n0, n1, kc};
      } catch (...) {
        fg.drop();
        throw;
      }
      CPSGPU_CUDA(cudaGraphInstantiate(&fg.ge, fg.g, 0));
      fg.key = key2;
    }
    cudaEvent_t ev_start;
    CPSGPU_CUDA(cudaEventCreate(&ev_start));
    CPSGPU_CUDA(cudaMemcpyAsync(mw.ctl.ptr, hctl, sizeof(hctl), cudaMemcpyHostToDevice, s));
    CPSGPU_CUDA(cudaEventRecord(ev_start, s));
    CPSGPU_CUDA(cudaGraphLaunch(fg.ge, s));
    CPSGPU_CUDA(cudaMemcpyAsync(&mh, msd, sizeof(mh), cudaMemcpyDeviceToHost, s));
    CPSGPU_CUDA(cudaMemcpyAsync(&bodies, mw.ctl.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    const int refine_bodies = cg->loop_bodies_run();  // synchronises
    float rec_ms = 0.f;
    CPSGPU_CUDA(cudaEventElapsedTime(&rec_ms, ev_start, cg->tev0));
    cudaEventDestroy(ev_start);
    launch_counter() += fg.counts[0] + (long long)bodies * fg.body_kernels + fg.counts[1];
    std::vector<CgResult> res;
    cg->end(res, (long long)refine_bodies * fg.counts[2]);
    for (int k = 0; k < nshift; k++) {
      rsdcg[k] = res[k].true_res * std::sqrt(cp);  // absolute, as minvcg.C:315-327
      mw.refine_max = std::max(mw.refine_max, res[k].iterations);
      mw.refine_sum += res[k].iterations;
    }
    // the phases on the device clock: recurrences up to the event between
    // the phases, the refinement (with its final FP64 residuals) after it
    t_ref = t_rec + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(rec_ms * 1e-3));
  }
  const int iters = mh.k + 1;

  // FP64 view of solution k: the refined solution, else psi_k (converted
  // into tmp64 when it is FP32; used before the next call)
  auto solution = [&](int k) -> SpinorView {
    if (cg) return x64_of(k);
    if (PS == PREC_DOUBLE) return psi[k].view();
    launch_convert(s, PREC_DOUBLE, tmp64.view(), PS, psi[k].view());
    return tmp64.view();
  };
  CPSGPU_CUDA(cudaStreamSynchronize(s));
  const clk::time_point t_out = clk::now();

  // outputs
  if (type == 0 && dev_type != 0) {
    // SINGLE requested: psi_h[0] += sum_s alpha_s psi_s
    std::vector<double> acc(nreal), tmp(nreal);
    CPSGPU_CUDA(cudaStreamSynchronize(s));
    for (size_t q = 0; q < nreal; q++) acc[q] = psi_h[0][q];
    for (int k = 0; k < nshift; k++) {
      launch_export_fermion(s, PREC_DOUBLE, solution(k), L.staging.as<double>());
      CPSGPU_CUDA(cudaMemcpyAsync(tmp.data(), L.staging.ptr, nreal * sizeof(double), cudaMemcpyDeviceToHost, s));
      CPSGPU_CUDA(cudaStreamSynchronize(s));
      for (size_t q = 0; q < nreal; q++) acc[q] += alpha[k] * tmp[q];
    }
    for (size_t q = 0; q < nreal; q++) psi_h[0][q] = acc[q];
  } else {
    for (int k = 0; k < npsi; k++) {
      launch_export_fermion(s, PREC_DOUBLE, solution(k), L.staging.as<double>());
      CPSGPU_CUDA(cudaMemcpyAsync(psi_h[k], L.staging.ptr, nreal * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CPSGPU_CUDA(cudaStreamSynchronize(s));
  }
  mw.upload_s = secs(t_start, t_rec);
  mw.recurrence_s = secs(t_rec, t_ref);
  mw.refine_s = secs(t_ref, t_out);
  mw.download_s = secs(t_out, clk::now());
  return iters;
}

}  // namespace cpsgpu
