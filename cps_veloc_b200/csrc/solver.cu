// Device-resident Krylov solvers on MatPcDagMatPc.
//
//   cg_solve  CG of DiracOp::InvCgShift (inv_cg.C:84-448), same stop test
//             |r|^2 <= stop_rsd^2 |b|^2, same iteration bookkeeping (returns
//             itr + 1) and the true residual recomputed in FP64 at the end.
//             With a sloppy precision (FP32 or FP16 + per-site norm) it runs
//             as a reliable-update mixed-precision CG: the Krylov iteration
//             in the sloppy precision, the solution accumulated in FP64 at
//             every reliable update, where the FP64 true residual b - A x
//             replaces the iterated one and decides convergence.  Every
//             global reduction is done in FP64.
//
// One CG iteration is a fixed sequence of kernels, all of which read their
// scalars (alpha, beta, stop flags) from device memory and return at once
// when the solve is finished.  The solve is one CUDA graph: a WHILE node
// whose body is a chunk of iterations and a one-thread kernel that decides,
// from the solver state, whether another chunk runs (with a hard bound on
// the chunk count); inside each iteration the reliable update sits in an IF
// node.  Without graphs the host enqueues chunks and polls the stop flags
// one chunk behind, so the GPU never waits for the host.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "cpsgpu_impl.h"
#include "hop.cuh"
#include "solver.h"

namespace cpsgpu {

namespace {
SpinorView none() { return SpinorView(); }

// the condition of a reliable-update body: some solve still running has an
// update pending (the gate the body's kernels apply per right-hand side)
__global__ void reliable_cond_kernel(cudaGraphConditionalHandle h, const SolverScalars *st, int nrhs) {
  if (threadIdx.x != 0) return;
  unsigned any = 0;
  for (int k = 0; k < nrhs; k++)
    if (!st[k].done && st[k].reliable) any = 1;
  cudaGraphSetConditional(h, any);
}

// the condition of the solve's WHILE node, after each body (one chunk of
// iterations): another body while some solve is running, never more than
// ctl[1] bodies (ctl[0] counts them), so the loop always ends
__global__ void loop_cond_kernel(cudaGraphConditionalHandle h, const SolverScalars *st, int nrhs, int *ctl) {
  if (threadIdx.x != 0) return;
  const int bodies = ++ctl[0];
  unsigned more = 0;
  for (int k = 0; k < nrhs; k++)
    if (!st[k].done) more = 1;
  if (bodies >= ctl[1]) more = 0;
  cudaGraphSetConditional(h, more);
}
}  // namespace

void CgSolver::setup(int nrhs_) {
  Lattice &L = *D.lat;
  nrhs = nrhs_;
  const long vh = L.vh;
  const int ls = D.ls;
  ensure_field(b64, PREC_DOUBLE, vh, ls, nrhs);
  ensure_field(x64, PREC_DOUBLE, vh, ls, nrhs);
  ensure_field(r, sloppy, vh, ls, nrhs);
  ensure_field(p, sloppy, vh, ls, nrhs);
  const int px = (sloppy == PREC_DOUBLE) ? PREC_DOUBLE : PREC_SINGLE;
  if (sloppy != PREC_DOUBLE) {
    ensure_field(xs, px, vh, ls, nrhs);
    ensure_field(rtmp, PREC_DOUBLE, vh, ls, nrhs);
  }
  ensure_field(ws.t1, sloppy, vh, ls, nrhs);
  ensure_field(ws.t2, sloppy, vh, ls, nrhs);
  if (D.kind == KIND_MOBIUS) ensure_field(ws.t0, sloppy, vh, ls, nrhs);
  ensure_field(wd.t1, PREC_DOUBLE, vh, ls, nrhs);
  ensure_field(wd.t2, PREC_DOUBLE, vh, ls, nrhs);
  if (D.kind == KIND_MOBIUS) ensure_field(wd.t0, PREC_DOUBLE, vh, ls, nrhs);
  // the X = M5 in term of the ORIG preconditioning (allocated here: the
  // operator is captured into graphs, where no allocation may happen)
  if (D.kind == KIND_MOBIUS && (D.plan[0].xmix || D.plan[1].xmix)) {
    ensure_field(ws.t3, sloppy, vh, ls, nrhs);
    ensure_field(wd.t3, PREC_DOUBLE, vh, ls, nrhs);
  }
  st.ensure(sizeof(SolverScalars) * nrhs);
  // partials: 2 values per block; the smallest hop block is 32 threads
  size_t nblk = (size_t)((vh + 31) / 32) * ls + 1024;
  L.partials.ensure(nblk * 2 * nrhs * sizeof(double));
  partials.ensure(nblk * 2 * nrhs * sizeof(double));
  static unsigned long long next_id = 0;
  id = ++next_id;
  drop_graph();
}

void CgSolver::drop_graph() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (graph) cudaGraphDestroy(graph);
  graph_exec = nullptr;
  graph = nullptr;
}

CgSolver::~CgSolver() {
  drop_graph();
  if (side) cudaStreamDestroy(side);
  if (tev0) cudaEventDestroy(tev0);
  if (tev1) cudaEventDestroy(tev1);
}

// Emit out-of-place MatPcDagMatPc on `in` with a final epilogue.
//   final == EP_CG: r -= alpha A in; sol += alpha in; RED_CG_RR
//   final == EP_RES: r_out = b - A in; reduce with red_op
// The M half reduces |M in|^2 (RED_PAP) when pap is set.
void CgSolver::emit_mdagm(int prec, const SpinorView &in, OpWork &w, int final_ep, int pap, int red_op, int gate,
                          const SpinorView &rv, int pr, const SpinorView &solv, int px) {
  SolverScalars *stp = st.as<SolverScalars>();
  const bool mob = (D.kind == KIND_MOBIUS);
  HopLaunch Lh;
  Lh.prec = prec;
  Lh.gate = gate;
  Lh.partials = partials.as<double>();
  // ---- M = MatPc ----
  Lh.dag = 0;
  SpinorView hop_in = w.t1.view(), x = in;
  if (mob) {
    // the preconditioning's plan up to its last hop (mobius_head)
    const MobiusTail t = mobius_head(D, prec, 0, in, w, Lh, stp);
    hop_in = t.hop_in;
    x = t.x;
    Lh.mix = t.mix;
    Lh.coef.assign(D.ls, t.coef);
    Lh.ep = t.mix ? EP_MIX_AXPY : EP_AXPY;
  } else {
    Lh.ep = EP_STORE;
    Lh.cb = 1;
    launch_hop(D, Lh, in, w.t1.view(), none(), none(), none(), none(), none(), stp);
    Lh.coef.assign(D.ls, -D.kappa * D.kappa);
    Lh.ep = EP_AXPY;
  }
  Lh.cb = 0;
  Lh.norm = pap;
  Lh.red_op = RED_PAP;
  launch_hop(D, Lh, hop_in, w.t2.view(), x, none(), none(), none(), none(), stp);
  Lh.mix = nullptr;
  // ---- M^dagger ----
  Lh.norm = 0;
  Lh.dag = 1;
  bool mix_last = false;
  x = w.t2.view();
  if (mob) {
    const MobiusTail t = mobius_head(D, prec, 1, w.t2.view(), w, Lh, stp);
    hop_in = t.hop_in;
    x = t.x;
    Lh.mix = t.mix;
    Lh.coef.assign(D.ls, t.coef);
    mix_last = (t.mix != nullptr);
  } else {
    Lh.ep = EP_STORE;
    Lh.cb = 1;
    launch_hop(D, Lh, w.t2.view(), w.t1.view(), none(), none(), none(), none(), none(), stp);
    hop_in = w.t1.view();
  }
  Lh.cb = 0;
  Lh.red_op = red_op;
  Lh.pr = pr;
  Lh.px = px;
  if (final_ep == EP_CG) {
    Lh.ep = mix_last ? EP_MIX_CG : EP_CG;
    launch_hop(D, Lh, hop_in, none(), x, rv, solv, in, none(), stp);
  } else {
    Lh.ep = mix_last ? EP_MIX_RES : EP_RES;
    launch_hop(D, Lh, hop_in, none(), x, rv, in, none(), b64.view(), stp);
  }
}

// The reliable update: x64 += xs, r = b - A x64 in FP64 (stored in the
// sloppy precision); its kernels skip every solve without a pending update.
void CgSolver::emit_reliable_update() {
  Lattice &L = *D.lat;
  SolverScalars *stp = st.as<SolverScalars>();
  launch_accum_reliable(L.stream, x64.view(), px_of(sloppy), xs.view(), stp, nrhs, 0);
  emit_mdagm(PREC_DOUBLE, x64.view(), wd, EP_RES, 0, RED_RELIABLE, GATE_RELIABLE, r.view(), sloppy, none(),
             PREC_DOUBLE);
}

// One CG iteration.  conditional (while capturing a graph): the reliable
// update sits in the body of an IF node whose condition a one-thread kernel
// sets from the solver state, so the iterations without an update do not
// launch its FP64 operator's grids at all.
void CgSolver::emit_iteration(bool conditional) {
  Lattice &L = *D.lat;
  const int px = (sloppy == PREC_DOUBLE) ? PREC_DOUBLE : PREC_SINGLE;
  SolverScalars *stp = st.as<SolverScalars>();
  const SpinorView solv = (sloppy == PREC_DOUBLE) ? x64.view() : xs.view();
  emit_mdagm(sloppy, p.view(), ws, EP_CG, 1, RED_CG_RR, GATE_RUNNING, r.view(), sloppy, solv, px);
  if (sloppy != PREC_DOUBLE) {
    if (!conditional) {
      emit_reliable_update();
    } else {
      const cudaStream_t s = L.stream;
      cudaStreamCaptureStatus cs;
      cudaGraph_t g;
      const cudaGraphNode_t *deps = nullptr;
      size_t nd = 0;
      CPSGPU_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
      cudaGraphConditionalHandle h;
      CPSGPU_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
      reliable_cond_kernel<<<1, 32, 0, s>>>(h, stp, nrhs);
      CPSGPU_CUDA(cudaGetLastError());
      launch_counter()++;
      CPSGPU_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
      cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      CPSGPU_CUDA(cudaGraphAddNode(&node, g, deps, nd, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      CPSGPU_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
      if (!side) CPSGPU_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
      CPSGPU_CUDA(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
      const long long b0 = launch_counter();
      L.stream = side;
      try {
        emit_reliable_update();
      } catch (...) {
        L.stream = s;
        cudaGraph_t junk;
        cudaStreamEndCapture(side, &junk);
        throw;
      }
      L.stream = s;
      cudaGraph_t captured;
      CPSGPU_CUDA(cudaStreamEndCapture(side, &captured));
      body_kernels = launch_counter() - b0;
      launch_counter() = b0;  // counted when a body runs
    }
  }
  launch_xpay(L.stream, sloppy, p.view(), r.view(), stp, nrhs);
}

// Poll the done flags of all right-hand sides (pinned copy issued earlier).
static bool all_done(const int *flags, int n) {
  for (int k = 0; k < n; k++)
    if (flags[k] == 0) return false;
  return true;
}

void CgSolver::begin(const CgArgs &a) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  SolverScalars *stp = st.as<SolverScalars>();
  if (sloppy != PREC_DOUBLE && L.recon_err > 1e-5)
    throw Error(-1, "mixed precision needs SU(3) links (12-real reconstruction failed)");
  args = a;
  k0 = launch_counter();
  if (!tev0) CPSGPU_CUDA(cudaEventCreate(&tev0));
  if (!tev1) CPSGPU_CUDA(cudaEventCreate(&tev1));
  CPSGPU_CUDA(cudaEventRecord(tev0, s));

  // |b|^2 per right-hand side
  launch_init_scalars(s, stp, nrhs, SolverScalars{});
  launch_norm(s, PREC_DOUBLE, b64.view(), stp, partials.as<double>(), RED_STORE, GATE_NONE);
  std::vector<SolverScalars> host(nrhs);
  CPSGPU_CUDA(cudaMemcpyAsync(host.data(), stp, sizeof(SolverScalars) * nrhs, cudaMemcpyDeviceToHost, s));
  CPSGPU_CUDA(cudaStreamSynchronize(s));
  std::vector<SolverScalars> init(nrhs);
  for (int k = 0; k < nrhs; k++) {
    SolverScalars z;
    memset(&z, 0, sizeof(z));
    double bn = host[k].sum[0];
    z.src_norm = (a.src_norm_sq > 0) ? a.src_norm_sq : bn;
    const double rsd = (k < (int)a.stop_rsds.size()) ? a.stop_rsds[k] : a.stop_rsd;
    z.stop = z.src_norm * rsd * rsd;
    z.max_iter = a.max_num_iter - 1;  // inv_cg.C:275
    z.shift = (k < (int)a.shifts.size()) ? a.shifts[k] : a.shift;
    z.delta2 = (sloppy == PREC_DOUBLE) ? 0.0 : a.delta * a.delta;
    init[k] = z;
  }
  CPSGPU_CUDA(cudaMemcpyAsync(stp, init.data(), sizeof(SolverScalars) * nrhs, cudaMemcpyHostToDevice, s));

  // r = b - A x0 (FP64), p = r
  Field &rinit = (sloppy == PREC_DOUBLE) ? r : rtmp;
  emit_mdagm(PREC_DOUBLE, x64.view(), wd, EP_RES, 0, RED_INIT, GATE_NONE, rinit.view(), PREC_DOUBLE, none(),
             PREC_DOUBLE);
  if (sloppy != PREC_DOUBLE) {
    launch_convert(s, sloppy, r.view(), PREC_DOUBLE, rtmp.view());
    launch_zero(s, xs);
  }
  launch_convert(s, sloppy, p.view(), sloppy, r.view());
}

namespace {
// begin()'s scalars on the device: st[k].sum[0] holds |b_k|^2
__global__ void init_from_norms_kernel(SolverScalars *st, int nrhs, const double *prm, double src_norm_sq,
                                       int max_iter, double delta2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nrhs) return;
  SolverScalars z;
  memset(&z, 0, sizeof(z));
  z.src_norm = (src_norm_sq > 0) ? src_norm_sq : st[k].sum[0];
  const double rsd = prm[2 * k];
  z.stop = z.src_norm * rsd * rsd;
  z.max_iter = max_iter;
  z.shift = prm[2 * k + 1];
  z.delta2 = delta2;
  st[k] = z;
}
}  // namespace

void CgSolver::begin_params(const CgArgs &a) {
  Lattice &L = *D.lat;
  if (sloppy != PREC_DOUBLE && L.recon_err > 1e-5)
    throw Error(-1, "mixed precision needs SU(3) links (12-real reconstruction failed)");
  args = a;
  k0 = launch_counter();
  if (!tev0) CPSGPU_CUDA(cudaEventCreate(&tev0));
  if (!tev1) CPSGPU_CUDA(cudaEventCreate(&tev1));
  std::vector<double> h(2 * (size_t)nrhs);
  for (int k = 0; k < nrhs; k++) {
    h[2 * k] = (k < (int)a.stop_rsds.size()) ? a.stop_rsds[k] : a.stop_rsd;
    h[2 * k + 1] = (k < (int)a.shifts.size()) ? a.shifts[k] : a.shift;
  }
  prm.ensure(h.size() * sizeof(double));
  CPSGPU_CUDA(cudaMemcpyAsync(prm.ptr, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, L.stream));
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
}

void CgSolver::begin_device() {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  SolverScalars *stp = st.as<SolverScalars>();
  launch_init_scalars(s, stp, nrhs, SolverScalars{});
  launch_norm(s, PREC_DOUBLE, b64.view(), stp, partials.as<double>(), RED_STORE, GATE_NONE);
  init_from_norms_kernel<<<(nrhs + 63) / 64, 64, 0, s>>>(stp, nrhs, prm.as<double>(), args.src_norm_sq,
                                                          args.max_num_iter - 1,
                                                          (sloppy == PREC_DOUBLE) ? 0.0 : args.delta * args.delta);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
  // r = b - A x0 (FP64), p = r, as begin()
  Field &rinit = (sloppy == PREC_DOUBLE) ? r : rtmp;
  emit_mdagm(PREC_DOUBLE, x64.view(), wd, EP_RES, 0, RED_INIT, GATE_NONE, rinit.view(), PREC_DOUBLE, none(),
             PREC_DOUBLE);
  if (sloppy != PREC_DOUBLE) {
    launch_convert(s, sloppy, r.view(), PREC_DOUBLE, rtmp.view());
    launch_zero(s, xs);
  }
  launch_convert(s, sloppy, p.view(), sloppy, r.view());
}

// The loop as a WHILE node of graph g whose body is one chunk of iterations
// followed by the condition kernel: no host polling, and the loop stops
// after the chunk in which the last solve finished.
long long CgSolver::add_loop(cudaGraph_t g, int chunk, const cudaGraphNode_t *deps, size_t ndeps) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  SolverScalars *stp = st.as<SolverScalars>();
  ctl.ensure(2 * sizeof(int));
  cudaGraphConditionalHandle hw;
  CPSGPU_CUDA(cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = hw;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wn;
  CPSGPU_CUDA(cudaGraphAddNode(&wn, g, deps, ndeps, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  const long long c0 = launch_counter();
  CPSGPU_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  try {
    for (int k = 0; k < chunk; k++) emit_iteration(true);
    loop_cond_kernel<<<1, 32, 0, s>>>(hw, stp, nrhs, ctl.as<int>());
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
  const long long kernels = launch_counter() - c0;
  launch_counter() = c0;
  return kernels;
}

// the WHILE loop's counters: no body run yet, at most the bound of max_num_iter
void CgSolver::set_loop_limit() {
  const int chunk = args.chunk > 0 ? args.chunk : 8;
  const long max_chunks = (long)args.max_num_iter / chunk + 4;
  const int hctl[2] = {0, (int)std::min<long>(max_chunks, 1L << 30)};
  ctl.ensure(2 * sizeof(int));
  CPSGPU_CUDA(cudaMemcpyAsync(ctl.ptr, hctl, sizeof(hctl), cudaMemcpyHostToDevice, D.lat->stream));
}

int CgSolver::loop_bodies_run() {
  int bodies_run = 0;
  CPSGPU_CUDA(cudaMemcpyAsync(&bodies_run, ctl.ptr, sizeof(int), cudaMemcpyDeviceToHost, D.lat->stream));
  CPSGPU_CUDA(cudaStreamSynchronize(D.lat->stream));
  return bodies_run;
}

void CgSolver::end(std::vector<CgResult> &res, long long replayed) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  SolverScalars *stp = st.as<SolverScalars>();
  // final solution and true residual in FP64 (inv_cg.C:403-415)
  if (sloppy != PREC_DOUBLE) launch_accum_reliable(s, x64.view(), px_of(sloppy), xs.view(), stp, nrhs, 1);
  ensure_field(rtmp, PREC_DOUBLE, L.vh, D.ls, nrhs);
  std::vector<SolverScalars> host(nrhs);
  CPSGPU_CUDA(cudaMemcpyAsync(host.data(), stp, sizeof(SolverScalars) * nrhs, cudaMemcpyDeviceToHost, s));
  CPSGPU_CUDA(cudaStreamSynchronize(s));
  std::vector<SolverScalars> fin = host;
  emit_mdagm(PREC_DOUBLE, x64.view(), wd, EP_RES, 0, RED_STORE, GATE_NONE, rtmp.view(), PREC_DOUBLE, none(),
             PREC_DOUBLE);
  CPSGPU_CUDA(cudaEventRecord(tev1, s));
  CPSGPU_CUDA(cudaMemcpyAsync(host.data(), stp, sizeof(SolverScalars) * nrhs, cudaMemcpyDeviceToHost, s));
  CPSGPU_CUDA(cudaStreamSynchronize(s));
  float dev_ms = 0.f;
  CPSGPU_CUDA(cudaEventElapsedTime(&dev_ms, tev0, tev1));
  int bodies = 0;  // reliable-update bodies that ran (one per iteration in which any solve had one)
  for (int k = 0; k < nrhs; k++) bodies = std::max(bodies, fin[k].n_reliable);
  const long long kernels = launch_counter() - k0 + replayed + (graph_exec || replayed ? (long long)bodies * body_kernels : 0);
  res.resize(nrhs);
  for (int k = 0; k < nrhs; k++) {
    CgResult &o = res[k];
    o.iterations = fin[k].iter + 1;
    o.status = fin[k].done ? fin[k].done : ST_MAX_ITER;
    o.true_res = std::sqrt(host[k].sum[0] / fin[k].src_norm);
    o.reliable_updates = fin[k].n_reliable;
    o.seconds = dev_ms * 1e-3;
    o.final_rr = fin[k].rr;
    o.kernels = kernels;
  }
}

void CgSolver::run(const CgArgs &a, std::vector<CgResult> &res) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  SolverScalars *stp = st.as<SolverScalars>();
  begin(a);
  const int chunk = a.chunk > 0 ? a.chunk : 8;
  const long max_chunks = (long)a.max_num_iter / chunk + 4;
  if (graph_exec && graph_chunk != chunk) drop_graph();
  long long replayed = 0;
  if (a.use_graph) {
    if (!graph_exec) {
      CPSGPU_CUDA(cudaGraphCreate(&graph, 0));
      try {
        graph_kernels = add_loop(graph, chunk);
      } catch (...) {
        drop_graph();
        throw;
      }
      CPSGPU_CUDA(cudaGraphInstantiate(&graph_exec, graph, 0));
      graph_chunk = chunk;
    }
    set_loop_limit();
    CPSGPU_CUDA(cudaGraphLaunch(graph_exec, s));
    replayed = (long long)loop_bodies_run() * graph_kernels;
  } else {
    int *flags = reinterpret_cast<int *>(L.pinned);  // [2][nrhs] ring
    if (nrhs * 2 > 64 * 2) throw Error(-1, "too many right-hand sides for the poll buffer");
    cudaEvent_t ev[2];
    CPSGPU_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    CPSGPU_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    long launched = 0;
    int slot = 0;
    bool finished = false;
    for (long c = 0; c < max_chunks && !finished; c++) {
      for (int k = 0; k < chunk; k++) emit_iteration();
      for (int k = 0; k < nrhs; k++)
        CPSGPU_CUDA(cudaMemcpyAsync(flags + slot * nrhs + k, &stp[k].done, sizeof(int), cudaMemcpyDeviceToHost, s));
      CPSGPU_CUDA(cudaEventRecord(ev[slot], s));
      launched++;
      if (launched >= 2) {
        // look at the chunk before this one while this one runs
        int prev = 1 - slot;
        CPSGPU_CUDA(cudaEventSynchronize(ev[prev]));
        if (all_done(flags + prev * nrhs, nrhs)) finished = true;
      }
      slot = 1 - slot;
    }
    CPSGPU_CUDA(cudaStreamSynchronize(s));
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
  }
  end(res, replayed);
}

// Several independent solves (their own operators, lattices, precisions and
// arguments) as ONE graph launch: every solver's iteration loop is a root
// WHILE node of the graph, so the loops run concurrently on the GPU (the
// small systems in the shadow of the large ones) and finish independently.
namespace {
// The instantiated graph of the last batch: rebuilt when the batch's solvers,
// their set-ups (ids) or their chunk lengths change.
struct BatchGraph {
  std::vector<CgSolver *> solvers;
  std::vector<unsigned long long> ids;
  std::vector<int> chunks;
  std::vector<long long> kernels;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  void drop() {
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    ge = nullptr;
    g = nullptr;
    solvers.clear();
  }
};
BatchGraph g_batch;
}  // namespace

void solve_batch(std::vector<CgSolver *> &solvers, const std::vector<CgArgs> &a,
                 std::vector<std::vector<CgResult>> &res) {
  const size_t n = solvers.size();
  std::vector<int> chunks(n);
  std::vector<unsigned long long> ids(n);
  for (size_t k = 0; k < n; k++) {
    chunks[k] = a[k].chunk > 0 ? a[k].chunk : 8;
    ids[k] = solvers[k]->id;
  }
  for (size_t k = 0; k < n; k++) solvers[k]->begin(a[k]);
  const bool cached = g_batch.ge && g_batch.solvers == solvers && g_batch.ids == ids && g_batch.chunks == chunks;
  if (!cached) {
    g_batch.drop();
    try {
      CPSGPU_CUDA(cudaGraphCreate(&g_batch.g, 0));
      g_batch.kernels.assign(n, 0);
      for (size_t k = 0; k < n; k++) g_batch.kernels[k] = solvers[k]->add_loop(g_batch.g, chunks[k]);
      CPSGPU_CUDA(cudaGraphInstantiate(&g_batch.ge, g_batch.g, 0));
    } catch (...) {
      g_batch.drop();
      throw;
    }
    g_batch.solvers = solvers;
    g_batch.ids = ids;
    g_batch.chunks = chunks;
  }
  for (size_t k = 0; k < n; k++) solvers[k]->set_loop_limit();
  // every loop's set-up is ordered before the launch on the first solver's stream
  cudaStream_t s0 = solvers[0]->D.lat->stream;
  std::vector<cudaEvent_t> ready(n, nullptr);
  cudaEvent_t done = nullptr;
  try {
    for (size_t k = 0; k < n; k++) {
      CPSGPU_CUDA(cudaEventCreateWithFlags(&ready[k], cudaEventDisableTiming));
      CPSGPU_CUDA(cudaEventRecord(ready[k], solvers[k]->D.lat->stream));
      CPSGPU_CUDA(cudaStreamWaitEvent(s0, ready[k], 0));
    }
    CPSGPU_CUDA(cudaGraphLaunch(g_batch.ge, s0));
    CPSGPU_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    CPSGPU_CUDA(cudaEventRecord(done, s0));
    for (size_t k = 0; k < n; k++) CPSGPU_CUDA(cudaStreamWaitEvent(solvers[k]->D.lat->stream, done, 0));
    CPSGPU_CUDA(cudaStreamSynchronize(s0));
  } catch (...) {
    for (auto e : ready)
      if (e) cudaEventDestroy(e);
    if (done) cudaEventDestroy(done);
    throw;
  }
  for (auto e : ready) cudaEventDestroy(e);
  cudaEventDestroy(done);
  res.resize(n);
  for (size_t k = 0; k < n; k++) {
    const long long replayed = (long long)solvers[k]->loop_bodies_run() * g_batch.kernels[k];
    solvers[k]->end(res[k], replayed);
  }
}

int px_of(int sloppy) { return sloppy == PREC_DOUBLE ? PREC_DOUBLE : PREC_SINGLE; }

}  // namespace cpsgpu
