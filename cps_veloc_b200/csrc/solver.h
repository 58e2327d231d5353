// Krylov solvers (solver.cu, multishift.cu).
#pragma once
#include <vector>

#include "cpsgpu_impl.h"

namespace cpsgpu {

struct CgArgs {
  double stop_rsd = 1e-8;
  int max_num_iter = 10000;
  double src_norm_sq = 0.0;  // 0: computed from the source (inv_cg.C:166-169)
  double shift = 0.0;
  double delta = 0.1;        // reliable-update threshold (mixed precision)
  int chunk = 8;             // iterations per captured graph
  int use_graph = 1;
  // per right-hand side, when given (one entry per right-hand side): the
  // shift and the stopping residual of each system of a batched solve
  std::vector<double> shifts, stop_rsds;
};

struct CgResult {
  int iterations = 0;        // reference convention: iterations done + 1
  int status = 0;
  double true_res = 0.0;     // |b - A x| / |b|
  int reliable_updates = 0;
  double seconds = 0.0;
  double final_rr = 0.0;
  long long kernels = 0;     // kernels executed (early-exit ones included)
};

int px_of(int sloppy);

// Solves (MatPcDagMatPc + shift) x = b for nrhs right-hand sides at once
// (each with its own scalars and convergence) in precision `sloppy`
// (PREC_DOUBLE: plain FP64 CG).  b64 and x64 (initial guess in, solution
// out) are filled by the caller.
struct CgSolver {
  Dirac &D;
  int sloppy;
  int nrhs = 0;
  Field b64, x64, r, p, xs, rtmp;
  OpWork ws, wd;
  DeviceBuffer st;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  long long graph_kernels = 0;  // kernels of one chunk outside the conditional bodies
  long long body_kernels = 0;   // kernels of one reliable-update body
  int graph_chunk = 0;
  cudaStream_t side = nullptr;  // captures the conditional bodies
  DeviceBuffer ctl;              // the WHILE loop's body count and limit
  DeviceBuffer partials;         // this solver's reduction partials (solves may share a lattice)
  DeviceBuffer prm;              // begin_params: [nrhs][stop_rsd, shift]
  unsigned long long id = 0;     // new at every setup(): a graph holding this solver's buffers is current while it matches
  // state of one run between begin() and end()
  CgArgs args;
  long long k0 = 0;
  cudaEvent_t tev0 = nullptr, tev1 = nullptr;

  CgSolver(Dirac &d, int sloppy_prec) : D(d), sloppy(sloppy_prec) {}
  ~CgSolver();
  void setup(int nrhs);
  void run(const CgArgs &a, std::vector<CgResult> &res);
  // run() in three steps, so that several solvers' loops can share one graph:
  // begin() sets up the scalars and the initial residual (it synchronises);
  // add_loop() adds the iteration loop as a WHILE node (a root) to graph g
  // and returns the kernels of one body; end() finishes after the loop ran.
  void begin(const CgArgs &a);
  // begin() without its host synchronisation, for a caller that captures
  // the set-up into a graph: begin_params() uploads the per-right-hand-side
  // stopping residuals and shifts (not capturable), begin_device() enqueues
  // the rest, the scalars derived on the device from |b|^2 exactly as
  // begin() derives them on the host
  void begin_params(const CgArgs &a);
  void begin_device();
  long long add_loop(cudaGraph_t g, int chunk, const cudaGraphNode_t *deps = nullptr, size_t ndeps = 0);
  void set_loop_limit();
  void end(std::vector<CgResult> &res, long long replayed);
  int loop_bodies_run();
  void drop_graph();
  void emit_iteration(bool conditional = false);
  void emit_reliable_update();
  void emit_mdagm(int prec, const SpinorView &in, OpWork &w, int final_ep, int pap, int red_op, int gate,
                  const SpinorView &rv, int pr, const SpinorView &solv, int px);
};

// Independent solves in one graph launch (solver.cu); each solver set up for
// its right-hand sides, with b64 / x64 filled.  res[k] per solver.
void solve_batch(std::vector<CgSolver *> &solvers, const std::vector<CgArgs> &a,
                 std::vector<std::vector<CgResult>> &res);

}  // namespace cpsgpu
