// Deterministic grid reductions in FP64 and the solver's device-resident
// scalars.
//
// Every reducing kernel sums its per-thread values in a fixed order (warp
// shuffle, then warps in index order) and writes one partial per block; a
// small finalize kernel then adds one solve's partials in block order and
// updates its scalars.  Results are therefore bit-reproducible run to run,
// and the host never has to read a scalar to keep the Krylov loop going.
#pragma once
#include <cuda_runtime.h>

namespace cpsgpu {

// Solver status codes (also returned through the C ABI).
enum SolverStatus {
  ST_RUNNING = 0,
  ST_CONVERGED = 1,
  ST_MAX_ITER = 2,
  ST_BREAKDOWN = 3,  // p.Ap == 0: the reference exits the process (inv_cg.C:326-329)
  ST_NONFINITE = 4,
};

// Scalars of one Krylov solve, resident in device memory.
struct SolverScalars {
  double rr;        // |r|^2 of the iterated residual
  double rr_prev;   // previous |r|^2
  double d;         // p . A p
  double alpha, beta;
  double stop;      // stop when |r|^2 <= stop  (src_norm_sq * stop_rsd^2)
  double src_norm;  // |b|^2
  double rr_max;    // largest |r|^2 since the last reliable update
  double delta2;    // reliable-update threshold (squared)
  double shift;     // A + shift
  double sum[4];    // raw reduction results of the last finalize
  int iter;
  int max_iter;
  int done;         // SolverStatus once finished, else 0
  int reliable;     // 1 while a reliable update is pending in this iteration
  int n_reliable;   // reliable updates performed
  int pad[1];
  void *ext;        // solver-specific extension (multishift scalars)
  unsigned int pad2[4];
};

// What the finalize step does with the reduced sums.
enum ReduceOp {
  RED_STORE = 0,      // sum[] only
  RED_PAP = 1,        // sum[0] = |M p|^2, sum[1] = |p|^2: d, alpha
  RED_CG_RR = 2,      // sum[0] = |r_new|^2: iteration bookkeeping, beta
  RED_RELIABLE = 3,   // sum[0] = |b - A x|^2 (true residual): reset sloppy state
  RED_INIT = 4,       // sum[0] = |r0|^2 of the initial residual
  RED_MS_PAP = 5,     // multishift: d, b, shifted z / beta recurrences
  RED_MS_RR = 6,      // multishift: c = |r|^2, per-shift convergence
};

constexpr int MS_MAX = 64;

// Device-resident scalars of the multishift CG (DiracOp::MInvCG,
// minvcg.C:47-353), reached through SolverScalars::ext.
struct MsScalars {
  int nshift, iz, first, type;
  int k, max_iter, conv_all, upd_done_iter;
  double a, b, bp, c, cp, d;
  double mass[MS_MAX], rsd_sq[MS_MAX], weight[MS_MAX];
  double z[2][MS_MAX], bs[MS_MAX], as[MS_MAX];
  double rsd_out[MS_MAX];
  int conv[MS_MAX], conv_prev[MS_MAX], conv_iter[MS_MAX];
};

// the shifted-system recurrences of minvcg.C, run by the last block
__device__ inline void finalize_multishift(SolverScalars *st, int op, const double *sum) {
  MsScalars *ms = reinterpret_cast<MsScalars *>(st->ext);
  const int n = ms->nshift;
  if (op == RED_MS_PAP) {
    // d = <p, (A + m_0) p>   (minvcg.C:141-148, :228-236)
    double d = sum[0] + ms->mass[0] * sum[1];
    ms->d = d;
    if (!isfinite(d)) { st->done = ST_NONFINITE; return; }
    if (d == 0.0) { st->done = ST_BREAKDOWN; return; }
    ms->bp = ms->b;
    ms->b = -ms->cp / d;
    if (ms->first) {
      // minvcg.C:152-165
      ms->z[0][0] = ms->z[1][0] = 1.0;
      ms->bs[0] = ms->b;
      ms->iz = 1;
      for (int s = 1; s < n; s++) {
        ms->z[1 - ms->iz][s] = 1.0;
        ms->z[ms->iz][s] = 1.0 / (1.0 - ms->b * (ms->mass[s] - ms->mass[0]));
        ms->bs[s] = ms->b * ms->z[ms->iz][s];
      }
    } else {
      // minvcg.C:238-252
      const double b = ms->b, bp = ms->bp, a = ms->a;
      ms->bs[0] = b;
      ms->iz = 1 - ms->iz;
      const int iz = ms->iz;
      for (int s = 1; s < n; s++) {
        if (ms->conv[s]) continue;
        double zt = ms->z[1 - iz][s] * ms->z[iz][s] * bp /
                    (b * a * (ms->z[iz][s] - ms->z[1 - iz][s]) +
                     ms->z[iz][s] * bp * (1 - b * (ms->mass[s] - ms->mass[0])));
        ms->bs[s] = b * zt / ms->z[1 - iz][s];
        ms->z[iz][s] = zt;
      }
    }
    st->alpha = -ms->b;  // r += b A p is r -= alpha A p
    return;
  }
  // RED_MS_RR: c = |r|^2 and per-shift convergence (minvcg.C:255-304)
  const double c = sum[0];
  ms->c = c;
  if (!isfinite(c)) { st->done = ST_NONFINITE; return; }
  for (int s = 0; s < n; s++) ms->conv_prev[s] = ms->conv[s];
  if (ms->first) {
    ms->first = 0;
    ms->conv_all = (c < ms->rsd_sq[0]) ? 1 : 0;
  } else {
    ms->k += 1;
    const int iz = ms->iz;
    for (int s = 0; s < n; s++) {
      if (ms->conv[s]) continue;
      double css = c * ms->z[iz][s] * ms->z[iz][s];
      if (css < ms->rsd_sq[s]) {
        ms->conv[s] = 1;
        ms->rsd_out[s] = css;
        ms->conv_iter[s] = ms->k;
      }
    }
    int all = ms->conv[0];
    if (all)
      for (int s = 0; s < n; s++)
        if (!ms->conv[s]) all = 0;
    ms->conv_all = all;
  }
  if (ms->conv_all) st->done = ST_CONVERGED;
  else if (ms->k >= ms->max_iter) st->done = ST_MAX_ITER;
  // coefficients of the next direction update (minvcg.C:204-225)
  ms->a = c / ms->cp;
  const int iz = ms->iz;
  for (int s = 1; s < n; s++)
    if (!ms->conv[s]) ms->as[s] = ms->a * (ms->z[iz][s] * ms->bs[s]) / (ms->z[1 - iz][s] * ms->b);
  ms->cp = c;
}

__device__ __forceinline__ bool finite_d(double x) { return isfinite(x); }

__device__ inline void finalize_scalars(SolverScalars *st, int op, const double *sum) {
  for (int k = 0; k < 4; k++) st->sum[k] = sum[k];
  switch (op) {
    case RED_PAP: {
      double d = sum[0] + st->shift * sum[1];
      st->d = d;
      if (!finite_d(d)) { st->done = ST_NONFINITE; break; }
      if (d == 0.0) { st->done = ST_BREAKDOWN; break; }
      st->alpha = st->rr / d;
      break;
    }
    case RED_CG_RR: {
      double rr = sum[0];
      st->iter += 1;
      st->rr_prev = st->rr;
      st->rr = rr;
      if (!finite_d(rr)) { st->done = ST_NONFINITE; break; }
      if (st->delta2 > 0.0) {
        // mixed precision: ask for a reliable update when the iterated
        // residual has dropped by delta since the last one, or claims
        // convergence; the true residual then decides.
        if (rr > st->rr_max) st->rr_max = rr;
        if (rr <= st->stop || rr < st->delta2 * st->rr_max) {
          st->reliable = 1;
          break;
        }
      } else if (rr <= st->stop) {
        st->done = ST_CONVERGED;
        break;
      }
      if (st->iter >= st->max_iter) { st->done = ST_MAX_ITER; break; }
      st->beta = rr / st->rr_prev;
      break;
    }
    case RED_RELIABLE: {
      double rr = sum[0];
      st->n_reliable += 1;
      st->reliable = 0;
      st->rr = rr;
      st->rr_max = rr;
      if (!finite_d(rr)) { st->done = ST_NONFINITE; break; }
      if (rr <= st->stop) { st->done = ST_CONVERGED; break; }
      if (st->iter >= st->max_iter) { st->done = ST_MAX_ITER; break; }
      st->beta = rr / st->rr_prev;
      break;
    }
    case RED_INIT: {
      st->rr = sum[0];
      st->rr_max = sum[0];
      if (!finite_d(sum[0])) st->done = ST_NONFINITE;
      else if (sum[0] <= st->stop || st->max_iter <= 0) st->done = ST_CONVERGED;
      break;
    }
    case RED_MS_PAP:
    case RED_MS_RR:
      finalize_multishift(st, op, sum);
      break;
    default:
      break;
  }
}

template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
}

// Global reductions are two-step and deterministic: every block of the
// reducing kernel writes its own NV partial sums (block_partial), and a
// following finalize_kernel sums one solve's partials in a fixed order and
// updates its scalars (finalize_scalars).  No block waits on another, no
// atomics: the order of the additions never depends on scheduling.

// Sum NV values over the block; thread 0 writes them as partial number blk of
// solve `solve` (partials hold NV * nblk doubles per solve).  Must be called
// by every thread of the block.
template <int NV>
__device__ void block_partial(double (&v)[NV], double *partials, unsigned solve, unsigned blk, unsigned nblk) {
  __shared__ double sm[32][NV];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  const int lane = tid & 31, warp = tid >> 5, nwarp = (nthr + 31) >> 5;
  warp_sum(v);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) sm[warp][k] = v[k];
  __syncthreads();
  if (tid == 0) {
    double *part = partials + ((size_t)solve * nblk + blk) * NV;
    for (int k = 0; k < NV; k++) {
      double s = 0.0;
      for (int w = 0; w < nwarp; w++) s += sm[w][k];
      part[k] = s;
    }
  }
}

// The common case: one solve per blockIdx.z, all its blocks in x and y.
template <int NV>
__device__ void block_partial(double (&v)[NV], double *partials) {
  block_partial<NV>(v, partials, blockIdx.z, blockIdx.x + gridDim.x * blockIdx.y, gridDim.x * gridDim.y);
}

constexpr int FINALIZE_THREADS = 1024;

// One block per solve: sum its nblk partials (thread-strided, then the warp
// and block trees, always in the same order) and finalize its scalars.  The
// gate is the one the reducing kernel had, so a solve it skipped is skipped
// here too.
template <int NV>
__global__ void __launch_bounds__(FINALIZE_THREADS)
    finalize_kernel(const double *partials, SolverScalars *st, int op, unsigned nblk, int gate) {
  const unsigned solve = blockIdx.x;
  if (gate == 1 && st[solve].done) return;                              // GATE_RUNNING
  if (gate == 2 && (st[solve].done || !st[solve].reliable)) return;     // GATE_RELIABLE
  __shared__ double sm[FINALIZE_THREADS / 32][NV];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double *part = partials + (size_t)solve * nblk * NV;
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) acc[k] = 0.0;
  // eight independent loads in flight per thread (the sum order stays fixed)
  constexpr int U = 8;
  unsigned b = tid;
  for (; b + (U - 1) * FINALIZE_THREADS < nblk; b += U * FINALIZE_THREADS) {
    double v[U][NV];
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int k = 0; k < NV; k++) v[u][k] = part[(size_t)(b + u * FINALIZE_THREADS) * NV + k];
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int k = 0; k < NV; k++) acc[k] += v[u][k];
  }
  for (; b < nblk; b += FINALIZE_THREADS)
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] += part[(size_t)b * NV + k];
  warp_sum(acc);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) sm[warp][k] = acc[k];
  __syncthreads();
  if (tid == 0) {
    double tot[4] = {0, 0, 0, 0};
    for (int k = 0; k < NV; k++)
      for (int w = 0; w < FINALIZE_THREADS / 32; w++) tot[k] += sm[w][k];
    finalize_scalars(&st[solve], op, tot);
  }
}

}  // namespace cpsgpu
