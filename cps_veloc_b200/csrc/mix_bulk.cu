// The Ls x Ls chirality mixing (Mobius M5^-1, the s-local chains of MatPc)
// of FP16 fields with the input staged in shared memory by bulk copies.
//
// The register-tiled kernel (mix_reg.cu) loads each input value straight
// into a register, and with 48 accumulators per thread the compiler keeps
// few of those loads in flight: the kernel waits on global memory (DRAM
// ~30% busy).  Here a persistent block walks tiles of 32 sites (all Ls
// slices, both chiralities) with two shared-memory stages: one thread
// issues the next tile's copies (cp.async.bulk, global -> shared, 3 x 512 B
// of half groups and 128 B of norms per slice, completing on an mbarrier)
// while the block computes the current tile from the other stage.  No copy
// uses cluster multicast; every source is this GPU's own memory.
//
// The arithmetic is mix_reg's, operation for operation (each thread: 4
// reals of one site, all Ls output slices, the matrices as a kernel
// parameter, FP16 norms combined through shared memory), so the outputs are
// bit-identical to it.  Every wait on an mbarrier is bounded in time (one
// second by the global timer, each try_wait suspending at most ~1 us): a
// wait that runs out sets g_mix_bulk_err, writes NaN to the tile (a solver
// on it ends NONFINITE) and the block stops after waiting, again bounded,
// for its copies in flight.
#include <cstdint>

#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

__device__ int g_mix_bulk_err;  // nonzero once a bounded wait ran out

namespace {

// the matrices transposed, [t][s]: output slices s, s + 1 of input slice t
// are one 8-byte operand of a packed multiply-add
template <int LS> struct __align__(8) MixMatF {
  float up[LS * LS], dn[LS * LS];
};

constexpr int TS = 32;  // sites per tile (threadIdx.x)
constexpr int NB = 6;   // blocks of 4 reals per site (threadIdx.y)
constexpr unsigned long long WAIT_NS = 1000000000ull;  // a wait gives up after one second
constexpr unsigned SUSPEND_NS = 1000;                    // each try_wait suspends at most ~1 us

template <int LS> struct Tile {
  static constexpr int DATA = LS * 3 * TS * 16;  // [t][group][site] 16-byte groups
  static constexpr int NORM = LS * TS * 4;       // [t][site]
  static constexpr int STAGE = DATA + NORM;
};

__device__ __forceinline__ uint32_t sptr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sptr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sptr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(sptr(bar)), "r"(parity), "r"(SUSPEND_NS)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded in time: true once the phase of this parity has completed, false
// after WAIT_NS
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > WAIT_NS) return false;
  }
}

// global -> shared, completing on bar; both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(sptr(dst)),
      "l"(src), "r"(bytes), "r"(sptr(bar))
      : "memory");
}

__device__ __forceinline__ bool tile_live(long rhs, const SolverScalars *st, int gate) {
  if (gate == GATE_RUNNING) return !st[rhs].done;
  if (gate == GATE_RELIABLE) return !st[rhs].done && st[rhs].reliable;
  return true;
}

// the next tile of this block after q (its tiles: blockIdx.x + k gridDim.x)
// that the gate lets through, or ntiles
__device__ __forceinline__ long next_tile(long q, long ntiles, long per_rhs, const SolverScalars *st, int gate) {
  for (q += gridDim.x; q < ntiles; q += gridDim.x)
    if (tile_live(q / per_rhs, st, gate)) return q;
  return ntiles;
}

// acc(s) += M[s][t] x_t over t ascending, x_t from stage buf; acc[s / 2][k]
// packs slices s, s + 1 (each lane the scalar fmaf of the same operands)
template <int LS>
__device__ __forceinline__ void mix_tile(const unsigned char *buf, int cb, int x, const float (&MT)[LS * LS],
                                         float2 (&acc)[LS / 2][4]) {
#pragma unroll
  for (int t = 0; t < LS; t++) {
    const uint2 qv = *reinterpret_cast<const uint2 *>(buf + ((t * 3 + (cb >> 1)) * TS + x) * 16 + (cb & 1) * 8);
    const float sc = *reinterpret_cast<const float *>(buf + Tile<LS>::DATA + (t * TS + x) * 4);
    const __half2 *h = reinterpret_cast<const __half2 *>(&qv);
    const float2 a = __half22float2(h[0]), c = __half22float2(h[1]);
    const float xv[4] = {a.x * sc, a.y * sc, c.x * sc, c.y * sc};
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      const float2 xx = make_float2(xv[kk], xv[kk]);
#pragma unroll
      for (int s = 0; s < LS / 2; s++)
        acc[s][kk] = __ffma2_rn(*reinterpret_cast<const float2 *>(&MT[t * LS + 2 * s]), xx, acc[s][kk]);
    }
  }
}

template <int LS>
__global__ void __launch_bounds__(TS * NB) mix_bulk_kernel(SpinorView in, SpinorView out, const MixMatF<LS> m,
                                                          const SolverScalars *st, int gate) {
  using T = Tile<LS>;
  extern __shared__ __align__(128) unsigned char stage_mem[];  // [2][STAGE]
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ float pmax[LS][NB][TS];
  __shared__ int abort_flag;
  const int x = threadIdx.x, cb = threadIdx.y;
  const bool producer = (x == 0 && cb == 0);
  const long per_rhs = in.vh / TS;
  const long ntiles = per_rhs * in.nrhs;

  auto issue = [&](long q, int b) {
    const long rhs = q / per_rhs, site0 = (q % per_rhs) * TS;
    unsigned char *dst = stage_mem + b * T::STAGE;
    mbar_expect_tx(&bar[b], T::STAGE);
    const uint4 *src = reinterpret_cast<const uint4 *>(in.data);
    for (int t = 0; t < LS; t++) {
      const long sl = rhs * LS + t;
#pragma unroll
      for (int g = 0; g < 3; g++)
        bulk_copy(dst + (t * 3 + g) * TS * 16, src + (sl * 3 + g) * in.vh + site0, TS * 16, &bar[b]);
      bulk_copy(dst + T::DATA + t * TS * 4, in.norm + sl * in.vh + site0, TS * 4, &bar[b]);
    }
  };

  if (producer) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    abort_flag = 0;
  }
  __syncthreads();

  long q = blockIdx.x;
  if (q < ntiles && !tile_live(q / per_rhs, st, gate)) q = next_tile(q, ntiles, per_rhs, st, gate);
  // producer: copies issued into a stage and not yet waited for, with the
  // parity of the phase they complete
  // (bit b of each mask: stage b)
  unsigned pending = 0, pend_par = 0;
  if (producer && q < ntiles) {
    issue(q, 0);
    pending = 1u;
  }
  for (int k = 0; q < ntiles; k++) {
    const int b = k & 1;
    const unsigned parity = (unsigned)((k >> 1) & 1);
    const long qn = next_tile(q, ntiles, per_rhs, st, gate);
    if (producer && qn < ntiles) {
      issue(qn, b ^ 1);  // that stage's readers finished at the end of the previous round
      pending |= 1u << (b ^ 1);
      pend_par = (pend_par & ~(1u << (b ^ 1))) | ((unsigned)(((k + 1) >> 1) & 1) << (b ^ 1));
    }
    const bool ok = mbar_wait(&bar[b], parity);
    if (producer && ok) pending &= ~(1u << b);
    const long rhs = q / per_rhs, site0 = (q % per_rhs) * TS;
    const long i = site0 + x;
    const unsigned char *buf = stage_mem + b * T::STAGE;
    // mix_reg's arithmetic: x_t = the 4 halves of this block times the
    // site's norm; out(s) = sum_t M_chi[s][t] x_t, t ascending
    float2 acc2[LS / 2][4];
#pragma unroll
    for (int s = 0; s < LS / 2; s++)
#pragma unroll
      for (int kk = 0; kk < 4; kk++) acc2[s][kk] = make_float2(0.f, 0.f);
    if (ok) {
      // warp-uniform branch (a warp is one cb): the matrix operands stay
      // compile-time offsets into the parameter block
      if (cb < NB / 2) mix_tile<LS>(buf, cb, x, m.up, acc2);
      else mix_tile<LS>(buf, cb, x, m.dn, acc2);
    } else {
      atomicExch(&g_mix_bulk_err, 1);
      abort_flag = 1;
    }
    auto acc = [&](int s, int kk) { return (s & 1) ? acc2[s >> 1][kk].y : acc2[s >> 1][kk].x; };
#pragma unroll
    for (int s = 0; s < LS; s++) {
      float mx = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; kk++) mx = fmaxf(mx, fabsf(acc(s, kk)));
      pmax[s][cb][x] = mx;
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < LS; s++) {
      float mx = 0.f;
#pragma unroll
      for (int bb = 0; bb < NB; bb++) mx = fmaxf(mx, pmax[s][bb][x]);
      const float inv = (mx > 0.f) ? 1.0f / mx : 0.f;
      uint2 qo;
      __half2 *h = reinterpret_cast<__half2 *>(&qo);
      h[0] = __floats2half2_rn(acc(s, 0) * inv, acc(s, 1) * inv);
      h[1] = __floats2half2_rn(acc(s, 2) * inv, acc(s, 3) * inv);
      if (!ok) qo = make_uint2(0x7e007e00u, 0x7e007e00u);  // FP16 NaN: a run-out wait poisons the tile
      const long sl = rhs * LS + s;
      reinterpret_cast<uint2 *>(out.data)[((sl * 3 + (cb >> 1)) * out.vh + i) * 2 + (cb & 1)] = qo;
      if (cb == 0) out.norm[sl * out.vh + i] = ok ? mx : __int_as_float(0x7fc00000);
    }
    __syncthreads();  // the stage and pmax are free again
    if (abort_flag) break;
    q = qn;
  }
  if (producer) {
    // after a wait ran out: the block's copies still in flight land before it exits
    for (int bb = 0; bb < 2; bb++)
      if (pending & (1u << bb)) mbar_wait(&bar[bb], (pend_par >> bb) & 1u);
  }
}

template <int LS>
void launch_ls(const Dirac &D, const std::vector<double> &h, const SpinorView &in, const SpinorView &out,
               const SolverScalars *st, int gate) {
  MixMatF<LS> m;  // transposed: m.up[t * LS + s] = M_up[s][t]
  for (int s = 0; s < LS; s++)
    for (int t = 0; t < LS; t++) {
      m.up[t * LS + s] = float(h[s * LS + t]);
      m.dn[t * LS + s] = float(h[LS * LS + s * LS + t]);
    }
  const int smem = 2 * Tile<LS>::STAGE;
  // the shared-memory attribute and the occupancy belong to one device
  constexpr int MAXDEV = 64;
  static int blocks_per_sm[MAXDEV] = {}, sms[MAXDEV] = {};
  const int dev = D.lat->device;
  if (dev < 0 || dev >= MAXDEV) throw Error(-1, "device index out of range");
  if (!blocks_per_sm[dev]) {
    CPSGPU_CUDA(cudaFuncSetAttribute(mix_bulk_kernel<LS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CPSGPU_CUDA(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev));
    int b = 0;
    CPSGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, mix_bulk_kernel<LS>, TS * NB, smem));
    blocks_per_sm[dev] = b < 1 ? 1 : b;
  }
  const long ntiles = (in.vh / TS) * in.nrhs;
  const long nblocks = std::min<long>(ntiles, (long)blocks_per_sm[dev] * sms[dev]);
  mix_bulk_kernel<LS><<<(unsigned)nblocks, dim3(TS, NB), smem, D.lat->stream>>>(in, out, m, st, gate);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

}  // namespace

bool launch_mix_bulk(const Dirac &D, int prec, const double *mix, const SpinorView &in, const SpinorView &out,
                     const SolverScalars *st, int gate) {
  if (prec != PREC_HALF || D.cplx) return false;
  const auto it = D.mix_host.find(mix);
  if (it == D.mix_host.end() || it->second.size() != 2 * (size_t)D.ls * D.ls) return false;
  if (in.ls != D.ls || in.vh % TS != 0 || in.vh != out.vh) return false;
  // bulk copies need 16-byte aligned sources; every row of norms starts on a multiple of 128 bytes
  if (((uintptr_t)in.data | (uintptr_t)in.norm) % 16 != 0) return false;
  switch (D.ls) {
    case 8: launch_ls<8>(D, it->second, in, out, st, gate); return true;
    case 10: launch_ls<10>(D, it->second, in, out, st, gate); return true;
    case 12: launch_ls<12>(D, it->second, in, out, st, gate); return true;
    case 16: launch_ls<16>(D, it->second, in, out, st, gate); return true;
    default: return false;
  }
}

// the flag of the current device, cleared by the read
int mix_bulk_error() {
  int e = 0;
  CPSGPU_CUDA(cudaMemcpyFromSymbol(&e, g_mix_bulk_err, sizeof(int)));
  if (e) {
    const int zero = 0;
    CPSGPU_CUDA(cudaMemcpyToSymbol(g_mix_bulk_err, &zero, sizeof(int)));
  }
  return e;
}

}  // namespace cpsgpu
