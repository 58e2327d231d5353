// The Ls x Ls chirality mixing (Mobius M5^-1, the s-local chains of MatPc)
// with the matrix in registers' reach: the two real Ls x Ls matrices are a
// kernel parameter (the constant bank), Ls is a template argument, and every
// thread computes all Ls output slices of one block of reals of one site,
//
//     out(s, k) = sum_t M_chi(k)[s][t] in(t, k),   k in the thread's block,
//
// so each input value is loaded once from HBM into a register and used for
// Ls multiply-adds whose matrix operand comes from the constant bank (no
// shared-memory traffic; the kernel it replaces read one shared-memory word
// per multiply-add).  Blocks of reals never straddle the chiralities: 4 reals
// (one float4 group, or half an FP16 group).  FP32 and FP16 fields only: the
// FP64 fields keep the shared-memory kernel, which is faster for them.  FP16
// output needs the largest magnitude of all 24 reals of a site and slice: the
// six threads of a site combine their partial maxima in shared memory.
#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

namespace {

// the two matrices transposed, [t][s], so that the entries of output
// slices s and s + 1 for one input slice t are adjacent (one 8-byte operand
// of a packed multiply-add)
template <int LS, typename T> struct __align__(8) MixMat {
  T up[LS * LS], dn[LS * LS];
};

template <int P> struct RegBlock;
template <> struct RegBlock<PREC_SINGLE> { static constexpr int NR = 4, NB = 6; };   // float4 per block
template <> struct RegBlock<PREC_HALF> { static constexpr int NR = 4, NB = 6; };     // 4 of the 8 halves of a group

constexpr int REG_SITES = 32;  // sites per block: threadIdx.x; the reals block is threadIdx.y

// load block cb (NR reals) of site i, slice sl
template <int P>
__device__ __forceinline__ void load_block(const SpinorView &f, long sl, long i, int cb, float (&v)[4]) {
  if constexpr (P == PREC_SINGLE) {
    const float4 q = __ldg(reinterpret_cast<const float4 *>(f.data) + (sl * 6 + cb) * f.vh + i);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  } else {
    // FP16: group cb / 2 holds 8 halves; this block is its half cb % 2
    const uint2 q = __ldg(reinterpret_cast<const uint2 *>(f.data) + ((sl * 3 + (cb >> 1)) * f.vh + i) * 2 + (cb & 1));
    const float s = __ldg(f.norm + sl * f.vh + i);
    const __half2 *h = reinterpret_cast<const __half2 *>(&q);
    const float2 a = __half22float2(h[0]), b = __half22float2(h[1]);
    v[0] = a.x * s; v[1] = a.y * s; v[2] = b.x * s; v[3] = b.y * s;
  }
}

// out(s) for all s of one block of reals, matrix MT transposed ([t][s]);
// acc[s / 2][k] holds slices s, s + 1 of real k: one packed fused
// multiply-add per pair, each lane the scalar fmaf of the same operands
template <int P, int LS, int NR>
__device__ __forceinline__ void mix_block(const SpinorView &in, long rhs, long i, int cb, const float (&MT)[LS * LS],
                                          float2 (&acc)[LS / 2][NR]) {
#pragma unroll
  for (int s = 0; s < LS / 2; s++)
#pragma unroll
    for (int k = 0; k < NR; k++) acc[s][k] = make_float2(0.f, 0.f);
#pragma unroll
  for (int t = 0; t < LS; t++) {
    float x[NR];
    load_block<P>(in, rhs * LS + t, i, cb, x);
#pragma unroll
    for (int k = 0; k < NR; k++) {
      const float2 xx = make_float2(x[k], x[k]);
#pragma unroll
      for (int s = 0; s < LS / 2; s++)
        acc[s][k] = __ffma2_rn(*reinterpret_cast<const float2 *>(&MT[t * LS + 2 * s]), xx, acc[s][k]);
    }
  }
}

template <int P, int LS>
__global__ void __launch_bounds__(REG_SITES * RegBlock<P>::NB)
    mix_reg_kernel(SpinorView in, SpinorView out, const MixMat<LS, float> m, const SolverScalars *st, int gate) {
  static_assert(LS % 2 == 0, "slices are paired");
  constexpr int NR = RegBlock<P>::NR, NB = RegBlock<P>::NB;
  if (gate == GATE_RUNNING && st[blockIdx.z].done) return;
  if (gate == GATE_RELIABLE && (st[blockIdx.z].done || !st[blockIdx.z].reliable)) return;
  const int cb = threadIdx.y;  // block of reals: the first NB/2 are the upper chirality
  const long i = (long)blockIdx.x * REG_SITES + threadIdx.x;
  const long rhs = blockIdx.z;
  const bool active = i < in.vh;
  float2 acc2[LS / 2][NR];
  // warp-uniform branch (a warp is one cb): the matrix operands stay compile-time offsets
  if (active) {
    if (cb < NB / 2) mix_block<P, LS>(in, rhs, i, cb, m.up, acc2);
    else mix_block<P, LS>(in, rhs, i, cb, m.dn, acc2);
  }
  auto acc = [&](int s, int k) { return (s & 1) ? acc2[s >> 1][k].y : acc2[s >> 1][k].x; };
  if constexpr (P == PREC_SINGLE) {
    if (!active) return;
#pragma unroll
    for (int s = 0; s < LS; s++)
      reinterpret_cast<float4 *>(out.data)[((rhs * LS + s) * 6 + cb) * out.vh + i] =
          make_float4(acc(s, 0), acc(s, 1), acc(s, 2), acc(s, 3));
  } else {
    // FP16: every slice's norm is the largest magnitude over the 6 blocks
    __shared__ float pmax[LS][NB][REG_SITES];
#pragma unroll
    for (int s = 0; s < LS; s++) {
      float mx = 0.f;
#pragma unroll
      for (int k = 0; k < NR; k++) mx = fmaxf(mx, fabsf(active ? acc(s, k) : 0.f));
      pmax[s][cb][threadIdx.x] = mx;
    }
    __syncthreads();
    if (!active) return;
#pragma unroll
    for (int s = 0; s < LS; s++) {
      float mx = 0.f;
#pragma unroll
      for (int b = 0; b < NB; b++) mx = fmaxf(mx, pmax[s][b][threadIdx.x]);
      const float inv = (mx > 0.f) ? 1.0f / mx : 0.f;
      uint2 q;
      __half2 *h = reinterpret_cast<__half2 *>(&q);
      h[0] = __floats2half2_rn(acc(s, 0) * inv, acc(s, 1) * inv);
      h[1] = __floats2half2_rn(acc(s, 2) * inv, acc(s, 3) * inv);
      const long sl = rhs * LS + s;
      reinterpret_cast<uint2 *>(out.data)[((sl * 3 + (cb >> 1)) * out.vh + i) * 2 + (cb & 1)] = q;
      if (cb == 0) out.norm[sl * out.vh + i] = mx;
    }
  }
}

template <int P, int LS>
void launch_ls(const Dirac &D, const std::vector<double> &h, const SpinorView &in, const SpinorView &out,
               const SolverScalars *st, int gate) {
  MixMat<LS, float> m;  // transposed: m.up[t * LS + s] = M_up[s][t]
  for (int s = 0; s < LS; s++)
    for (int t = 0; t < LS; t++) {
      m.up[t * LS + s] = float(h[s * LS + t]);
      m.dn[t * LS + s] = float(h[LS * LS + s * LS + t]);
    }
  const dim3 block(REG_SITES, RegBlock<P>::NB);
  const dim3 grid((unsigned)((in.vh + REG_SITES - 1) / REG_SITES), 1, in.nrhs);
  mix_reg_kernel<P, LS><<<grid, block, 0, D.lat->stream>>>(in, out, m, st, gate);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

template <int P>
bool launch_prec(const Dirac &D, const std::vector<double> &h, const SpinorView &in, const SpinorView &out,
                 const SolverScalars *st, int gate) {
  static_assert(P != PREC_DOUBLE, "FP64 mixings use the shared-memory kernel");
  switch (D.ls) {
    case 8: launch_ls<P, 8>(D, h, in, out, st, gate); return true;
    case 10: launch_ls<P, 10>(D, h, in, out, st, gate); return true;
    case 12: launch_ls<P, 12>(D, h, in, out, st, gate); return true;
    case 16: launch_ls<P, 16>(D, h, in, out, st, gate); return true;
    case 20: launch_ls<P, 20>(D, h, in, out, st, gate); return true;
    case 24: launch_ls<P, 24>(D, h, in, out, st, gate); return true;
    default: return false;
  }
}

}  // namespace

bool launch_mix_reg(const Dirac &D, int prec, const double *mix, const SpinorView &in, const SpinorView &out,
                    const SolverScalars *st, int gate) {
  if (D.cplx) return false;
  const auto it = D.mix_host.find(mix);
  if (it == D.mix_host.end() || it->second.size() != 2 * (size_t)D.ls * D.ls) return false;
  if (in.ls != D.ls) return false;
  // FP64: the shared-memory kernel is the faster (0.467 against 0.504 ms for
  // M5^-1 at 24^3x64, Ls = 12: its loads are already 16-byte double2 groups)
  if (prec == PREC_DOUBLE) return false;
  if (prec == PREC_SINGLE) return launch_prec<PREC_SINGLE>(D, it->second, in, out, st, gate);
  return launch_prec<PREC_HALF>(D, it->second, in, out, st, gate);
}

}  // namespace cpsgpu
