// The Ls x Ls chirality mixing (Mobius M5^-1 and the other s-local
// matrices, zmobius_m5inv.C:247-396 as a dense matrix) on the tensor cores,
// for FP16 storage with per-site norms: per block of TS sites and both
// chiralities,
//
//     Y_chi (Ls x 12 TS) = M_chi (Ls x Ls) X_chi (Ls x 12 TS)
//
// with mma.sync m16n8k16 (FP16 operands, FP32 accumulation).  M is split
// into FP16 high and low parts (two MMAs, about 22 significant bits), so the
// matrix loses nothing against the FP32 arithmetic of the CUDA-core kernel.
// X holds the stored FP16 values of the site times norm_t / max_t norm_t,
// rounded to FP16 once more (values in [-1, 1]); the result is rescaled by
// max_t norm_t and re-normalised per output slice.  Real matrices, Ls <= 16.
//
// Shared memory per block: the X tile [column][t] in FP16 (column = chirality,
// site, 12 reals; t padded to 24 halves so the B-fragment loads hit 32
// distinct banks) and the FP32 result [column][16].
#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

namespace {

constexpr int TC_TS = 16;           // sites per block
constexpr int TC_KS = 24;           // halves per X column (t padded)
constexpr int TC_COLS = 2 * 12 * TC_TS;  // 384 columns: [chi][site][12]
constexpr int TC_THREADS = 128;

__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned pack_h2(float lo, float hi) {
  __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<unsigned *>(&h);
}

// M(row, col) of chirality chi from the packed [2][ls][ls] FP64 matrices,
// zero outside ls x ls; part 0: FP16 high part, 1: the low remainder
__device__ __forceinline__ float mel(const double *mix, int ls, int chi, int row, int col, int part) {
  if (row >= ls || col >= ls) return 0.f;
  const double m = mix[(size_t)chi * ls * ls + (size_t)row * ls + col];
  const float hi = __half2float(__float2half_rn((float)m));
  return part ? (float)(m - (double)hi) : hi;
}

__global__ void __launch_bounds__(TC_THREADS) mix_tc_kernel(SpinorView in, SpinorView out, const double *mix, int ls,
                                                            const SolverScalars *st, int gate) {
  if (gate == GATE_RUNNING && st[blockIdx.z].done) return;
  if (gate == GATE_RELIABLE && (st[blockIdx.z].done || !st[blockIdx.z].reliable)) return;
  __shared__ __align__(16) __half xs[TC_COLS * TC_KS];
  __shared__ float ys[TC_COLS * 16];
  __shared__ float nrm[16 * TC_TS];
  __shared__ float nmax[TC_TS];
  const int tid = threadIdx.x;
  const long i0 = (long)blockIdx.x * TC_TS;
  const long rhs = blockIdx.z;
  const int nsite = (int)min((long)TC_TS, in.vh - i0);
  // norms of every slice of the block's sites, and their maximum per site
  for (int k = tid; k < 16 * TC_TS; k += TC_THREADS) {
    const int t = k / TC_TS, site = k % TC_TS;
    nrm[k] = (t < ls && site < nsite) ? __ldg(in.norm + (rhs * ls + t) * in.vh + i0 + site) : 0.f;
  }
  // zero padding of X (t >= ls)
  for (int k = tid; k < TC_COLS * TC_KS / 2; k += TC_THREADS) reinterpret_cast<unsigned *>(xs)[k] = 0u;
  __syncthreads();
  if (tid < TC_TS) {
    float m = 0.f;
    for (int t = 0; t < ls; t++) m = fmaxf(m, nrm[t * TC_TS + tid]);
    nmax[tid] = m;
  }
  __syncthreads();
  // X tile: group g (8 halves: reals 8g .. 8g+7) of slice t, site
  const uint4 *src = reinterpret_cast<const uint4 *>(in.data);
  for (int k = tid; k < ls * 3 * TC_TS; k += TC_THREADS) {
    const int site = k % TC_TS, g = (k / TC_TS) % 3, t = k / (3 * TC_TS);
    if (site >= nsite) continue;
    const uint4 q = __ldg(src + ((rhs * ls + t) * 3 + g) * in.vh + i0 + site);
    const float r = nmax[site] > 0.f ? nrm[t * TC_TS + site] / nmax[site] : 0.f;
    const __half2 *h = reinterpret_cast<const __half2 *>(&q);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float2 f = __half22float2(h[e]);
#pragma unroll
      for (int w = 0; w < 2; w++) {
        const int real = 8 * g + 2 * e + w, chi = real / 12, c = real % 12;
        const int col = (chi * TC_TS + site) * 12 + c;
        xs[col * TC_KS + t] = __float2half_rn((w ? f.y : f.x) * r);
      }
    }
  }
  __syncthreads();
  // MMAs: warp w takes column tiles w, w + 4, ...; A fragments per chirality
  const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
  unsigned A[2][2][4];  // [chi][hi/lo][frag]
#pragma unroll
  for (int chi = 0; chi < 2; chi++)
#pragma unroll
    for (int part = 0; part < 2; part++) {
      A[chi][part][0] = pack_h2(mel(mix, ls, chi, g, 2 * q, part), mel(mix, ls, chi, g, 2 * q + 1, part));
      A[chi][part][1] = pack_h2(mel(mix, ls, chi, g + 8, 2 * q, part), mel(mix, ls, chi, g + 8, 2 * q + 1, part));
      A[chi][part][2] = pack_h2(mel(mix, ls, chi, g, 2 * q + 8, part), mel(mix, ls, chi, g, 2 * q + 9, part));
      A[chi][part][3] =
          pack_h2(mel(mix, ls, chi, g + 8, 2 * q + 8, part), mel(mix, ls, chi, g + 8, 2 * q + 9, part));
    }
  const unsigned *xw = reinterpret_cast<const unsigned *>(xs);
  for (int tile = warp; tile < TC_COLS / 8; tile += TC_THREADS / 32) {
    const int n0 = tile * 8, chi = n0 / (12 * TC_TS);
    const unsigned b0 = xw[((n0 + g) * TC_KS + 2 * q) / 2];
    const unsigned b1 = xw[((n0 + g) * TC_KS + 2 * q + 8) / 2];
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    mma16816(d, A[chi][0], b0, b1);
    mma16816(d, A[chi][1], b0, b1);
    // d: rows (output slices) g and g + 8, columns n0 + 2q, n0 + 2q + 1
    ys[(n0 + 2 * q) * 16 + g] = d[0];
    ys[(n0 + 2 * q + 1) * 16 + g] = d[1];
    ys[(n0 + 2 * q) * 16 + g + 8] = d[2];
    ys[(n0 + 2 * q + 1) * 16 + g + 8] = d[3];
  }
  __syncthreads();
  // output: thread per (slice, site), re-normalised FP16 storage
  for (int k = tid; k < ls * TC_TS; k += TC_THREADS) {
    const int s = k / TC_TS, site = k % TC_TS;
    if (site >= nsite) continue;
    float v[24];
#pragma unroll
    for (int real = 0; real < 24; real++) {
      const int chi = real / 12, c = real % 12;
      v[real] = ys[((chi * TC_TS + site) * 12 + c) * 16 + s] * nmax[site];
    }
    SpinorIO<PREC_HALF>::store(out, rhs * ls + s, i0 + site, v);
  }
}

}  // namespace

bool mix_tc_applies(const Dirac &D, int prec) { return prec == PREC_HALF && !D.cplx && D.ls <= 16; }

void launch_mix_tc(const Dirac &D, const double *mix, const SpinorView &in, const SpinorView &out,
                   const SolverScalars *st, int gate) {
  if (!mix_tc_applies(D, PREC_HALF)) throw Error(-2, "tensor-core mixing: FP16 storage, real matrices, Ls <= 16");
  dim3 grid((unsigned)((in.vh + TC_TS - 1) / TC_TS), 1, in.nrhs);
  mix_tc_kernel<<<grid, TC_THREADS, 0, D.lat->stream>>>(in, out, mix, D.ls, st, gate);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

}  // namespace cpsgpu
