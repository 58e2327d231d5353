// The Ls x Ls chirality mixing (Mobius M5^-1 and the other s-local
// matrices, zmobius_m5inv.C:247-396 as a dense matrix) on the tensor cores,
// for FP16 storage with per-site norms: per block of TC_TS sites and both
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
// Shared memory per block:
//   xs [t][column] FP16, column = site * 24 + real: each 16-byte group of a
//      site's stored spinor lands as one 16-byte store, and ldmatrix.trans
//      reads the B fragments (k = t) straight from the rows; rows are padded
//      to 392 halves (784 B) so the eight row addresses of an 8 x 8 matrix
//      fall in distinct bank groups;
//   ys [s][column] FP32, the products, read back per (slice, site) for the
//      re-normalised FP16 store.
// An 8-column tile holds reals 8g .. 8g+7 of one site: g = 0 is chirality 0,
// g = 2 chirality 1, and g = 1 straddles both (reals 8-11 | 12-15), so its
// tile is multiplied by both matrices and each thread keeps the product of
// its own columns' chirality.
#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

namespace {

constexpr int TC_TS = 16;                 // sites per block
constexpr int TC_COLS = 24 * TC_TS;       // 384 columns
constexpr int TC_XS = TC_COLS + 8;        // halves per xs row
constexpr int TC_YS = TC_COLS + 8;        // floats per ys row
constexpr int TC_THREADS = 128;

__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// four 8 x 8 FP16 matrices from shared memory, transposed: thread T supplies
// the address of row T % 8 of matrix T / 8
__device__ __forceinline__ void ldmatrix_x4_trans(unsigned (&r)[4], const __half *row) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(row);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
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

// The A fragments (m16n8k16, row-major A = M[s][t]) of both chiralities,
// high and low FP16 parts, for every lane: frag[((chi * 2 + part) * 32 + lane) * 4 + e].
// One warp, once per application (the matrices are the operator's).
__global__ void mix_tc_frag_kernel(const double *mix, int ls, unsigned *frag) {
  const int lane = threadIdx.x, g = lane >> 2, q = lane & 3;
  for (int chi = 0; chi < 2; chi++)
    for (int part = 0; part < 2; part++) {
      unsigned *f = frag + ((chi * 2 + part) * 32 + lane) * 4;
      f[0] = pack_h2(mel(mix, ls, chi, g, 2 * q, part), mel(mix, ls, chi, g, 2 * q + 1, part));
      f[1] = pack_h2(mel(mix, ls, chi, g + 8, 2 * q, part), mel(mix, ls, chi, g + 8, 2 * q + 1, part));
      f[2] = pack_h2(mel(mix, ls, chi, g, 2 * q + 8, part), mel(mix, ls, chi, g, 2 * q + 9, part));
      f[3] = pack_h2(mel(mix, ls, chi, g + 8, 2 * q + 8, part), mel(mix, ls, chi, g + 8, 2 * q + 9, part));
    }
}

constexpr int TC_LOADS = (16 * 3 * TC_TS + TC_THREADS - 1) / TC_THREADS;  // X groups per thread, at most

__global__ void __launch_bounds__(TC_THREADS) mix_tc_kernel(SpinorView in, SpinorView out, const unsigned *frag,
                                                            int ls, const SolverScalars *st, int gate) {
  if (gate == GATE_RUNNING && st[blockIdx.z].done) return;
  if (gate == GATE_RELIABLE && (st[blockIdx.z].done || !st[blockIdx.z].reliable)) return;
  __shared__ __align__(16) __half xs[16 * TC_XS];
  __shared__ __align__(16) float ys[16 * TC_YS];
  __shared__ float nrm[16 * TC_TS];
  __shared__ float nmax[TC_TS];
  const int tid = threadIdx.x;
  const long i0 = (long)blockIdx.x * TC_TS;
  const long rhs = blockIdx.z;
  const int nsite = (int)min((long)TC_TS, in.vh - i0);
  // norms of every slice of the block's sites; X zeroed (padding rows t >= ls
  // and the columns of absent sites stay zero)
  for (int k = tid; k < 16 * TC_TS; k += TC_THREADS) {
    const int t = k / TC_TS, site = k % TC_TS;
    nrm[k] = (t < ls && site < nsite) ? __ldg(in.norm + (rhs * ls + t) * in.vh + i0 + site) : 0.f;
  }
  for (int k = tid; k < 16 * TC_XS / 8; k += TC_THREADS) reinterpret_cast<uint4 *>(xs)[k] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  if (tid < TC_TS) {
    float m = 0.f;
    for (int t = 0; t < ls; t++) m = fmaxf(m, nrm[t * TC_TS + tid]);
    nmax[tid] = m;
  }
  __syncthreads();
  // X: group g (reals 8g .. 8g+7) of slice t and site, rescaled to the
  // site's largest norm, one 16-byte store; every load of the thread is
  // issued before the first is used
  const uint4 *src = reinterpret_cast<const uint4 *>(in.data);
  uint4 qv[TC_LOADS];
#pragma unroll
  for (int j = 0; j < TC_LOADS; j++) {
    const int k = tid + j * TC_THREADS;
    const int site = k % TC_TS, g = (k / TC_TS) % 3, t = k / (3 * TC_TS);
    qv[j] = (t < ls && site < nsite) ? __ldg(src + ((rhs * ls + t) * 3 + g) * in.vh + i0 + site)
                                     : make_uint4(0, 0, 0, 0);
  }
  unsigned A[2][2][4];  // [chi][hi/lo][frag] of this lane
  const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int cp = 0; cp < 4; cp++) {
    const uint4 f = __ldg(reinterpret_cast<const uint4 *>(frag) + cp * 32 + lane);
    A[cp >> 1][cp & 1][0] = f.x;
    A[cp >> 1][cp & 1][1] = f.y;
    A[cp >> 1][cp & 1][2] = f.z;
    A[cp >> 1][cp & 1][3] = f.w;
  }
#pragma unroll
  for (int j = 0; j < TC_LOADS; j++) {
    const int k = tid + j * TC_THREADS;
    const int site = k % TC_TS, gg = (k / TC_TS) % 3, t = k / (3 * TC_TS);
    if (t >= ls || site >= nsite) continue;
    const float r = nmax[site] > 0.f ? nrm[t * TC_TS + site] / nmax[site] : 0.f;
    const __half2 *h = reinterpret_cast<const __half2 *>(&qv[j]);
    uint4 o;
    unsigned *op = reinterpret_cast<unsigned *>(&o);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float2 f = __half22float2(h[e]);
      op[e] = pack_h2(f.x * r, f.y * r);
    }
    *reinterpret_cast<uint4 *>(xs + t * TC_XS + site * 24 + 8 * gg) = o;
  }
  __syncthreads();
  // MMAs: warp w takes the column-tile pairs w, w + 4, ... (16 columns each)
  const int mrow = lane & 7, mat = lane >> 3;  // this thread's ldmatrix row and matrix
  for (int pair = warp; pair < TC_COLS / 16; pair += TC_THREADS / 32) {
    const int n0 = pair * 16;
    unsigned b[4];
    // matrices: (k 0-7, n0..), (k 8-15, n0..), (k 0-7, n0+8..), (k 8-15, n0+8..)
    ldmatrix_x4_trans(b, xs + (mrow + 8 * (mat & 1)) * TC_XS + n0 + 8 * (mat >> 1));
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int nt = n0 + 8 * half;          // 8-column tile: reals 8 gt .. of one site
      const int gt = (nt / 8) % 3;
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      if (gt != 1) {
        const int chi = gt >> 1;
        mma16816(d, A[chi][0], b[2 * half], b[2 * half + 1]);
        mma16816(d, A[chi][1], b[2 * half], b[2 * half + 1]);
      } else {
        // columns 2q, 2q+1 are reals 8 + 2q, 9 + 2q: chirality 0 for q < 2
        float d1[4] = {0.f, 0.f, 0.f, 0.f};
        mma16816(d, A[0][0], b[2 * half], b[2 * half + 1]);
        mma16816(d, A[0][1], b[2 * half], b[2 * half + 1]);
        mma16816(d1, A[1][0], b[2 * half], b[2 * half + 1]);
        mma16816(d1, A[1][1], b[2 * half], b[2 * half + 1]);
        if (q >= 2) {
#pragma unroll
          for (int e = 0; e < 4; e++) d[e] = d1[e];
        }
      }
      // d: rows (output slices) g and g + 8, columns nt + 2q, nt + 2q + 1
      *reinterpret_cast<float2 *>(ys + g * TC_YS + nt + 2 * q) = make_float2(d[0], d[1]);
      *reinterpret_cast<float2 *>(ys + (g + 8) * TC_YS + nt + 2 * q) = make_float2(d[2], d[3]);
    }
  }
  __syncthreads();
  // output: thread per (slice, site), re-normalised FP16 storage
  for (int k = tid; k < ls * TC_TS; k += TC_THREADS) {
    const int s = k / TC_TS, site = k % TC_TS;
    if (site >= nsite) continue;
    float v[24];
    const float4 *row = reinterpret_cast<const float4 *>(ys + s * TC_YS + site * 24);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      const float4 f = row[c];
      v[4 * c] = f.x * nmax[site];
      v[4 * c + 1] = f.y * nmax[site];
      v[4 * c + 2] = f.z * nmax[site];
      v[4 * c + 3] = f.w * nmax[site];
    }
    SpinorIO<PREC_HALF>::store(out, rhs * ls + s, i0 + site, v);
  }
}

}  // namespace

bool mix_tc_applies(const Dirac &D, int prec) { return prec == PREC_HALF && !D.cplx && D.ls <= 16; }

void launch_mix_tc(const Dirac &D, const double *mix, const SpinorView &in, const SpinorView &out,
                   const SolverScalars *st, int gate) {
  if (!mix_tc_applies(D, PREC_HALF)) throw Error(-2, "tensor-core mixing: FP16 storage, real matrices, Ls <= 16");
  // the fragments of this matrix, then the mixing (same stream: ordered)
  DeviceBuffer &frag = const_cast<Dirac &>(D).mixTcFrag;
  frag.ensure(2 * 2 * 32 * 4 * sizeof(unsigned));
  mix_tc_frag_kernel<<<1, 32, 0, D.lat->stream>>>(mix, D.ls, frag.as<unsigned>());
  CPSGPU_CUDA(cudaGetLastError());
  dim3 grid((unsigned)((in.vh + TC_TS - 1) / TC_TS), 1, in.nrhs);
  mix_tc_kernel<<<grid, TC_THREADS, 0, D.lat->stream>>>(in, out, frag.as<unsigned>(), D.ls, st, gate);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter() += 2;
}

}  // namespace cpsgpu
