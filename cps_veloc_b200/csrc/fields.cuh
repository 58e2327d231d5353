// Device storage of gauge links and fermion fields, in three precisions.
//
// Layout in HBM (site-SoA, one 16- or 8-byte group per load):
//   fermion field: group g of checkerboard site i in slice sl = rhs*Ls + s at
//       data[(sl * NG + g) * vh + i]
//     double: 12 groups of double2 (2 reals)      192 B / site
//     single:  6 groups of float4  (4 reals)       96 B / site
//     half:    3 groups of 8 x fp16 (uint4)        48 B / site
//              + one float norm per site at norm[sl * vh + i]  (52 B / site)
//   gauge field: group g of the link (parity p, direction mu, site i) at
//       data[((p * 4 + mu) * NG + g) * vh + i]
//     double, 18 reals: 9 x double2   double, 12 reals: 6 x double2
//     single, 12 reals: 3 x float4    half, 12 reals: 3 x (4 x fp16, uint2)
// A warp reading group g of 32 consecutive sites touches 512 (or 256)
// contiguous bytes, so every spinor and link load is a fully coalesced
// 128-bit (or 64-bit) access.
//
// The 12-real form keeps the first two rows of each SU(3) link; the third is
// rebuilt in registers as conj(row0 x row1).  That identity holds only for
// det U = +1, which is why antiperiodic boundary signs are never folded into
// the stored links: the sign is applied to the hop instead.
#pragma once
#include "device_math.cuh"

namespace cpsgpu {

enum Precision { PREC_DOUBLE = 0, PREC_SINGLE = 1, PREC_HALF = 2 };

template <int P> struct PrecTraits;
template <> struct PrecTraits<PREC_DOUBLE> {
  using real = double;
  static constexpr int NG = 12;          // spinor groups
  static constexpr int SITE_BYTES = 192;
};
template <> struct PrecTraits<PREC_SINGLE> {
  using real = float;
  static constexpr int NG = 6;
  static constexpr int SITE_BYTES = 96;
};
template <> struct PrecTraits<PREC_HALF> {
  using real = float;
  static constexpr int NG = 3;
  static constexpr int SITE_BYTES = 52;
};

// Non-owning device view of a fermion field.
struct SpinorView {
  void *data = nullptr;
  float *norm = nullptr;  // half precision only
  long vh = 0;            // checkerboard sites per slice
  int ls = 1;             // slices per right-hand side
  int nrhs = 1;
};

// Non-owning device view of a gauge field.
struct GaugeView {
  const void *data = nullptr;
  long vh = 0;
};

template <int P> struct SpinorIO;

template <> struct SpinorIO<PREC_DOUBLE> {
  static __device__ __forceinline__ void load(const SpinorView &f, long sl, long i, double *v) {
    const double2 *d = reinterpret_cast<const double2 *>(f.data) + sl * 12 * f.vh + i;
#pragma unroll
    for (int g = 0; g < 12; g++) {
      double2 q = __ldg(d + g * f.vh);
      v[2 * g] = q.x;
      v[2 * g + 1] = q.y;
    }
  }
  static __device__ __forceinline__ void store(const SpinorView &f, long sl, long i, const double *v) {
    double2 *d = reinterpret_cast<double2 *>(f.data) + sl * 12 * f.vh + i;
#pragma unroll
    for (int g = 0; g < 12; g++) d[g * f.vh] = make_double2(v[2 * g], v[2 * g + 1]);
  }
  // one chiral half: reals [12*half, 12*half+12)
  static __device__ __forceinline__ void load_half(const SpinorView &f, long sl, long i, int half, double *v) {
    const double2 *d = reinterpret_cast<const double2 *>(f.data) + (sl * 12 + 6 * half) * f.vh + i;
#pragma unroll
    for (int g = 0; g < 6; g++) {
      double2 q = __ldg(d + g * f.vh);
      v[2 * g] = q.x;
      v[2 * g + 1] = q.y;
    }
  }
};

template <> struct SpinorIO<PREC_SINGLE> {
  static __device__ __forceinline__ void load(const SpinorView &f, long sl, long i, float *v) {
    const float4 *d = reinterpret_cast<const float4 *>(f.data) + sl * 6 * f.vh + i;
#pragma unroll
    for (int g = 0; g < 6; g++) {
      float4 q = __ldg(d + g * f.vh);
      v[4 * g] = q.x; v[4 * g + 1] = q.y; v[4 * g + 2] = q.z; v[4 * g + 3] = q.w;
    }
  }
  static __device__ __forceinline__ void store(const SpinorView &f, long sl, long i, const float *v) {
    float4 *d = reinterpret_cast<float4 *>(f.data) + sl * 6 * f.vh + i;
#pragma unroll
    for (int g = 0; g < 6; g++) d[g * f.vh] = make_float4(v[4 * g], v[4 * g + 1], v[4 * g + 2], v[4 * g + 3]);
  }
  static __device__ __forceinline__ void load_half(const SpinorView &f, long sl, long i, int half, float *v) {
    const float4 *d = reinterpret_cast<const float4 *>(f.data) + (sl * 6 + 3 * half) * f.vh + i;
#pragma unroll
    for (int g = 0; g < 3; g++) {
      float4 q = __ldg(d + g * f.vh);
      v[4 * g] = q.x; v[4 * g + 1] = q.y; v[4 * g + 2] = q.z; v[4 * g + 3] = q.w;
    }
  }
};

__device__ __forceinline__ void unpack8(uint4 q, float s, float *v) {
  const __half2 *h = reinterpret_cast<const __half2 *>(&q);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    float2 f = __half22float2(h[k]);
    v[2 * k] = f.x * s;
    v[2 * k + 1] = f.y * s;
  }
}

__device__ __forceinline__ void unpack8_raw(uint4 q, float *v) {
  const __half2 *h = reinterpret_cast<const __half2 *>(&q);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    float2 f = __half22float2(h[k]);
    v[2 * k] = f.x;
    v[2 * k + 1] = f.y;
  }
}

// Half precision: 24 fp16 values scaled by a per-site float norm (the
// largest magnitude in the spinor), so every stored value lies in [-1, 1].
template <> struct SpinorIO<PREC_HALF> {
  static __device__ __forceinline__ void load(const SpinorView &f, long sl, long i, float *v) {
    const uint4 *d = reinterpret_cast<const uint4 *>(f.data) + sl * 3 * f.vh + i;
    float s = __ldg(f.norm + sl * f.vh + i);
#pragma unroll
    for (int g = 0; g < 3; g++) unpack8(__ldg(d + g * f.vh), s, v + 8 * g);
  }
  static __device__ __forceinline__ void store(const SpinorView &f, long sl, long i, const float *v) {
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < 24; k++) m = fmaxf(m, fabsf(v[k]));
    float inv = (m > 0.f) ? 1.0f / m : 0.f;
    uint4 *d = reinterpret_cast<uint4 *>(f.data) + sl * 3 * f.vh + i;
#pragma unroll
    for (int g = 0; g < 3; g++) {
      uint4 q;
      __half2 *h = reinterpret_cast<__half2 *>(&q);
#pragma unroll
      for (int k = 0; k < 4; k++) h[k] = __floats2half2_rn(v[8 * g + 2 * k] * inv, v[8 * g + 2 * k + 1] * inv);
      d[g * f.vh] = q;
    }
    f.norm[sl * f.vh + i] = m;
  }
  static __device__ __forceinline__ void load_half(const SpinorView &f, long sl, long i, int half, float *v) {
    // a chiral half spans 1.5 groups; load the two groups it touches
    const uint4 *d = reinterpret_cast<const uint4 *>(f.data) + sl * 3 * f.vh + i;
    float s = __ldg(f.norm + sl * f.vh + i);
    float tmp[16];
    if (half == 0) {
      unpack8(__ldg(d), s, tmp);
      unpack8(__ldg(d + f.vh), s, tmp + 8);
#pragma unroll
      for (int k = 0; k < 12; k++) v[k] = tmp[k];
    } else {
      unpack8(__ldg(d + f.vh), s, tmp);
      unpack8(__ldg(d + 2 * f.vh), s, tmp + 8);
#pragma unroll
      for (int k = 0; k < 12; k++) v[k] = tmp[4 + k];
    }
  }
};

// ---- one slice of a field, 32-bit site indices ----
// Slice<P>(f, sl) points at slice sl; load(j) reads site j with the group
// stride vh.  Site indices are 32-bit (vh < 2^31 for any lattice that fits).
template <int P> struct Slice;
template <> struct Slice<PREC_DOUBLE> {
  const double2 *d;
  int vh;
  __device__ __forceinline__ Slice(const SpinorView &f, long sl)
      : d(reinterpret_cast<const double2 *>(f.data) + sl * 12 * f.vh), vh((int)f.vh) {}
  __device__ __forceinline__ void load(int j, double *v) const {
#pragma unroll
    for (int g = 0; g < 12; g++) {
      double2 q = __ldg(d + j + g * vh);
      v[2 * g] = q.x;
      v[2 * g + 1] = q.y;
    }
  }
  // values and their common scale (always 1 here; FP16 storage returns its norm)
  __device__ __forceinline__ void load_raw(int j, double *v, double &scale) const {
    load(j, v);
    scale = 1.0;
  }
  __device__ __forceinline__ void load_half_raw(int j, int half, double *v, double &scale) const {
    load_half(j, half, v);
    scale = 1.0;
  }
  __device__ __forceinline__ void load_half(int j, int half, double *v) const {
    const double2 *b = d + 6 * half * vh + j;
#pragma unroll
    for (int g = 0; g < 6; g++) {
      double2 q = __ldg(b + g * vh);
      v[2 * g] = q.x;
      v[2 * g + 1] = q.y;
    }
  }
};
template <> struct Slice<PREC_SINGLE> {
  const float4 *d;
  int vh;
  __device__ __forceinline__ Slice(const SpinorView &f, long sl)
      : d(reinterpret_cast<const float4 *>(f.data) + sl * 6 * f.vh), vh((int)f.vh) {}
  __device__ __forceinline__ void load(int j, float *v) const {
#pragma unroll
    for (int g = 0; g < 6; g++) {
      float4 q = __ldg(d + j + g * vh);
      v[4 * g] = q.x; v[4 * g + 1] = q.y; v[4 * g + 2] = q.z; v[4 * g + 3] = q.w;
    }
  }
  __device__ __forceinline__ void load_raw(int j, float *v, float &scale) const {
    load(j, v);
    scale = 1.0f;
  }
  __device__ __forceinline__ void load_half_raw(int j, int half, float *v, float &scale) const {
    load_half(j, half, v);
    scale = 1.0f;
  }
  __device__ __forceinline__ void load_half(int j, int half, float *v) const {
    const float4 *b = d + 3 * half * vh + j;
#pragma unroll
    for (int g = 0; g < 3; g++) {
      float4 q = __ldg(b + g * vh);
      v[4 * g] = q.x; v[4 * g + 1] = q.y; v[4 * g + 2] = q.z; v[4 * g + 3] = q.w;
    }
  }
};
template <> struct Slice<PREC_HALF> {
  const uint4 *d;
  const float *n;
  int vh;
  __device__ __forceinline__ Slice(const SpinorView &f, long sl)
      : d(reinterpret_cast<const uint4 *>(f.data) + sl * 3 * f.vh), n(f.norm + sl * f.vh), vh((int)f.vh) {}
  __device__ __forceinline__ void load(int j, float *v) const {
    const float s = __ldg(n + j);
#pragma unroll
    for (int g = 0; g < 3; g++) unpack8(__ldg(d + j + g * vh), s, v + 8 * g);
  }
  // the stored values unscaled, and the site's norm: the caller folds the
  // norm into a multiply it does anyway (24 fewer multiplies per site)
  __device__ __forceinline__ void load_raw(int j, float *v, float &scale) const {
    scale = __ldg(n + j);
#pragma unroll
    for (int g = 0; g < 3; g++) unpack8_raw(__ldg(d + j + g * vh), v + 8 * g);
  }
  __device__ __forceinline__ void load_half_raw(int j, int half, float *v, float &scale) const {
    scale = __ldg(n + j);
    float tmp[16];
    if (half == 0) {
      unpack8_raw(__ldg(d + j), tmp);
      unpack8_raw(__ldg(d + j + vh), tmp + 8);
#pragma unroll
      for (int k = 0; k < 12; k++) v[k] = tmp[k];
    } else {
      unpack8_raw(__ldg(d + j + vh), tmp);
      unpack8_raw(__ldg(d + j + 2 * vh), tmp + 8);
#pragma unroll
      for (int k = 0; k < 12; k++) v[k] = tmp[4 + k];
    }
  }
  __device__ __forceinline__ void load_half(int j, int half, float *v) const {
    const float s = __ldg(n + j);
    float tmp[16];
    if (half == 0) {
      unpack8(__ldg(d + j), s, tmp);
      unpack8(__ldg(d + j + vh), s, tmp + 8);
#pragma unroll
      for (int k = 0; k < 12; k++) v[k] = tmp[k];
    } else {
      unpack8(__ldg(d + j + vh), s, tmp);
      unpack8(__ldg(d + j + 2 * vh), s, tmp + 8);
#pragma unroll
      for (int k = 0; k < 12; k++) v[k] = tmp[4 + k];
    }
  }
};

// ---- 4-real chunks (reals 4c .. 4c+3) for register-light epilogues ----
template <int P> struct Chunk4;
template <> struct Chunk4<PREC_DOUBLE> {
  static __device__ __forceinline__ void load(const SpinorView &f, long sl, long i, int c, double *v) {
    const double2 *d = reinterpret_cast<const double2 *>(f.data) + (sl * 12 + 2 * c) * f.vh + i;
    double2 a = __ldg(d), b = __ldg(d + f.vh);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
  static __device__ __forceinline__ void store(const SpinorView &f, long sl, long i, int c, const double *v) {
    double2 *d = reinterpret_cast<double2 *>(f.data) + (sl * 12 + 2 * c) * f.vh + i;
    d[0] = make_double2(v[0], v[1]);
    d[f.vh] = make_double2(v[2], v[3]);
  }
};
template <> struct Chunk4<PREC_SINGLE> {
  static __device__ __forceinline__ void load(const SpinorView &f, long sl, long i, int c, float *v) {
    float4 q = __ldg(reinterpret_cast<const float4 *>(f.data) + (sl * 6 + c) * f.vh + i);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  }
  static __device__ __forceinline__ void store(const SpinorView &f, long sl, long i, int c, const float *v) {
    reinterpret_cast<float4 *>(f.data)[(sl * 6 + c) * f.vh + i] = make_float4(v[0], v[1], v[2], v[3]);
  }
};
template <> struct Chunk4<PREC_HALF> {
  // 4 fp16 = one half of a 16-byte group; stores need the whole site (norm)
  static __device__ __forceinline__ void load(const SpinorView &f, long sl, long i, int c, float *v) {
    const uint2 *d = reinterpret_cast<const uint2 *>(f.data) + 2 * ((sl * 3 + (c >> 1)) * f.vh + i) + (c & 1);
    const float s = __ldg(f.norm + sl * f.vh + i);
    uint2 q = __ldg(d);
    const __half2 *h = reinterpret_cast<const __half2 *>(&q);
    float2 a = __half22float2(h[0]), b = __half22float2(h[1]);
    v[0] = a.x * s; v[1] = a.y * s; v[2] = b.x * s; v[3] = b.y * s;
  }
};

// Chunk-by-chunk reads of one site of a field (chunks 0..5 in order, as the
// fused epilogues stream them): the FP16 form loads the site's norm once and
// each 16-byte group once for its two chunks, where Chunk4 would load a norm
// and half a group per chunk.  The values are Chunk4's.
template <int P> struct ChunkReader {
  const SpinorView f;  // a copy: a reference to a kernel parameter can force it into local memory
  long sl, i;
  __device__ __forceinline__ ChunkReader(const SpinorView &f_, long sl_, long i_) : f(f_), sl(sl_), i(i_) {}
  __device__ __forceinline__ void get(int c, typename PrecTraits<P>::real *v) { Chunk4<P>::load(f, sl, i, c, v); }
};
template <> struct ChunkReader<PREC_HALF> {
  const uint4 *d;
  long vh;
  float s;
  uint4 q;
  __device__ __forceinline__ ChunkReader(const SpinorView &f, long sl, long i)
      : d(reinterpret_cast<const uint4 *>(f.data) + sl * 3 * f.vh + i), vh(f.vh), s(__ldg(f.norm + sl * f.vh + i)) {}
  // c in increasing order; an even c loads the group, the odd one reuses it
  __device__ __forceinline__ void get(int c, float *v) {
    if ((c & 1) == 0) q = __ldg(d + (c >> 1) * vh);
    const __half2 *h = reinterpret_cast<const __half2 *>(&q) + 2 * (c & 1);
    const float2 a = __half22float2(h[0]), b = __half22float2(h[1]);
    v[0] = a.x * s; v[1] = a.y * s; v[2] = b.x * s; v[3] = b.y * s;
  }
};

// ---- gauge links ----
// The FP32 / FP16 forms index the gauge field with 32-bit offsets (at most
// 8 x 4 x vh elements: the Lattice constructor refuses a larger checkerboard
// volume); FP16 storage runs 2-3% faster for it.  The FP64 forms keep 64-bit
// offsets: 32-bit ones cost their MatPcDagMatPc 4% (register allocation).
template <int P, int RECON> struct LinkIO;

template <> struct LinkIO<PREC_DOUBLE, 18> {
  static constexpr int NG = 9;
  static __device__ __forceinline__ void load(const GaugeView &g, int p, int mu, long i, su3<double> &u) {
    const double2 *d = reinterpret_cast<const double2 *>(g.data) + ((p * 4 + mu) * NG) * g.vh + i;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 q = __ldg(d + k * g.vh);
      u.m[k / 3][k % 3] = {q.x, q.y};
    }
  }
};
template <> struct LinkIO<PREC_DOUBLE, 12> {
  static constexpr int NG = 6;
  static __device__ __forceinline__ void load(const GaugeView &g, int p, int mu, long i, su3<double> &u) {
    const double2 *d = reinterpret_cast<const double2 *>(g.data) + ((p * 4 + mu) * NG) * g.vh + i;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      double2 q = __ldg(d + k * g.vh);
      u.m[k / 3][k % 3] = {q.x, q.y};
    }
    reconstruct_row2(u);
  }
};
template <> struct LinkIO<PREC_SINGLE, 12> {
  static constexpr int NG = 3;
  static __device__ __forceinline__ void load(const GaugeView &g, int p, int mu, long i, su3<float> &u) {
    const int vh = (int)g.vh;
    const float4 *d = reinterpret_cast<const float4 *>(g.data) + ((p * 4 + mu) * NG * vh + (int)i);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float4 q = __ldg(d + k * vh);
      int e = 2 * k;
      u.m[e / 3][e % 3] = {q.x, q.y};
      u.m[(e + 1) / 3][(e + 1) % 3] = {q.z, q.w};
    }
    reconstruct_row2(u);
  }
};
template <> struct LinkIO<PREC_HALF, 12> {
  static constexpr int NG = 3;
  static __device__ __forceinline__ void load(const GaugeView &g, int p, int mu, long i, su3<float> &u) {
    const int vh = (int)g.vh;
    const uint2 *d = reinterpret_cast<const uint2 *>(g.data) + ((p * 4 + mu) * NG * vh + (int)i);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      uint2 q = __ldg(d + k * vh);
      const __half2 *h = reinterpret_cast<const __half2 *>(&q);
      float2 a = __half22float2(h[0]), b = __half22float2(h[1]);
      int e = 2 * k;
      u.m[e / 3][e % 3] = {a.x, a.y};
      u.m[(e + 1) / 3][(e + 1) % 3] = {b.x, b.y};
    }
    reconstruct_row2(u);
  }
};

// Full 18-real sloppy links: no third-row rebuild (24 fewer flops per link),
// for kernels bound by instruction issue rather than by HBM.
//   FP32: elements 0-7 as four float4 (two complex each) at
//         f4[((p*4 + mu)*4 + k)*vh + i], element 8 as float2 at
//         f2[(p*4 + mu)*vh + i] after the 32*vh float4            (72 B)
//   FP16: elements 0-7 as two uint4 (four complex each) at
//         u4[((p*4 + mu)*2 + k)*vh + i], element 8 as one half2 at
//         u1[(p*4 + mu)*vh + i] after the 16*vh uint4             (36 B)
template <> struct LinkIO<PREC_SINGLE, 18> {
  static __device__ __forceinline__ void load(const GaugeView &g, int p, int mu, long i, su3<float> &u) {
    const int vh = (int)g.vh;
    const float4 *d = reinterpret_cast<const float4 *>(g.data) + ((p * 4 + mu) * 4 * vh + (int)i);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float4 q = __ldg(d + k * vh);
      u.m[(2 * k) / 3][(2 * k) % 3] = {q.x, q.y};
      u.m[(2 * k + 1) / 3][(2 * k + 1) % 3] = {q.z, q.w};
    }
    const float2 *e = reinterpret_cast<const float2 *>(reinterpret_cast<const float4 *>(g.data) + 32 * vh) +
                      ((p * 4 + mu) * vh + (int)i);
    float2 q = __ldg(e);
    u.m[2][2] = {q.x, q.y};
  }
};
template <> struct LinkIO<PREC_HALF, 18> {
  static __device__ __forceinline__ void load(const GaugeView &g, int p, int mu, long i, su3<float> &u) {
    const int vh = (int)g.vh;
    const uint4 *d = reinterpret_cast<const uint4 *>(g.data) + ((p * 4 + mu) * 2 * vh + (int)i);
#pragma unroll
    for (int k = 0; k < 2; k++) {
      uint4 q = __ldg(d + k * vh);
      const __half2 *h = reinterpret_cast<const __half2 *>(&q);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        float2 a = __half22float2(h[c]);
        u.m[(4 * k + c) / 3][(4 * k + c) % 3] = {a.x, a.y};
      }
    }
    const unsigned *e = reinterpret_cast<const unsigned *>(reinterpret_cast<const uint4 *>(g.data) + 16 * vh) +
                        ((p * 4 + mu) * vh + (int)i);
    unsigned q = __ldg(e);
    float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&q));
    u.m[2][2] = {a.x, a.y};
  }
};
// FP16 spinors with FP32 links (LINK_F32_12 / LINK_F32_18): the links cost
// no conversions; their extra bytes are shared by every slice of a site.
constexpr int LINK_F32_12 = 112;
constexpr int LINK_F32_18 = 118;
template <> struct LinkIO<PREC_HALF, LINK_F32_12> : LinkIO<PREC_SINGLE, 12> {};
template <> struct LinkIO<PREC_HALF, LINK_F32_18> : LinkIO<PREC_SINGLE, 18> {};

}  // namespace cpsgpu
