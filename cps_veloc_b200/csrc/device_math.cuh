// Device arithmetic for the fermion operators: complex numbers, SU(3)
// links (full 18-real or compressed 12-real), Dirac spinors, and the
// spin projection (1 -/+ gamma_mu) used by every hop.
//
// Spinor components are held in registers as 24 reals in the reference's
// element order, index 2*(colour + 3*spin) + re/im (wilson_dslash.C:60), so
// chiral halves are reals 0-11 (gamma_5 = +1) and 12-23 (gamma_5 = -1).
//
// The gamma-matrix convention is the one the reference expands in
// OneMinusPlusGammaTimesPsi (wilson_dslash.C:64-128).  Because (1 + k g_mu)
// has rank 2, each hop is computed on a two-spin half spinor h = P psi,
// multiplied by the link, and reconstructed: the same value as the
// reference's full four-spin product, at half the flops (the 1320 flops per
// site the reference counts, wilson_dslash.C:515).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace cpsgpu {

template <typename R> struct cplx {
  R re, im;
};

template <typename R> __device__ __forceinline__ cplx<R> mk(R a, R b) { return {a, b}; }
template <typename R> __device__ __forceinline__ cplx<R> operator+(cplx<R> a, cplx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R> __device__ __forceinline__ cplx<R> operator-(cplx<R> a, cplx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R> __device__ __forceinline__ cplx<R> operator*(cplx<R> a, cplx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R> __device__ __forceinline__ cplx<R> conj(cplx<R> a) { return {a.re, -a.im}; }
// a * conj(b)
template <typename R> __device__ __forceinline__ cplx<R> mul_conj(cplx<R> a, cplx<R> b) {
  return {a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im};
}
// conj(a) * b
template <typename R> __device__ __forceinline__ cplx<R> conj_mul(cplx<R> a, cplx<R> b) {
  return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}
// i * a
template <typename R> __device__ __forceinline__ cplx<R> times_i(cplx<R> a) { return {-a.im, a.re}; }

// SU(3) matrix, m[row][col]
template <typename R> struct su3 {
  cplx<R> m[3][3];
};

__device__ __forceinline__ float fmac_(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmac_(double a, double b, double c) { return fma(a, b, c); }

// conj(a b - c d) as one fused chain per component
template <typename R> __device__ __forceinline__ cplx<R> conj_cross(cplx<R> a, cplx<R> b, cplx<R> c, cplx<R> d) {
  R re = c.im * d.im;
  re = fmac_(-c.re, d.re, re);
  re = fmac_(-a.im, b.im, re);
  re = fmac_(a.re, b.re, re);
  R im = c.re * d.im;
  im = fmac_(c.im, d.re, im);
  im = fmac_(-a.re, b.im, im);
  im = fmac_(-a.im, b.re, im);
  return {re, im};
}

// third row of an SU(3) matrix from its first two: r2 = conj(r0 x r1)
template <typename R> __device__ __forceinline__ void reconstruct_row2(su3<R> &u) {
  u.m[2][0] = conj_cross(u.m[0][1], u.m[1][2], u.m[0][2], u.m[1][1]);
  u.m[2][1] = conj_cross(u.m[0][2], u.m[1][0], u.m[0][0], u.m[1][2]);
  u.m[2][2] = conj_cross(u.m[0][0], u.m[1][1], u.m[0][1], u.m[1][0]);
}

// Half spinor: two spin components of a colour vector.
template <typename R> struct half_spinor {
  cplx<R> h[2][3];
};

template <typename R> __device__ __forceinline__ cplx<R> sp(const R *v, int spin, int col) {
  return {v[2 * (col + 3 * spin)], v[2 * (col + 3 * spin) + 1]};
}

// h = first two spin rows of (1 + k gamma_mu) psi.
template <typename R>
__device__ __forceinline__ half_spinor<R> project(const R *psi, int mu, R k) {
  half_spinor<R> h;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    cplx<R> p0 = sp(psi, 0, c), p1 = sp(psi, 1, c), p2 = sp(psi, 2, c), p3 = sp(psi, 3, c);
    cplx<R> a, b;
    switch (mu) {
      case 0: a = times_i(p3); b = times_i(p2); break;             // g_x: rows (0,3,+i) (1,2,+i)
      case 1: a = mk(-p3.re, -p3.im); b = p2; break;                // g_y: rows (0,3,-1) (1,2,+1)
      case 2: a = times_i(p2); b = mk(p3.im, -p3.re); break;        // g_z: rows (0,2,+i) (1,3,-i)
      default: a = p2; b = p3; break;                               // g_t: rows (0,2,+1) (1,3,+1)
    }
    h.h[0][c] = mk(p0.re + k * a.re, p0.im + k * a.im);
    h.h[1][c] = mk(p1.re + k * b.re, p1.im + k * b.im);
  }
  return h;
}

template <typename R>
__device__ __forceinline__ void negate(half_spinor<R> &h) {
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int c = 0; c < 3; c++) h.h[s][c] = mk(-h.h[s][c].re, -h.h[s][c].im);
}

// acc += w * (full four-spin spinor rebuilt from the half spinor g = U h),
// the rows 2,3 of (1 + k gamma_mu) expressed through rows 0,1.
template <typename R>
__device__ __forceinline__ void reconstruct_acc(R *acc, const half_spinor<R> &g, int mu, R k, R w) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    cplx<R> g0 = g.h[0][c], g1 = g.h[1][c];
    cplx<R> r2, r3;
    switch (mu) {
      case 0: { cplx<R> a = times_i(g1), b = times_i(g0); r2 = mk(-k * a.re, -k * a.im); r3 = mk(-k * b.re, -k * b.im); } break;
      case 1: r2 = mk(k * g1.re, k * g1.im); r3 = mk(-k * g0.re, -k * g0.im); break;
      case 2: { cplx<R> a = times_i(g0), b = times_i(g1); r2 = mk(-k * a.re, -k * a.im); r3 = mk(k * b.re, k * b.im); } break;
      default: r2 = mk(k * g0.re, k * g0.im); r3 = mk(k * g1.re, k * g1.im); break;
    }
    acc[2 * (c + 0)] += w * g0.re;      acc[2 * (c + 0) + 1] += w * g0.im;
    acc[2 * (c + 3)] += w * g1.re;      acc[2 * (c + 3) + 1] += w * g1.im;
    acc[2 * (c + 6)] += w * r2.re;      acc[2 * (c + 6) + 1] += w * r2.im;
    acc[2 * (c + 9)] += w * r3.re;      acc[2 * (c + 9) + 1] += w * r3.im;
  }
}

// Multiply-add chains are written as explicit fused multiply-adds: the
// compiler may not re-associate v + (a * b) into them on its own, and the
// split form costs 6 instructions per complex multiply-add instead of 4.

// g = U h  (dagger = false) or U^dagger h (dagger = true)
template <typename R>
__device__ __forceinline__ half_spinor<R> link_mul(const su3<R> &u, const half_spinor<R> &h, bool dagger) {
  half_spinor<R> g;
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      // v = sum_b m(a, b) h_b with m = u[a][b] or conj(u[b][a])
      const cplx<R> m0 = dagger ? conj(u.m[0][a]) : u.m[a][0];
      const cplx<R> h0 = h.h[s][0];
      R re = m0.re * h0.re, im = m0.re * h0.im;
      re = fmac_(-m0.im, h0.im, re);
      im = fmac_(m0.im, h0.re, im);
#pragma unroll
      for (int b = 1; b < 3; b++) {
        const cplx<R> m = dagger ? conj(u.m[b][a]) : u.m[a][b];
        const cplx<R> hb = h.h[s][b];
        re = fmac_(m.re, hb.re, re);
        re = fmac_(-m.im, hb.im, re);
        im = fmac_(m.re, hb.im, im);
        im = fmac_(m.im, hb.re, im);
      }
      g.h[s][a] = {re, im};
    }
  return g;
}


// ---- Packed FP32 forms (sm_100 FFMA2: two FP32 fused multiply-adds per
// lane and instruction) ----
// The two spins of a half spinor sit in the two lanes of a float2, so every
// link element enters as a scalar broadcast to both lanes (a broadcast and a
// negated broadcast cost no extra instruction), and the link multiply, the
// upper-spin accumulation and, for mu = z, t, the lower-spin accumulation
// each take half the instructions of the scalar form.  The arithmetic per
// lane is the scalar form's, operation for operation.
struct hs2 {
  float2 re[3], im[3];  // re[c] = (h[0][c].re, h[1][c].re)
};
// 24-real accumulator: spins (0, 1) in u*, spins (2, 3) in l*
struct acc2 {
  float2 ur[3], ui[3], lr[3], li[3];
};
__device__ __forceinline__ float2 b2(float s) { return make_float2(s, s); }

__device__ __forceinline__ void acc2_zero(acc2 &a) {
#pragma unroll
  for (int c = 0; c < 3; c++) a.ur[c] = a.ui[c] = a.lr[c] = a.li[c] = make_float2(0.f, 0.f);
}

__device__ __forceinline__ hs2 pack_hs2(const half_spinor<float> &h) {
  hs2 r;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    r.re[c] = make_float2(h.h[0][c].re, h.h[1][c].re);
    r.im[c] = make_float2(h.h[0][c].im, h.h[1][c].im);
  }
  return r;
}

// g = U h (dagger = false) or U^dagger h (dagger = true), both spins at once
__device__ __forceinline__ hs2 link_mul2(const su3<float> &u, const hs2 &h, bool dagger) {
  hs2 g;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    // m(a, b) = u[a][b] or conj(u[b][a]); re += m.re h.re - m.im h.im, im += m.re h.im + m.im h.re
    const cplx<float> m0 = dagger ? conj(u.m[0][a]) : u.m[a][0];
    float2 re = __fmul2_rn(b2(m0.re), h.re[0]);
    float2 im = __fmul2_rn(b2(m0.re), h.im[0]);
    re = __ffma2_rn(b2(-m0.im), h.im[0], re);
    im = __ffma2_rn(b2(m0.im), h.re[0], im);
#pragma unroll
    for (int b = 1; b < 3; b++) {
      const cplx<float> m = dagger ? conj(u.m[b][a]) : u.m[a][b];
      re = __ffma2_rn(b2(m.re), h.re[b], re);
      re = __ffma2_rn(b2(-m.im), h.im[b], re);
      im = __ffma2_rn(b2(m.re), h.im[b], im);
      im = __ffma2_rn(b2(m.im), h.re[b], im);
    }
    g.re[a] = re;
    g.im[a] = im;
  }
  return g;
}

// a += w * (four-spin spinor rebuilt from g), as reconstruct_acc
__device__ __forceinline__ void reconstruct_acc2(acc2 &a, const hs2 &g, int mu, float k, float w) {
  const float wk = w * k;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    a.ur[c] = __ffma2_rn(b2(w), g.re[c], a.ur[c]);
    a.ui[c] = __ffma2_rn(b2(w), g.im[c], a.ui[c]);
    switch (mu) {
      case 0:  // r2 = -k i g1, r3 = -k i g0
        a.lr[c].x = fmaf(wk, g.im[c].y, a.lr[c].x);
        a.lr[c].y = fmaf(wk, g.im[c].x, a.lr[c].y);
        a.li[c].x = fmaf(-wk, g.re[c].y, a.li[c].x);
        a.li[c].y = fmaf(-wk, g.re[c].x, a.li[c].y);
        break;
      case 1:  // r2 = k g1, r3 = -k g0
        a.lr[c].x = fmaf(wk, g.re[c].y, a.lr[c].x);
        a.lr[c].y = fmaf(-wk, g.re[c].x, a.lr[c].y);
        a.li[c].x = fmaf(wk, g.im[c].y, a.li[c].x);
        a.li[c].y = fmaf(-wk, g.im[c].x, a.li[c].y);
        break;
      case 2:  // r2 = -k i g0, r3 = k i g1
        a.lr[c] = __ffma2_rn(make_float2(wk, -wk), g.im[c], a.lr[c]);
        a.li[c] = __ffma2_rn(make_float2(-wk, wk), g.re[c], a.li[c]);
        break;
      default:  // r2 = k g0, r3 = k g1
        a.lr[c] = __ffma2_rn(b2(wk), g.re[c], a.lr[c]);
        a.li[c] = __ffma2_rn(b2(wk), g.im[c], a.li[c]);
        break;
    }
  }
}

// the accumulator in the reference's element order, 2 (colour + 3 spin) + re/im
__device__ __forceinline__ void acc2_store(const acc2 &a, float *acc) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc[2 * c] = a.ur[c].x;           acc[2 * c + 1] = a.ui[c].x;
    acc[2 * (c + 3)] = a.ur[c].y;     acc[2 * (c + 3) + 1] = a.ui[c].y;
    acc[2 * (c + 6)] = a.lr[c].x;     acc[2 * (c + 6) + 1] = a.li[c].x;
    acc[2 * (c + 9)] = a.lr[c].y;     acc[2 * (c + 9) + 1] = a.li[c].y;
  }
}

// The accumulator of one hop site: the scalar form for FP64, the packed
// form for FP32 arithmetic (FP32 and FP16 storage).
template <typename R> struct HopAcc {
  R a[24];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int k = 0; k < 24; k++) a[k] = R(0);
  }
  // += w * reconstruct(U h or U^dagger h)
  __device__ __forceinline__ void hop(const su3<R> &u, const half_spinor<R> &h, bool dagger, int mu, R k, R w) {
    reconstruct_acc(a, link_mul(u, h, dagger), mu, k, w);
  }
  // += w * reconstruct(g)
  __device__ __forceinline__ void add(const half_spinor<R> &g, int mu, R k, R w) { reconstruct_acc(a, g, mu, k, w); }
  __device__ __forceinline__ void store(R *acc) const {
#pragma unroll
    for (int k = 0; k < 24; k++) acc[k] = a[k];
  }
};
template <> struct HopAcc<float> {
  acc2 a;
  __device__ __forceinline__ void zero() { acc2_zero(a); }
  __device__ __forceinline__ void hop(const su3<float> &u, const half_spinor<float> &h, bool dagger, int mu, float k,
                                      float w) {
    reconstruct_acc2(a, link_mul2(u, pack_hs2(h), dagger), mu, k, w);
  }
  __device__ __forceinline__ void add(const half_spinor<float> &g, int mu, float k, float w) {
    reconstruct_acc2(a, pack_hs2(g), mu, k, w);
  }
  __device__ __forceinline__ void store(float *acc) const { acc2_store(a, acc); }
};

}  // namespace cpsgpu
