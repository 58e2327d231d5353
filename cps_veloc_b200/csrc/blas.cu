// Vector kernels, storage-order conversion and the per-chirality s-mixing
// kernel.  All are HBM-bandwidth bound: one thread per site, each site's
// 24 reals moved with the coalesced group loads of fields.cuh.
#include <cmath>
#include <cstring>

#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

// ---------------------------------------------------------------- fields
size_t Field::site_bytes() const {
  return prec == PREC_DOUBLE ? 192 : prec == PREC_SINGLE ? 96 : 48;
}

void Field::create(int p, long vh_, int ls_, int nrhs_) {
  prec = p;
  vh = vh_;
  ls = ls_;
  nrhs = nrhs_;
  data.alloc(sites() * site_bytes());
  if (p == PREC_HALF)
    norm.alloc(sites() * sizeof(float));
  else
    norm.release();
}

SpinorView Field::view_rhs(int k) const {
  SpinorView v = view();
  size_t per = (size_t)vh * ls;
  v.data = static_cast<char *>(data.ptr) + per * site_bytes() * k;
  if (norm.ptr) v.norm = norm.as<float>() + per * k;
  v.nrhs = 1;
  return v;
}

long long &launch_counter() {
  static thread_local long long n = 0;
  return n;
}

void ensure_field(Field &f, int prec, long vh, int ls, int nrhs) {
  if (f.data.ptr && f.prec == prec && f.vh == vh && f.ls == ls && f.nrhs == nrhs) return;
  f.create(prec, vh, ls, nrhs);
}

namespace {
constexpr int TPB = 256;

inline unsigned blocks_for(size_t n) { return (unsigned)((n + TPB - 1) / TPB); }

template <int P> using RealT = typename PrecTraits<P>::real;

template <int PD, int PS>
__global__ void convert_kernel(SpinorView dst, SpinorView src, size_t n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  long sl = (long)(idx / src.vh), i = (long)(idx % src.vh);
  RealT<PS> a[24];
  RealT<PD> b[24];
  SpinorIO<PS>::load(src, sl, i, a);
#pragma unroll
  for (int k = 0; k < 24; k++) b[k] = RealT<PD>(a[k]);
  SpinorIO<PD>::store(dst, sl, i, b);
}

template <int P>
__global__ void zero_kernel(SpinorView dst, size_t n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  long sl = (long)(idx / dst.vh), i = (long)(idx % dst.vh);
  RealT<P> a[24];
#pragma unroll
  for (int k = 0; k < 24; k++) a[k] = RealT<P>(0);
  SpinorIO<P>::store(dst, sl, i, a);
}

// p = r + beta p  (inv_cg.C:360)
template <int P>
__global__ void xpay_kernel(SpinorView p, SpinorView r, const SolverScalars *st, size_t n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const long per = p.vh * p.ls;
  const int rhs = (int)(blockIdx.y);
  if (st[rhs].done) return;
  if (idx >= (size_t)per) return;
  long sl = rhs * p.ls + (long)(idx / p.vh), i = (long)(idx % p.vh);
  RealT<P> a[24], b[24];
  SpinorIO<P>::load(r, sl, i, a);
  SpinorIO<P>::load(p, sl, i, b);
  const RealT<P> beta = RealT<P>(st[rhs].beta);
#pragma unroll
  for (int k = 0; k < 24; k++) b[k] = a[k] + beta * b[k];
  SpinorIO<P>::store(p, sl, i, b);
}

// out = a x + y (fTimesV1PlusV2), FP64
__global__ void axpby_kernel(SpinorView out, double a, SpinorView x, SpinorView y, size_t n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  long sl = (long)(idx / x.vh), i = (long)(idx % x.vh);
  double xv[24], yv[24];
  SpinorIO<PREC_DOUBLE>::load(x, sl, i, xv);
  SpinorIO<PREC_DOUBLE>::load(y, sl, i, yv);
#pragma unroll
  for (int k = 0; k < 24; k++) yv[k] = fma(a, xv[k], yv[k]);
  SpinorIO<PREC_DOUBLE>::store(out, sl, i, yv);
}

// out = (scale a[0]) x + y with the coefficient read on the device
__global__ void axpby_dev_kernel(SpinorView out, const double *a, double scale, SpinorView x, SpinorView y,
                                 size_t n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const double c = scale * __ldg(a);
  long sl = (long)(idx / x.vh), i = (long)(idx % x.vh);
  double xv[24], yv[24];
  SpinorIO<PREC_DOUBLE>::load(x, sl, i, xv);
  SpinorIO<PREC_DOUBLE>::load(y, sl, i, yv);
#pragma unroll
  for (int k = 0; k < 24; k++) yv[k] = fma(c, xv[k], yv[k]);
  SpinorIO<PREC_DOUBLE>::store(out, sl, i, yv);
}

__global__ void scale_kernel(double a, SpinorView f, size_t n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  long sl = (long)(idx / f.vh), i = (long)(idx % f.vh);
  double v[24];
  SpinorIO<PREC_DOUBLE>::load(f, sl, i, v);
#pragma unroll
  for (int k = 0; k < 24; k++) v[k] *= a;
  SpinorIO<PREC_DOUBLE>::store(f, sl, i, v);
}

// x64 += xs; xs = 0  (reliable update: solution accumulated in FP64)
template <int PXS>
__global__ void accum_kernel(SpinorView x, SpinorView xs, const SolverScalars *st, int force) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const long per = x.vh * x.ls;
  const int rhs = (int)(blockIdx.y);
  if (!force && (st[rhs].done || !st[rhs].reliable)) return;
  if (idx >= (size_t)per) return;
  long sl = rhs * x.ls + (long)(idx / x.vh), i = (long)(idx % x.vh);
  double a[24];
  RealT<PXS> b[24];
  SpinorIO<PREC_DOUBLE>::load(x, sl, i, a);
  SpinorIO<PXS>::load(xs, sl, i, b);
#pragma unroll
  for (int k = 0; k < 24; k++) {
    a[k] += double(b[k]);
    b[k] = RealT<PXS>(0);
  }
  SpinorIO<PREC_DOUBLE>::store(x, sl, i, a);
  SpinorIO<PXS>::store(xs, sl, i, b);
}

template <int P>
__global__ void norm_kernel(SpinorView f, SolverScalars *st, double *partials, int op, int gate) {
  const int rhs = blockIdx.z;
  if (gate == GATE_RUNNING && st[rhs].done) return;
  if (gate == GATE_RELIABLE && (st[rhs].done || !st[rhs].reliable)) return;
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const long per = f.vh * f.ls;
  double v[1] = {0.0};
  if (idx < (size_t)per) {
    long sl = rhs * f.ls + (long)(idx / f.vh), i = (long)(idx % f.vh);
    RealT<P> a[24];
    SpinorIO<P>::load(f, sl, i, a);
#pragma unroll
    for (int k = 0; k < 24; k++) v[0] += double(a[k]) * double(a[k]);
  }
  block_partial<1>(v, partials);
}

__global__ void init_scalars_kernel(SolverScalars *st, int nrhs, SolverScalars init) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nrhs) st[k] = init;
}

template <int P>
__global__ void import_kernel(SpinorView dst, const double *src, size_t n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  long sl = (long)(idx / dst.vh), i = (long)(idx % dst.vh);
  const double2 *s2 = reinterpret_cast<const double2 *>(src + 24 * idx);
  RealT<P> a[24];
#pragma unroll
  for (int k = 0; k < 12; k++) {
    double2 q = s2[k];
    a[2 * k] = RealT<P>(q.x);
    a[2 * k + 1] = RealT<P>(q.y);
  }
  SpinorIO<P>::store(dst, sl, i, a);
}

template <int P>
__global__ void export_kernel(SpinorView src, double *dst, size_t n) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  long sl = (long)(idx / src.vh), i = (long)(idx % src.vh);
  RealT<P> a[24];
  SpinorIO<P>::load(src, sl, i, a);
  double2 *d2 = reinterpret_cast<double2 *>(dst + 24 * idx);
#pragma unroll
  for (int k = 0; k < 12; k++) d2[k] = make_double2(double(a[2 * k]), double(a[2 * k + 1]));
}

// out(s) = sum_t Mix_chi[s][t] in(t), block = (BX sites, all Ls slices)
template <int P>
__global__ void mix_kernel(SpinorView in, SpinorView out, const double *mix, int ls, const SolverScalars *st,
                           int gate, int cplx) {
  using R = RealT<P>;
  if (gate == GATE_RUNNING && st[blockIdx.z].done) return;
  if (gate == GATE_RELIABLE && (st[blockIdx.z].done || !st[blockIdx.z].reliable)) return;
  extern __shared__ unsigned char smraw[];
  R *sm = reinterpret_cast<R *>(smraw);
  double *mx = reinterpret_cast<double *>(sm + (size_t)ls * blockDim.x * 24);
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  for (int k = tid; k < 2 * ls * ls * (cplx ? 2 : 1); k += blockDim.x * blockDim.y) mx[k] = mix[k];
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = threadIdx.y;
  const long rhs = blockIdx.z;
  const bool active = i < in.vh;
  R a[24];
  if (active) SpinorIO<P>::load(in, rhs * ls + s, i, a);
  // [ls][24][BX]: a warp's shared-memory accesses are consecutive words
  R *mine = sm + (size_t)s * 24 * blockDim.x + threadIdx.x;
#pragma unroll
  for (int k = 0; k < 24; k++) mine[k * blockDim.x] = active ? a[k] : R(0);
  __syncthreads();
  if (!active) return;
#pragma unroll
  for (int k = 0; k < 24; k++) a[k] = R(0);
  if (!cplx) {
    for (int t = 0; t < ls; t++) {
      const R mu_ = R(mx[s * ls + t]), md_ = R(mx[ls * ls + s * ls + t]);
      const R *src = sm + (size_t)t * 24 * blockDim.x + threadIdx.x;
#pragma unroll
      for (int k = 0; k < 12; k++) a[k] += mu_ * src[k * blockDim.x];
#pragma unroll
      for (int k = 12; k < 24; k++) a[k] += md_ * src[k * blockDim.x];
    }
  } else {
    // complex entries ([..][re, im]) on the (re, im) pairs of the spinor
    for (int t = 0; t < ls; t++) {
      const double *pu = mx + 2 * (s * ls + t), *pd = mx + 2 * (ls * ls + s * ls + t);
      const R ur = R(pu[0]), ui = R(pu[1]), dr = R(pd[0]), di = R(pd[1]);
      const R *src = sm + (size_t)t * 24 * blockDim.x + threadIdx.x;
#pragma unroll
      for (int k = 0; k < 24; k += 2) {
        const R xr = src[k * blockDim.x], xi = src[(k + 1) * blockDim.x];
        const R mr = k < 12 ? ur : dr, mi = k < 12 ? ui : di;
        a[k] += mr * xr - mi * xi;
        a[k + 1] += mr * xi + mi * xr;
      }
    }
  }
  SpinorIO<P>::store(out, rhs * ls + s, i, a);
}

// ---- gauge import: WILSON order (p, i, mu, col-major 3x3) -> device forms
__device__ __forceinline__ void atomic_max_pos(double *addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

__global__ void gauge_import_kernel(const double *src, long vh, int L0, int L1, int L2, int L3, double bc0,
                                    double bc1, double bc2, double bc3, int signs_applied, double2 *d18,
                                    double2 *d12, float4 *s12, uint2 *h12, float4 *s18, uint4 *h18,
                                    double *recon_err) {
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;  // over 2 * vh * 4
  if (idx >= 8 * vh) return;
  const int mu = (int)(idx % 4);
  const long gsite = idx / 4;  // p * vh + i
  const int p = (int)(gsite / vh);
  const long i = gsite % vh;
  const int hx = L0 / 2;
  long rem = i / hx;
  int c[4];
  c[1] = (int)(rem % L1);
  rem /= L1;
  c[2] = (int)(rem % L2);
  c[3] = (int)(rem / L2);
  c[0] = 2 * (int)(i % hx) + ((c[1] + c[2] + c[3] + p) & 1);
  const int Lm[4] = {L0, L1, L2, L3};
  const double bcm[4] = {bc0, bc1, bc2, bc3};
  double sign = 1.0;
  if (signs_applied && c[mu] == Lm[mu] - 1) sign = bcm[mu];
  const double *m = src + 72 * gsite + 18 * mu;
  cplx<double> u[3][3];
  for (int row = 0; row < 3; row++)
    for (int col = 0; col < 3; col++) u[row][col] = {sign * m[2 * (row + 3 * col)], sign * m[2 * (row + 3 * col) + 1]};
  const long gbase = (long)(p * 4 + mu);
  for (int k = 0; k < 9; k++) d18[(gbase * 9 + k) * vh + i] = make_double2(u[k / 3][k % 3].re, u[k / 3][k % 3].im);
  for (int k = 0; k < 6; k++) d12[(gbase * 6 + k) * vh + i] = make_double2(u[k / 3][k % 3].re, u[k / 3][k % 3].im);
  for (int k = 0; k < 3; k++) {
    cplx<double> a = u[(2 * k) / 3][(2 * k) % 3], b = u[(2 * k + 1) / 3][(2 * k + 1) % 3];
    s12[(gbase * 3 + k) * vh + i] = make_float4((float)a.re, (float)a.im, (float)b.re, (float)b.im);
    uint2 q;
    __half2 *h = reinterpret_cast<__half2 *>(&q);
    h[0] = __floats2half2_rn((float)a.re, (float)a.im);
    h[1] = __floats2half2_rn((float)b.re, (float)b.im);
    h12[(gbase * 3 + k) * vh + i] = q;
  }
  // full links (layouts at LinkIO<PREC_SINGLE / PREC_HALF, 18>)
  for (int k = 0; k < 4; k++) {
    cplx<double> a = u[(2 * k) / 3][(2 * k) % 3], b = u[(2 * k + 1) / 3][(2 * k + 1) % 3];
    s18[(gbase * 4 + k) * vh + i] = make_float4((float)a.re, (float)a.im, (float)b.re, (float)b.im);
  }
  reinterpret_cast<float2 *>(s18 + 32 * vh)[gbase * vh + i] = make_float2((float)u[2][2].re, (float)u[2][2].im);
  for (int k = 0; k < 2; k++) {
    uint4 q;
    __half2 *h = reinterpret_cast<__half2 *>(&q);
    for (int c = 0; c < 4; c++) {
      cplx<double> a = u[(4 * k + c) / 3][(4 * k + c) % 3];
      h[c] = __floats2half2_rn((float)a.re, (float)a.im);
    }
    h18[(gbase * 2 + k) * vh + i] = q;
  }
  {
    __half2 h = __floats2half2_rn((float)u[2][2].re, (float)u[2][2].im);
    reinterpret_cast<__half2 *>(h18 + 16 * vh)[gbase * vh + i] = h;
  }
  su3<double> w;
  for (int row = 0; row < 3; row++)
    for (int col = 0; col < 3; col++) w.m[row][col] = u[row][col];
  reconstruct_row2(w);
  double e = 0.0;
  for (int col = 0; col < 3; col++) {
    cplx<double> d = w.m[2][col] - u[2][col];
    e = fmax(e, sqrt(d.re * d.re + d.im * d.im));
  }
  atomic_max_pos(recon_err, e);
}

}  // namespace

// ---------------------------------------------------------------- launchers
template <int PD>
static void convert_dispatch(cudaStream_t s, const SpinorView &dst, int psrc, const SpinorView &src, size_t n) {
  if (psrc == PREC_DOUBLE) convert_kernel<PD, PREC_DOUBLE><<<blocks_for(n), TPB, 0, s>>>(dst, src, n);
  else if (psrc == PREC_SINGLE) convert_kernel<PD, PREC_SINGLE><<<blocks_for(n), TPB, 0, s>>>(dst, src, n);
  else convert_kernel<PD, PREC_HALF><<<blocks_for(n), TPB, 0, s>>>(dst, src, n);
}

void launch_convert(cudaStream_t s, int pdst, const SpinorView &dst, int psrc, const SpinorView &src) {
  size_t n = (size_t)src.vh * src.ls * src.nrhs;
  if (pdst == PREC_DOUBLE) convert_dispatch<PREC_DOUBLE>(s, dst, psrc, src, n);
  else if (pdst == PREC_SINGLE) convert_dispatch<PREC_SINGLE>(s, dst, psrc, src, n);
  else convert_dispatch<PREC_HALF>(s, dst, psrc, src, n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_axpby(cudaStream_t s, const SpinorView &out, double a, const SpinorView &x, const SpinorView &y) {
  size_t n = (size_t)x.vh * x.ls * x.nrhs;
  axpby_kernel<<<blocks_for(n), TPB, 0, s>>>(out, a, x, y, n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_axpby_dev(cudaStream_t s, const SpinorView &out, const double *a, double scale, const SpinorView &x,
                      const SpinorView &y) {
  size_t n = (size_t)x.vh * x.ls * x.nrhs;
  axpby_dev_kernel<<<blocks_for(n), TPB, 0, s>>>(out, a, scale, x, y, n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_scale(cudaStream_t s, double a, const SpinorView &f) {
  size_t n = (size_t)f.vh * f.ls * f.nrhs;
  scale_kernel<<<blocks_for(n), TPB, 0, s>>>(a, f, n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_zero(cudaStream_t s, const Field &f) {
  size_t n = f.sites();
  SpinorView v = f.view();
  if (f.prec == PREC_DOUBLE) zero_kernel<PREC_DOUBLE><<<blocks_for(n), TPB, 0, s>>>(v, n);
  else if (f.prec == PREC_SINGLE) zero_kernel<PREC_SINGLE><<<blocks_for(n), TPB, 0, s>>>(v, n);
  else zero_kernel<PREC_HALF><<<blocks_for(n), TPB, 0, s>>>(v, n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_xpay(cudaStream_t s, int prec, const SpinorView &p, const SpinorView &r, SolverScalars *st, int nrhs) {
  size_t per = (size_t)p.vh * p.ls;
  dim3 grid(blocks_for(per), nrhs);
  if (prec == PREC_DOUBLE) xpay_kernel<PREC_DOUBLE><<<grid, TPB, 0, s>>>(p, r, st, per);
  else if (prec == PREC_SINGLE) xpay_kernel<PREC_SINGLE><<<grid, TPB, 0, s>>>(p, r, st, per);
  else xpay_kernel<PREC_HALF><<<grid, TPB, 0, s>>>(p, r, st, per);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_accum_reliable(cudaStream_t s, const SpinorView &x64, int pxs, const SpinorView &xs, SolverScalars *st,
                           int nrhs, int force) {
  size_t per = (size_t)x64.vh * x64.ls;
  dim3 grid(blocks_for(per), nrhs);
  if (pxs == PREC_SINGLE) accum_kernel<PREC_SINGLE><<<grid, TPB, 0, s>>>(x64, xs, st, force);
  else if (pxs == PREC_DOUBLE) accum_kernel<PREC_DOUBLE><<<grid, TPB, 0, s>>>(x64, xs, st, force);
  else throw Error(-2, "accum: sloppy solution must be single or double");
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_norm(cudaStream_t s, int prec, const SpinorView &f, SolverScalars *st, double *partials, int op,
                 int gate) {
  size_t per = (size_t)f.vh * f.ls;
  dim3 grid(blocks_for(per), 1, f.nrhs);
  if (prec == PREC_DOUBLE) norm_kernel<PREC_DOUBLE><<<grid, TPB, 0, s>>>(f, st, partials, op, gate);
  else if (prec == PREC_SINGLE) norm_kernel<PREC_SINGLE><<<grid, TPB, 0, s>>>(f, st, partials, op, gate);
  else norm_kernel<PREC_HALF><<<grid, TPB, 0, s>>>(f, st, partials, op, gate);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
  launch_finalize(s, 1, partials, st, op, grid.x * grid.y, f.nrhs, gate);
}

void launch_finalize(cudaStream_t s, int nv, const double *partials, SolverScalars *st, int op, unsigned nblk,
                     int nsolves, int gate) {
  if (nv == 1) finalize_kernel<1><<<nsolves, FINALIZE_THREADS, 0, s>>>(partials, st, op, nblk, gate);
  else if (nv == 2) finalize_kernel<2><<<nsolves, FINALIZE_THREADS, 0, s>>>(partials, st, op, nblk, gate);
  else throw Error(-2, "finalize: 1 or 2 values per reduction");
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_init_scalars(cudaStream_t s, SolverScalars *st, int nrhs, const SolverScalars &init) {
  init_scalars_kernel<<<(nrhs + 63) / 64, 64, 0, s>>>(st, nrhs, init);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_import_fermion(cudaStream_t s, int prec, const SpinorView &dst, const double *staging) {
  size_t n = (size_t)dst.vh * dst.ls * dst.nrhs;
  if (prec == PREC_DOUBLE) import_kernel<PREC_DOUBLE><<<blocks_for(n), TPB, 0, s>>>(dst, staging, n);
  else if (prec == PREC_SINGLE) import_kernel<PREC_SINGLE><<<blocks_for(n), TPB, 0, s>>>(dst, staging, n);
  else import_kernel<PREC_HALF><<<blocks_for(n), TPB, 0, s>>>(dst, staging, n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_export_fermion(cudaStream_t s, int prec, const SpinorView &src, double *staging) {
  size_t n = (size_t)src.vh * src.ls * src.nrhs;
  if (prec == PREC_DOUBLE) export_kernel<PREC_DOUBLE><<<blocks_for(n), TPB, 0, s>>>(src, staging, n);
  else if (prec == PREC_SINGLE) export_kernel<PREC_SINGLE><<<blocks_for(n), TPB, 0, s>>>(src, staging, n);
  else export_kernel<PREC_HALF><<<blocks_for(n), TPB, 0, s>>>(src, staging, n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void launch_mix(const Dirac &D, int prec, const double *mix, const SpinorView &in, const SpinorView &out,
                const SolverScalars *st, int gate) {
  if (D.mix_tc && mix_tc_applies(D, prec)) {
    launch_mix_tc(D, mix, in, out, st, gate);
    return;
  }
  if (D.mix_bulk && launch_mix_bulk(D, prec, mix, in, out, st, gate)) return;
  if (D.mix_reg && launch_mix_reg(D, prec, mix, in, out, st, gate)) return;
  const int ls = D.ls;
  int bx = 256 / ls, p2 = 1;
  while (p2 * 2 <= bx) p2 *= 2;
  dim3 block(p2, ls);
  dim3 grid((unsigned)((in.vh + p2 - 1) / p2), 1, in.nrhs);
  size_t rs = prec == PREC_DOUBLE ? 8 : 4;
  size_t smem = (size_t)ls * p2 * 24 * rs + 2 * (size_t)ls * ls * sizeof(double) * (D.cplx ? 2 : 1);
  cudaStream_t s = D.lat->stream;
  if (prec == PREC_DOUBLE) {
    CPSGPU_CUDA(cudaFuncSetAttribute(mix_kernel<PREC_DOUBLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mix_kernel<PREC_DOUBLE><<<grid, block, smem, s>>>(in, out, mix, ls, st, gate, D.cplx ? 1 : 0);
  } else if (prec == PREC_SINGLE) {
    CPSGPU_CUDA(cudaFuncSetAttribute(mix_kernel<PREC_SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mix_kernel<PREC_SINGLE><<<grid, block, smem, s>>>(in, out, mix, ls, st, gate, D.cplx ? 1 : 0);
  } else {
    CPSGPU_CUDA(cudaFuncSetAttribute(mix_kernel<PREC_HALF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mix_kernel<PREC_HALF><<<grid, block, smem, s>>>(in, out, mix, ls, st, gate, D.cplx ? 1 : 0);
  }
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void import_gauge(Lattice &L, const double *host, int signs_applied) {
  const long vh = L.vh;
  const size_t nlinks = 8 * (size_t)vh;  // 2 parities x vh x 4
  L.staging.ensure(nlinks * 18 * sizeof(double));
  L.gD18.ensure(nlinks * 18 * sizeof(double));
  L.gD12.ensure(nlinks * 12 * sizeof(double));
  L.gS12.ensure(nlinks * 12 * sizeof(float));
  L.gH12.ensure(nlinks * 12 * sizeof(__half));
  L.gS18.ensure(nlinks * 18 * sizeof(float));
  L.gH18.ensure(nlinks * 18 * sizeof(__half));
  CPSGPU_CUDA(cudaMemcpyAsync(L.staging.ptr, host, nlinks * 18 * sizeof(double), cudaMemcpyHostToDevice, L.stream));
  DeviceBuffer err(sizeof(double));
  CPSGPU_CUDA(cudaMemsetAsync(err.ptr, 0, sizeof(double), L.stream));
  gauge_import_kernel<<<blocks_for(nlinks), TPB, 0, L.stream>>>(
      L.staging.as<double>(), vh, L.L[0], L.L[1], L.L[2], L.L[3], L.bc[0], L.bc[1], L.bc[2], L.bc[3],
      signs_applied, L.gD18.as<double2>(), L.gD12.as<double2>(), L.gS12.as<float4>(), L.gH12.as<uint2>(),
      L.gS18.as<float4>(), L.gH18.as<uint4>(), err.as<double>());
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
  double e = 0.0;
  CPSGPU_CUDA(cudaMemcpyAsync(&e, err.ptr, sizeof(double), cudaMemcpyDeviceToHost, L.stream));
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
  L.recon_err = e;
  // 12-real FP64 links only when the third row is rebuilt to FP64 accuracy
  L.use_recon12 = (e < 1e-14);
  L.have_gauge = true;
}

}  // namespace cpsgpu
