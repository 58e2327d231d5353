// Low-mode deflation: the eigenvector cache and DiracOp::InvLowModeApprox.
//
// The reference keeps eigenvectors (float) and eigenvalues in a global list
// of EigenCache objects found by name and count (util/eigen_container.h,
// EigenCacheListSearch), filled from disk by EigenContainer.  Here the
// cache lives on the lattice, resident in HBM as FP32 fields in the
// library's layout, filled by the caller from host vectors.
//
// InvLowModeApprox (d_op_base/comsrc/inv_lowmode_approx.C:272-512) is
//   out_i = sum_k (<v_k, in_i> / lambda_k) v_k,   k < neig,
// for len sources at once: one kernel computes every <v_k, in_i> (per-block
// partial sums, then a fixed-order sum over the blocks), the host divides by
// lambda_k, one kernel accumulates the sums in the reference's k order.
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

struct EigenCacheDev {
  std::string name;
  int neig = 0;
  std::vector<double> evals;
  std::vector<Field> evecs;  // FP32, the operator's half-checkerboard fields
  DeviceBuffer ptrs;         // device array of the evecs' data pointers
};

namespace {

constexpr int LM_TPB = 128;
constexpr int LM_NS = 8;  // sources per dot-product launch

struct LmSources {
  SpinorView s[LM_NS];
  int ns;
};

// per (site block, eigenvector k): partial sums of <v_k, in_i> over the
// block's sites for the ns sources, (re, im) pairs
__global__ void __launch_bounds__(LM_TPB) lowmode_dot_kernel(const float *const *evecs, long vh, int ls, LmSources src,
                                                             double *partials) {
  const int k = blockIdx.y;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v[2 * LM_NS];
#pragma unroll
  for (int q = 0; q < 2 * LM_NS; q++) v[q] = 0.0;
  if (idx < (size_t)vh * ls) {
    const long sl = (long)(idx / vh), i = (long)(idx % vh);
    SpinorView ev;
    ev.data = (void *)evecs[k];
    ev.vh = vh;
    ev.ls = ls;
    float e[24];
    SpinorIO<PREC_SINGLE>::load(ev, sl, i, e);
#pragma unroll
    for (int q = 0; q < LM_NS; q++) {
      if (q < src.ns) {
        double x[24];
        SpinorIO<PREC_DOUBLE>::load(src.s[q], sl, i, x);
#pragma unroll
        for (int c = 0; c < 24; c += 2) {
          v[2 * q] += (double)e[c] * x[c] + (double)e[c + 1] * x[c + 1];
          v[2 * q + 1] += (double)e[c] * x[c + 1] - (double)e[c + 1] * x[c];
        }
      }
    }
  }
  block_partial<2 * LM_NS>(v, partials, (unsigned)k, blockIdx.x, gridDim.x);
}

// sums[k][q] = sum over blocks of partials[k][blk][q], blocks in order
__global__ void lowmode_sum_kernel(const double *partials, unsigned nblk, double *sums) {
  const int k = blockIdx.x, q = threadIdx.x;
  if (q >= 2 * LM_NS) return;
  const double *p = partials + (size_t)k * nblk * (2 * LM_NS) + q;
  double s = 0.0;
  for (unsigned b = 0; b < nblk; b++) s += p[(size_t)b * (2 * LM_NS)];
  sums[(size_t)k * (2 * LM_NS) + q] = s;
}

// out = sum_k coef[k] v_k (coef complex, (re, im)), k in order; a thread per 5D site
__global__ void __launch_bounds__(LM_TPB) lowmode_accum_kernel(const float *const *evecs, long vh, int ls, int neig,
                                                               const double *coef, SpinorView out) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)vh * ls) return;
  const long sl = (long)(idx / vh), i = (long)(idx % vh);
  double acc[24];
#pragma unroll
  for (int c = 0; c < 24; c++) acc[c] = 0.0;
  SpinorView ev;
  ev.vh = vh;
  ev.ls = ls;
  for (int k = 0; k < neig; k++) {
    ev.data = (void *)evecs[k];
    float e[24];
    SpinorIO<PREC_SINGLE>::load(ev, sl, i, e);
    const double zr = coef[2 * k], zi = coef[2 * k + 1];
#pragma unroll
    for (int c = 0; c < 24; c += 2) {
      acc[c] += zr * e[c] - zi * e[c + 1];
      acc[c + 1] += zr * e[c + 1] + zi * e[c];
    }
  }
  SpinorIO<PREC_DOUBLE>::store(out, sl, i, acc);
}

}  // namespace

// Store neig FP32 eigenvectors (already uploaded into fields) and their
// eigenvalues under name, replacing a cache of the same name.
void eigencache_store(Lattice &L, const std::string &name, std::vector<Field> &&evecs, const double *evals) {
  auto c = std::make_shared<EigenCacheDev>();
  c->name = name;
  c->neig = (int)evecs.size();
  c->evals.assign(evals, evals + c->neig);
  c->evecs = std::move(evecs);
  std::vector<const void *> p(c->neig);
  for (int k = 0; k < c->neig; k++) p[k] = c->evecs[k].data.ptr;
  c->ptrs.alloc(sizeof(void *) * std::max(1, c->neig));
  CPSGPU_CUDA(cudaMemcpy(c->ptrs.ptr, p.data(), sizeof(void *) * c->neig, cudaMemcpyHostToDevice));
  for (auto &e : L.eig_caches)
    if (e->name == name) {
      e = c;
      return;
    }
  L.eig_caches.push_back(c);
}

void eigencache_clear(Lattice &L) { L.eig_caches.clear(); }

// EigenCacheListSearch (eigen_container.h:432): the cache of this name
// holding exactly neig vectors, or null
static EigenCacheDev *eigencache_find(Lattice &L, const std::string &name, int neig) {
  for (auto &e : L.eig_caches)
    if (e->name == name && e->neig == neig) return e.get();
  return nullptr;
}

// DiracOp::InvLowModeApprox (inv_lowmode_approx.C:272-512, the uncompressed
// cache's path): out_i = sum_k (<v_k, in_i> / lambda_k) v_k.  square: the
// RitzMatOper is MAT_HERM / MATPC_HERM, whose cached eigenvalues are
// squared first (the reference squares them in the cache itself, so a second
// call would square them again; here a copy is squared).
void inv_lowmode_approx(Dirac &D, const std::vector<SpinorView> &out, const std::vector<SpinorView> &in,
                        const std::string &name, int neig, bool square) {
  Lattice &L = *D.lat;
  cudaStream_t s = L.stream;
  EigenCacheDev *c = eigencache_find(L, name, neig);
  if (!c) throw Error(-1, "eigenvector cache does not exist: " + name + " with " + std::to_string(neig) + " vectors");
  if (!c->evecs.empty() && (c->evecs[0].vh != L.vh || c->evecs[0].ls != D.ls))
    throw Error(-1, "eigenvector cache " + name + " was stored for another operator size");
  std::vector<double> ev(c->evals);
  if (square)
    for (double &x : ev) x = x * x;
  const int len = (int)in.size();
  const size_t sites = (size_t)L.vh * D.ls;
  const unsigned nblk = (unsigned)((sites + LM_TPB - 1) / LM_TPB);
  DeviceBuffer part, sums, coef;
  part.alloc(sizeof(double) * (size_t)std::max(1, neig) * nblk * 2 * LM_NS);
  sums.alloc(sizeof(double) * (size_t)std::max(1, neig) * 2 * LM_NS);
  coef.alloc(sizeof(double) * (size_t)std::max(1, neig) * 2);
  std::vector<double> z((size_t)std::max(1, neig) * 2 * LM_NS), cf((size_t)std::max(1, neig) * 2);
  for (int i0 = 0; i0 < len; i0 += LM_NS) {
    const int ns = std::min(LM_NS, len - i0);
    if (neig > 0) {
      LmSources src;
      memset(&src, 0, sizeof(src));
      src.ns = ns;
      for (int q = 0; q < ns; q++) src.s[q] = in[i0 + q];
      lowmode_dot_kernel<<<dim3(nblk, neig), LM_TPB, 0, s>>>(c->ptrs.as<const float *>(), L.vh, D.ls, src,
                                                              part.as<double>());
      CPSGPU_CUDA(cudaGetLastError());
      launch_counter()++;
      lowmode_sum_kernel<<<neig, 32, 0, s>>>(part.as<double>(), nblk, sums.as<double>());
      CPSGPU_CUDA(cudaGetLastError());
      launch_counter()++;
      CPSGPU_CUDA(cudaMemcpyAsync(z.data(), sums.ptr, sizeof(double) * neig * 2 * LM_NS, cudaMemcpyDeviceToHost, s));
      CPSGPU_CUDA(cudaStreamSynchronize(s));
    }
    for (int q = 0; q < ns; q++) {
      for (int k = 0; k < neig; k++) {
        cf[2 * k] = z[(size_t)k * 2 * LM_NS + 2 * q] / ev[k];
        cf[2 * k + 1] = z[(size_t)k * 2 * LM_NS + 2 * q + 1] / ev[k];
      }
      if (neig > 0)
        CPSGPU_CUDA(cudaMemcpyAsync(coef.ptr, cf.data(), sizeof(double) * 2 * neig, cudaMemcpyHostToDevice, s));
      lowmode_accum_kernel<<<nblk, LM_TPB, 0, s>>>(c->ptrs.as<const float *>(), L.vh, D.ls, neig, coef.as<double>(),
                                                   out[i0 + q]);
      CPSGPU_CUDA(cudaGetLastError());
      launch_counter()++;
      CPSGPU_CUDA(cudaStreamSynchronize(s));
    }
  }
}

}  // namespace cpsgpu
