// Device-side timing used by the benchmark (cpsgpu_time_dslash / _mdagm).
#include <vector>

#include "../../include/cpsgpu.h"
#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

void gen_gaussian(double *out, long n, uint64_t seed, unsigned stream);

namespace {
size_t spinor_bytes(int prec) { return prec == PREC_DOUBLE ? 192 : prec == PREC_SINGLE ? 96 : 52; }
size_t link_bytes(int prec, int recon) {
  if (prec == PREC_DOUBLE) return recon == 18 ? 144 : 96;
  if (prec == PREC_SINGLE || recon == LINK_F32_18 || recon == LINK_F32_12)
    return (recon == 18 || recon == LINK_F32_18) ? 72 : 48;
  return recon == 18 ? 36 : 24;
}

// enough field pairs that the rotation's working set is > 2 x L2
int rotation(size_t pair_bytes) {
  const size_t l2 = 126ull << 20;
  int n = (int)((2 * l2) / (pair_bytes ? pair_bytes : 1)) + 1;
  return n < 2 ? 2 : (n > 16 ? 16 : n);
}

void fill(Lattice &L, Field &f) {
  size_t n = (size_t)24 * f.vh * f.ls * f.nrhs;
  std::vector<double> h(n);
  gen_gaussian(h.data(), (long)n, 12345, 7);
  L.staging.ensure(n * sizeof(double));
  CPSGPU_CUDA(cudaMemcpyAsync(L.staging.ptr, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, L.stream));
  launch_import_fermion(L.stream, f.prec, f.view(), L.staging.as<double>());
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
}
}  // namespace

double time_dslash(Dirac &D, int prec, int cb, int dag, int reps, double *bytes) {
  Lattice &L = *D.lat;
  const size_t sites = (size_t)L.vh * D.ls;
  const int rot = rotation(sites * 2 * spinor_bytes(prec));
  std::vector<Field> in(rot), out(rot);
  for (int k = 0; k < rot; k++) {
    in[k].create(prec, L.vh, D.ls, 1);
    out[k].create(prec, L.vh, D.ls, 1);
    fill(L, in[k]);
  }
  OpWork w;
  auto one = [&](int k) {
    if (D.kind == KIND_MOBIUS) {
      HopLaunch Lh;
      Lh.prec = prec;
      Lh.ep = EP_STORE;
      Lh.cb = cb;
      Lh.dag = dag;
      launch_hop(D, Lh, in[k].view(), out[k].view(), SpinorView(), SpinorView(), SpinorView(), SpinorView(),
                 SpinorView(), nullptr);
    } else {
      op_dslash(D, prec, out[k].view(), in[k].view(), cb, dag);
    }
  };
  for (int k = 0; k < 3; k++) one(k % rot);
  cudaEvent_t e0, e1;
  CPSGPU_CUDA(cudaEventCreate(&e0));
  CPSGPU_CUDA(cudaEventCreate(&e1));
  CPSGPU_CUDA(cudaEventRecord(e0, L.stream));
  for (int k = 0; k < reps; k++) one(k % rot);
  CPSGPU_CUDA(cudaEventRecord(e1, L.stream));
  CPSGPU_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  CPSGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (bytes) *bytes = (double)sites * 2 * spinor_bytes(prec) + 8.0 * L.vh * link_bytes(prec, L.recon(prec));
  return ms / reps;
}

// The standalone Mobius M5^-1 (dense Ls x Ls per chirality, CUDA cores,
// matrices in shared memory), timed like time_dslash.
double time_m5inv(Dirac &D, int prec, int reps, double *bytes) {
  if (D.kind != KIND_MOBIUS) throw Error(-2, "M5^-1 timing: Mobius operators only");
  Lattice &L = *D.lat;
  const size_t sites = (size_t)L.vh * D.ls;
  const int rot = rotation(sites * 2 * spinor_bytes(prec));
  std::vector<Field> in(rot), out(rot);
  for (int k = 0; k < rot; k++) {
    in[k].create(prec, L.vh, D.ls, 1);
    out[k].create(prec, L.vh, D.ls, 1);
    fill(L, in[k]);
  }
  for (int k = 0; k < 3; k++) op_mobius_m5inv(D, prec, out[k % rot].view(), in[k % rot].view(), 0);
  cudaEvent_t e0, e1;
  CPSGPU_CUDA(cudaEventCreate(&e0));
  CPSGPU_CUDA(cudaEventCreate(&e1));
  CPSGPU_CUDA(cudaEventRecord(e0, L.stream));
  for (int k = 0; k < reps; k++) op_mobius_m5inv(D, prec, out[k % rot].view(), in[k % rot].view(), 0);
  CPSGPU_CUDA(cudaEventRecord(e1, L.stream));
  CPSGPU_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  CPSGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (bytes) *bytes = (double)sites * 2 * spinor_bytes(prec);
  return ms / reps;
}

double time_mdagm(Dirac &D, int prec, int reps, double *bytes) {
  Lattice &L = *D.lat;
  const size_t sites = (size_t)L.vh * D.ls;
  const int rot = rotation(sites * 2 * spinor_bytes(prec));
  std::vector<Field> in(rot), out(rot);
  for (int k = 0; k < rot; k++) {
    in[k].create(prec, L.vh, D.ls, 1);
    out[k].create(prec, L.vh, D.ls, 1);
    fill(L, in[k]);
  }
  OpWork w;
  SolverScalars *st = L.scratch_st.as<SolverScalars>();
  CPSGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(SolverScalars), L.stream));
  for (int k = 0; k < 2; k++) op_mdagm(D, prec, out[k % rot].view(), in[k % rot].view(), w, st, RED_STORE);
  cudaEvent_t e0, e1;
  CPSGPU_CUDA(cudaEventCreate(&e0));
  CPSGPU_CUDA(cudaEventCreate(&e1));
  CPSGPU_CUDA(cudaEventRecord(e0, L.stream));
  for (int k = 0; k < reps; k++) op_mdagm(D, prec, out[k % rot].view(), in[k % rot].view(), w, st, RED_STORE);
  CPSGPU_CUDA(cudaEventRecord(e1, L.stream));
  CPSGPU_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  CPSGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (bytes) {
    const double sp = (double)sites * spinor_bytes(prec);
    const double links = 8.0 * L.vh * link_bytes(prec, L.recon(prec));
    // 4 hops (in + out + links); the two axpby epilogues read one more field;
    // Mobius adds the standalone mixing pass (in + out)
    double b = 4 * (2 * sp + links) + 2 * sp;
    if (D.kind == KIND_MOBIUS) b += 2 * sp;
    *bytes = b;
  }
  return ms / reps;
}

}  // namespace cpsgpu
