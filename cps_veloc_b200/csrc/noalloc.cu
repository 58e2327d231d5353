// MatPcDagMatPc on caller-owned device memory, with every temporary in one
// fixed, statically allocated device array (cpsgpu_matpc_dag_matpc_noalloc).
//
// Some callers cannot call cudaMalloc at the point where they apply the
// operator: a host code that has handed all device memory to its own pool
// allocator (a new cudaMalloc can fail or fragment that pool), or a caller
// inside a latency-critical loop that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree imply.  This variant takes the input
// and output as device pointers and keeps its two intermediate fields, the
// per-block reduction partials and the reduction scalars in the file-scope
// array below, so a call allocates nothing.
//
// Limits and caveats (also stated in include/cpsgpu.h):
//   * the array holds NOALLOC_SCRATCH_BYTES on every GPU that loads the
//     library, for the life of the process;
//   * two FP64 fields of the operator must fit in it (see noalloc_fits);
//   * every call shares the one array: calls whose kernels overlap on the GPU
//     (several host threads, several streams) race and corrupt each other;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress); make that first call before any stream capture;
//   * a call runs on the operator's lattice's device (made current for the
//     call, the caller's current device restored after it).
#include <cstring>
#include <mutex>

#include "cpsgpu_impl.h"
#include "hop.cuh"
#include "tune.h"

namespace cpsgpu {

constexpr size_t NOALLOC_SCRATCH_BYTES = 64ull << 20;  // 64 MiB per GPU

// The scratch.  In host code this name is only a host-side stand-in for the
// device symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
unsigned char *g_scratch_addr[MAX_DEVICES] = {nullptr};

// Makes `dev` the calling thread's current device for a scope and restores
// the caller's device afterwards: the scratch address is per device, and the
// kernels run on the lattice's stream, which belongs to the lattice's device.
struct CurrentDevice {
  int saved = -1;
  explicit CurrentDevice(int dev) {
    CPSGPU_CUDA(cudaGetDevice(&saved));
    if (saved != dev) CPSGPU_CUDA(cudaSetDevice(dev));
  }
  ~CurrentDevice() {
    int now = -1;
    if (cudaGetDevice(&now) == cudaSuccess && now != saved) cudaSetDevice(saved);
  }
};

// device address of the scratch on device dev, which must be current
// (looked up once per device)
unsigned char *scratch_address(int dev) {
  if (dev < 0 || dev >= MAX_DEVICES) throw Error(-2, "noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error(-3, std::string("noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<unsigned char *>(p);
  }
  return g_scratch_addr[dev];
}

size_t round_up(size_t n) { return (n + 255) & ~size_t(255); }

struct Carve {
  size_t scalars, partials, field, total;
};

// scratch layout: [SolverScalars][partials][t1][t2]
Carve carve(const Dirac &D) {
  const size_t sites = (size_t)D.lat->vh * D.ls;
  // blocks of the reducing launch (two partial sums each), as hop() sizes it
  const dim3 b = hop_block(TuneKey{PREC_DOUBLE, D.lat->recon(PREC_DOUBLE), EP_AXPY, D.kind, D.ls}, false);
  const size_t nblk = (size_t)((D.lat->vh + b.x - 1) / b.x) * ((D.ls + b.y - 1) / b.y);
  Carve c;
  c.scalars = round_up(sizeof(SolverScalars));
  c.partials = round_up(nblk * 2 * sizeof(double));
  c.field = round_up(sites * 192);
  c.total = c.scalars + c.partials + 2 * c.field;
  return c;
}

using HopFn = void (*)(const HopParams, const HopViews, SolverScalars *, double *);

template <int RECON, int EP, bool DAG>
HopFn fn() {
  return hop_kernel<PREC_DOUBLE, RECON, EP, PREC_DOUBLE, PREC_DOUBLE, DAG>;
}

HopFn pick(int recon, int ep, int dag) {
  if (recon == 18) {
    if (ep == EP_STORE) return dag ? fn<18, EP_STORE, true>() : fn<18, EP_STORE, false>();
    return dag ? fn<18, EP_AXPY, true>() : fn<18, EP_AXPY, false>();
  }
  if (ep == EP_STORE) return dag ? fn<12, EP_STORE, true>() : fn<12, EP_STORE, false>();
  return dag ? fn<12, EP_AXPY, true>() : fn<12, EP_AXPY, false>();
}

// one FP64 hop of the Wilson / DWF operator (the parameters launch_hop
// would set), reducing into st/partials when norm is set
void hop(const Dirac &D, int ep, int cb, int dag, int norm, const SpinorView &in, const SpinorView &out,
         const SpinorView &x, SolverScalars *st, double *partials) {
  const Lattice &lat = *D.lat;
  HopParams hp;
  memset(&hp, 0, sizeof(hp));
  for (int k = 0; k < 4; k++) {
    hp.L[k] = lat.L[k];
    hp.bc[k] = lat.bc[k];
  }
  hp.hx = lat.L[0] / 2;
  hp.dhx.init(hp.hx);
  hp.dly.init(lat.L[1]);
  hp.dlz.init(lat.L[2]);
  hp.vh = lat.vh;
  hp.iend = (int)lat.vh;  // every site
  hp.ls = D.ls;
  hp.cb = cb;
  hp.dag = dag;
  hp.dwf = (D.kind == KIND_DWF);
  hp.h5 = 2.0 * D.a5inv;
  hp.h5wall = -2.0 * D.mass * D.a5inv;
  for (int s = 0; s < D.ls && s < MAX_LS; s++) hp.coef[s] = -D.kappa * D.kappa;
  hp.norm = norm;
  hp.red_op = RED_STORE;
  hp.gate = GATE_NONE;
  HopViews v;
  v.U = lat.gauge(PREC_DOUBLE);
  v.in = in;
  v.out = out;
  v.x = x;
  const int recon = lat.recon(PREC_DOUBLE);
  dim3 block = hop_block(TuneKey{PREC_DOUBLE, recon, ep, D.kind, D.ls}, false);
  block.z = 1;  // one slice per thread here (a tuned z of 2 selects launch_hop's slice pairs)
  const unsigned nsb = (unsigned)((lat.vh + block.x - 1) / block.x);
  hp.nsg = (D.ls + block.y - 1) / block.y;
  hp.rtile = 1;
  hp.nrhs = 1;
  dim3 grid(nsb * hp.nsg, 1, 1);
  pick(recon, ep, dag)<<<grid, block, 0, lat.stream>>>(hp, v, st, partials);
  CPSGPU_CUDA(cudaGetLastError());
  if (norm) {  // sum the per-block partials of |out|^2, |x|^2 into st->sum
    finalize_kernel<2><<<1, FINALIZE_THREADS, 0, lat.stream>>>(partials, st, RED_STORE, grid.x, GATE_NONE);
    CPSGPU_CUDA(cudaGetLastError());
  }
}

SpinorView view_of(void *p, const Dirac &D) {
  SpinorView v;
  v.data = p;
  v.vh = D.lat->vh;
  v.ls = D.ls;
  v.nrhs = 1;
  return v;
}

}  // namespace

size_t noalloc_scratch_bytes() { return NOALLOC_SCRATCH_BYTES; }

bool noalloc_fits(const Dirac &D) { return carve(D).total <= NOALLOC_SCRATCH_BYTES; }

// out = MatPc^+ MatPc in, returns |MatPc in|^2; in and out are device
// pointers in the library's FP64 field layout.  Wilson and DWF operators.
double matpc_dag_matpc_noalloc(const Dirac &D, double *out, const double *in) {
  if (D.kind == KIND_MOBIUS) throw Error(-2, "noalloc: Mobius is not supported (Wilson and DWF only)");
  const Carve c = carve(D);
  if (c.total > NOALLOC_SCRATCH_BYTES)
    throw Error(-1, "noalloc: operator needs " + std::to_string(c.total >> 20) + " MiB of scratch, more than the " +
                        std::to_string(NOALLOC_SCRATCH_BYTES >> 20) + " MiB available (two FP64 fields must fit)");
  // the lattice's device, whatever the caller's current device is
  CurrentDevice on(D.lat->device);
  unsigned char *base = scratch_address(D.lat->device);
  SolverScalars *st = reinterpret_cast<SolverScalars *>(base);
  double *partials = reinterpret_cast<double *>(base + c.scalars);
  void *t1 = base + c.scalars + c.partials;
  void *t2 = base + c.scalars + c.partials + c.field;
  cudaStream_t s = D.lat->stream;
  // the array keeps the previous call's contents: start from zeroed scalars
  CPSGPU_CUDA(cudaMemsetAsync(st, 0, sizeof(SolverScalars), s));
  const SpinorView vin = view_of(const_cast<double *>(in), D), vout = view_of(out, D);
  const SpinorView v1 = view_of(t1, D), v2 = view_of(t2, D);
  // MatPc: t2 = in - kappa^2 D0 D1 in, with |t2|^2
  hop(D, EP_STORE, 1, 0, 0, vin, v1, SpinorView(), st, partials);
  hop(D, EP_AXPY, 0, 0, 1, v1, v2, vin, st, partials);
  // MatPc^dagger: out = t2 - kappa^2 D0^+ D1^+ t2
  hop(D, EP_STORE, 1, 1, 0, v2, v1, SpinorView(), st, partials);
  hop(D, EP_AXPY, 0, 1, 0, v1, vout, v2, st, partials);
  double dot = 0.0;
  CPSGPU_CUDA(cudaMemcpyAsync(&dot, &st->sum[0], sizeof(double), cudaMemcpyDeviceToHost, s));
  CPSGPU_CUDA(cudaStreamSynchronize(s));
  return dot;
}

}  // namespace cpsgpu
