// t-slab domain decomposition of the hop (one nearest-neighbour exchange
// per dslash), replacing the reference's QMP halo of wilson_dslash_vec
// (d_op_wilson/qmp/wilson_dslash_vec.C:184-278, 486-493).
//
// Each rank holds a slab of Lt / nodes_t t-slices (an even number, so the
// local checkerboard parity is the global one).  Before a dslash a rank
// packs, per slice of the input field, two faces of half spinors:
//   to_prev: (1 - sdag g_t) psi of its first t-slice, which the previous
//            slab's forward t hop multiplies by its own link;
//   to_next: U_t^dagger (1 + sdag g_t) psi of its last t-slice, with its own
//            links: the next slab's backward t hop only reconstructs it;
// so no gauge halo is exchanged and each face is 12 reals per site and
// slice.  The caller moves to_prev to the previous rank (its from_next) and
// to_next to the next rank (its from_prev), by NCCL, peer copies or MPI;
// the hop kernel then reads them at its t ends (hop.cuh).  The lattice's
// antiperiodic t sign applies only at the slab ends that are the lattice's
// own boundary.  To overlap the exchange with the hop, the interior
// t-slices (which read no halo) can be launched before the faces arrive
// and the two end slices after (the wilson_dslash_vec split of local and
// non-local parts, wilson_dslash_vec.C:184-278).
#include <cstring>

#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

namespace {

template <typename R>
__device__ __forceinline__ void store_halo(R *p, int face, long sl, int f, const half_spinor<R> &h) {
  R *q = p + (size_t)sl * 12 * face + f;
#pragma unroll
  for (int sp = 0; sp < 2; sp++)
#pragma unroll
    for (int col = 0; col < 3; col++) {
      const int k = 2 * (col + 3 * sp);
      q[(size_t)k * face] = h.h[sp][col].re;
      q[(size_t)(k + 1) * face] = h.h[sp][col].im;
    }
}

// a thread per (face site f, slice sl of every right-hand side)
template <int P, int RECON, bool DAG>
__global__ void face_pack_kernel(const HopParams hp, const GaugeView U, const SpinorView in,
                                 typename PrecTraits<P>::real *to_prev, typename PrecTraits<P>::real *to_next) {
  using R = typename PrecTraits<P>::real;
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const long sl = blockIdx.y;
  if (f >= hp.face) return;
  const int s = (int)(sl % hp.ls);
  const int pin = hp.dwf ? ((s + hp.cb) & 1) : hp.cb;
  constexpr R sdag = DAG ? R(-1) : R(1);
  const Slice<P> sin(in, sl);
  R psi[24], sc;
  sin.load_raw(f, psi, sc);  // first t-slice: checkerboard index f
  store_halo(to_prev, hp.face, sl, f, project(psi, 3, -sdag));
  const int j = (hp.L[3] - 1) * hp.face + f;  // last t-slice
  sin.load_raw(j, psi, sc);
  su3<R> u;
  LinkIO<P, RECON>::load(U, pin, 3, j, u);
  store_halo(to_next, hp.face, sl, f, link_mul(u, project(psi, 3, sdag), true));
}

template <int P, int RECON>
void pack_dispatch(bool dag, dim3 grid, cudaStream_t s, const HopParams &hp, const GaugeView &U, const SpinorView &in,
                   void *to_prev, void *to_next) {
  using R = typename PrecTraits<P>::real;
  if (dag)
    face_pack_kernel<P, RECON, true><<<grid, 128, 0, s>>>(hp, U, in, (R *)to_prev, (R *)to_next);
  else
    face_pack_kernel<P, RECON, false><<<grid, 128, 0, s>>>(hp, U, in, (R *)to_prev, (R *)to_next);
}

void check_dd(const Dirac &D, int prec) {
  const Lattice &L = *D.lat;
  if (L.t_nodes < 2) throw Error(-4, "the lattice is not t-partitioned");
  if (prec != PREC_DOUBLE && prec != PREC_SINGLE) throw Error(-2, "decomposed dslash: FP64 or FP32 fields");
  const int recon = L.recon(prec);
  if (recon != 12 && recon != 18) throw Error(-2, "decomposed dslash: 12- or 18-real links");
}

}  // namespace

size_t dd_face_bytes(const Dirac &D, int prec, int nrhs) {
  check_dd(D, prec);  // the sizes only of configurations the decomposed dslash runs
  const Lattice &L = *D.lat;
  return (size_t)(L.vh / L.L[3]) * 12 * D.ls * nrhs * (prec == PREC_DOUBLE ? 8 : 4);
}

void dd_pack(const Dirac &D, int prec, const SpinorView &in, int cb, int dag, void *to_prev, void *to_next) {
  check_dd(D, prec);
  const Lattice &L = *D.lat;
  HopParams hp;
  memset(&hp, 0, sizeof(hp));
  for (int k = 0; k < 4; k++) hp.L[k] = L.L[k];
  hp.face = (int)(L.vh / L.L[3]);
  hp.ls = D.ls;
  hp.cb = cb;
  hp.dwf = (D.kind == KIND_DWF);
  const dim3 grid((unsigned)((hp.face + 127) / 128), (unsigned)(D.ls * in.nrhs));
  const GaugeView U = L.gauge(prec);
  const bool recon12 = (L.recon(prec) == 12);
  if (prec == PREC_DOUBLE) {
    if (recon12) pack_dispatch<PREC_DOUBLE, 12>(dag, grid, L.stream, hp, U, in, to_prev, to_next);
    else pack_dispatch<PREC_DOUBLE, 18>(dag, grid, L.stream, hp, U, in, to_prev, to_next);
  } else {
    if (recon12) pack_dispatch<PREC_SINGLE, 12>(dag, grid, L.stream, hp, U, in, to_prev, to_next);
    else pack_dispatch<PREC_SINGLE, 18>(dag, grid, L.stream, hp, U, in, to_prev, to_next);
  }
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void dd_dslash(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int cb, int dag,
               const void *from_next, const void *from_prev, int sub) {
  check_dd(D, prec);
  if (sub < SUB_ALL || sub > SUB_BOUNDARY) throw Error(-1, "bad site subset");
  HopLaunch L;
  L.prec = prec;
  L.ep = EP_STORE;
  L.cb = cb;
  L.dag = dag;
  L.halo_fwd = from_next;
  L.halo_bwd = from_prev;
  L.sub = sub;
  launch_hop(D, L, in, out, SpinorView(), SpinorView(), SpinorView(), SpinorView(), SpinorView(), nullptr);
}

namespace {
// per-block partials of the local <a, b> of two FP64 fields, a thread per 5D site
__global__ void field_dot_kernel(SpinorView a, SpinorView b, double *partials, size_t n) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0.0, 0.0};
  if (idx < n) {
    const long sl = (long)(idx / a.vh), i = (long)(idx % a.vh);
    double x[24], y[24];
    SpinorIO<PREC_DOUBLE>::load(a, sl, i, x);
    SpinorIO<PREC_DOUBLE>::load(b, sl, i, y);
#pragma unroll
    for (int k = 0; k < 24; k += 2) {
      v[0] += x[k] * y[k] + x[k + 1] * y[k + 1];
      v[1] += x[k] * y[k + 1] - x[k + 1] * y[k];
    }
  }
  block_partial<2>(v, partials);
}
}  // namespace

// this rank's part of <a, b> (sum conj(a) b) over FP64 fields: the decomposed
// solvers add the ranks' parts themselves
// the same into dev_out[0..1] (device memory), enqueued on the lattice's stream
void field_dot_device(Lattice &L, const SpinorView &a, const SpinorView &b, double *dev_out) {
  const size_t n = (size_t)a.vh * a.ls * a.nrhs;
  const unsigned nblk = (unsigned)((n + 255) / 256);
  L.partials.ensure((size_t)nblk * 2 * sizeof(double));
  SolverScalars *st = L.scratch_st.as<SolverScalars>();
  field_dot_kernel<<<nblk, 256, 0, L.stream>>>(a, b, L.partials.as<double>(), n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
  launch_finalize(L.stream, 2, L.partials.as<double>(), st, RED_STORE, nblk, 1, GATE_NONE);
  CPSGPU_CUDA(cudaMemcpyAsync(dev_out, st->sum, 2 * sizeof(double), cudaMemcpyDeviceToDevice, L.stream));
}

void field_dot(Lattice &L, const SpinorView &a, const SpinorView &b, double *re, double *im) {
  const size_t n = (size_t)a.vh * a.ls * a.nrhs;
  const unsigned nblk = (unsigned)((n + 255) / 256);
  L.partials.ensure((size_t)nblk * 2 * sizeof(double));
  SolverScalars *st = L.scratch_st.as<SolverScalars>();
  field_dot_kernel<<<nblk, 256, 0, L.stream>>>(a, b, L.partials.as<double>(), n);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
  launch_finalize(L.stream, 2, L.partials.as<double>(), st, RED_STORE, nblk, 1, GATE_NONE);
  double s[2];
  CPSGPU_CUDA(cudaMemcpyAsync(s, st->sum, sizeof(s), cudaMemcpyDeviceToHost, L.stream));
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
  *re = s[0];
  *im = s[1];
}

}  // namespace cpsgpu
