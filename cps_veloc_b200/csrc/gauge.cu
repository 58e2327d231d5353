// Gauge-field observables on the resident links: the plaquette and the link
// trace as the reference's Lattice::SumReTrPlaq (lattice_base.C:2878-3060,
// ReTrPlaq of every site and plane mu < nu) and the link-trace sum of
// ReadLatticeParallel::CheckPlaqLinktrace (ReadLatticePar.C), used by the
// NERSC reader's check and writer's header.  The links read are the FP64
// 18-real copy, which carries no boundary signs (as the reference's field
// outside a DiracOp's scope).
#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

namespace {

constexpr int GTPB = 256;

struct GaugeGeom {
  int L[4];
  int hx;
  long vh;
};

__device__ __forceinline__ void mat_mul(cplx<double> (&c)[3][3], const su3<double> &a, const su3<double> &b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        re = fma(a.m[i][k].re, b.m[k][j].re, fma(-a.m[i][k].im, b.m[k][j].im, re));
        im = fma(a.m[i][k].re, b.m[k][j].im, fma(a.m[i][k].im, b.m[k][j].re, im));
      }
      c[i][j] = {re, im};
    }
}

// thread per (checkerboard site, parity), the two parities of a site block
// in consecutive blocks (their links are each other's neighbours): sum over mu < nu of
// Re tr[U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag] and sum over mu of Re tr U_mu(x)
__global__ void __launch_bounds__(GTPB) plaq_kernel(const GaugeGeom g, const GaugeView U, double *partials) {
  const int i = (blockIdx.x >> 1) * blockDim.x + threadIdx.x;
  const int p = blockIdx.x & 1;
  double v[2] = {0.0, 0.0};
  if (i < g.vh) {
    int r = i / g.hx;
    const int xh = i - r * g.hx;
    const int y = r % g.L[1];
    r /= g.L[1];
    const int z = r % g.L[2];
    const int t = r / g.L[2];
    const int x = 2 * xh + ((y + z + t + p) & 1);
    const int c[4] = {x, y, z, t};
    // checkerboard index of x + mu (parity 1 - p)
    int fwd[4];
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      const bool wrap = (c[mu] == g.L[mu] - 1);
      const int stride = mu == 1 ? g.hx : mu == 2 ? g.hx * g.L[1] : g.hx * g.L[1] * g.L[2];
      if (mu == 0) fwd[mu] = i - xh + ((wrap ? 0 : x + 1) >> 1);
      else fwd[mu] = wrap ? i - (g.L[mu] - 1) * stride : i + stride;
    }
    su3<double> u[4];
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      LinkIO<PREC_DOUBLE, 18>::load(U, p, mu, i, u[mu]);
      v[1] += u[mu].m[0][0].re + u[mu].m[1][1].re + u[mu].m[2][2].re;
    }
#pragma unroll
    for (int mu = 0; mu < 3; mu++)
#pragma unroll
      for (int nu = mu + 1; nu < 4; nu++) {
        su3<double> a, b;
        LinkIO<PREC_DOUBLE, 18>::load(U, 1 - p, nu, fwd[mu], a);  // U_nu(x + mu)
        LinkIO<PREC_DOUBLE, 18>::load(U, 1 - p, mu, fwd[nu], b);  // U_mu(x + nu)
        cplx<double> m1[3][3], m2[3][3];
        mat_mul(m1, u[mu], a);  // U_mu(x) U_nu(x+mu)
        mat_mul(m2, u[nu], b);  // U_nu(x) U_mu(x+nu)
        // Re tr[m1 m2^dag] = sum_ij Re(m1_ij conj(m2_ij))
        double s = 0.0;
#pragma unroll
        for (int a2 = 0; a2 < 3; a2++)
#pragma unroll
          for (int b2 = 0; b2 < 3; b2++) s = fma(m1[a2][b2].re, m2[a2][b2].re, fma(m1[a2][b2].im, m2[a2][b2].im, s));
        v[0] += s;
      }
  }
  block_partial<2>(v, partials, 0, blockIdx.x, gridDim.x);
}

}  // namespace

void gauge_sums(Lattice &L, double *sum_plaq, double *sum_link) {
  if (!L.have_gauge) throw Error(-1, "no gauge field imported");
  if (L.t_nodes > 1) throw Error(-4, "t-partitioned lattice: the plaquette needs the whole lattice");
  GaugeGeom g;
  for (int k = 0; k < 4; k++) g.L[k] = L.L[k];
  g.hx = L.L[0] / 2;
  g.vh = L.vh;
  GaugeView U;
  U.data = L.gD18.ptr;
  U.vh = L.vh;
  const unsigned nblk = 2 * (unsigned)((L.vh + GTPB - 1) / GTPB);
  const dim3 grid(nblk);
  L.partials.ensure((size_t)nblk * 2 * sizeof(double));
  SolverScalars *st = L.scratch_st.as<SolverScalars>();
  plaq_kernel<<<grid, GTPB, 0, L.stream>>>(g, U, L.partials.as<double>());
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
  launch_finalize(L.stream, 2, L.partials.as<double>(), st, RED_STORE, nblk, 1, GATE_NONE);
  double s[2];
  CPSGPU_CUDA(cudaMemcpyAsync(s, st->sum, sizeof(s), cudaMemcpyDeviceToHost, L.stream));
  CPSGPU_CUDA(cudaStreamSynchronize(L.stream));
  if (sum_plaq) *sum_plaq = s[0];
  if (sum_link) *sum_link = s[1];
}

}  // namespace cpsgpu
