// The storage-order conversions of convert.cpp on device memory: the same
// site and component tables, one thread per (site, slice) moving its 24
// reals (fermions) or one thread per site moving its 72 (links), out of
// place, on the lattice's stream.
//
//   fermion CANONICAL <-> WILSON   FwilsonTypes::Fconvert / FdwfBase::Fconvert
//                                  (convert.C:444-562, 639-1000)
//   gauge CANONICAL <-> WILSON     Lattice::Convert (convert.C:141-420)
//   4D <-> 5D wall placement       FdwfBase::Ffour2five / Ffive2four
//                                  (f_dwf_base.C:961-1140)
#include "../../include/cpsgpu.h"
#include "cpsgpu_impl.h"

namespace cpsgpu {

namespace {

struct DevGeom {
  int L[4];
  long vol, vh;
};

DevGeom geom_of(const Lattice &lat) {
  DevGeom g;
  for (int k = 0; k < 4; k++) g.L[k] = lat.L[k];
  g.vol = 2 * lat.vh;
  g.vh = lat.vh;
  return g;
}

// (x, y, z, t) of lexicographic site i
__device__ __forceinline__ void coords(const DevGeom &g, long i, int &x, int &y, int &z, int &t) {
  x = (int)(i % g.L[0]);
  i /= g.L[0];
  y = (int)(i % g.L[1]);
  i /= g.L[1];
  z = (int)(i % g.L[2]);
  t = (int)(i / g.L[2]);
}

__device__ __forceinline__ long cb_index(const DevGeom &g, int x, int y, int z, int t) {
  return (long)(x / 2) + (long)(g.L[0] / 2) * (y + (long)g.L[1] * (z + (long)g.L[2] * t));
}

// position (in sites) of site (x,y,z,t) of slice s in the WILSON order:
// 4D odd checkerboard first; 5D [odd part][even part], slice s of the odd
// part holding the 4D sites of parity (s+1)%2
__device__ __forceinline__ long wilson_pos(const DevGeom &g, int ls, int x, int y, int z, int t, int s) {
  const int p = (x + y + z + t) & 1;
  const long c = cb_index(g, x, y, z, t);
  if (ls == 1) return c + g.vh * (1 - p);
  const bool odd_part = ((p + s) & 1) == 1;
  return (odd_part ? 0 : (long)ls * g.vh) + (long)s * g.vh + c;
}

__global__ void fconvert_kernel(DevGeom g, int ls, double2 *dst, const double2 *src, int c2w) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= g.vol * ls) return;
  const int s = (int)(idx / g.vol);
  int x, y, z, t;
  coords(g, idx % g.vol, x, y, z, t);
  const long wil = wilson_pos(g, ls, x, y, z, t, s);
  const long d = c2w ? wil : idx, q = c2w ? idx : wil;
#pragma unroll
  for (int k = 0; k < 12; k++) dst[12 * d + k] = src[12 * q + k];
}

__global__ void gconvert_kernel(DevGeom g, double *dst, const double *src, int c2w) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.vol) return;
  int x, y, z, t;
  coords(g, i, x, y, z, t);
  const long wil = cb_index(g, x, y, z, t) + g.vh * ((x + y + z + t) & 1);  // even parity first
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
#pragma unroll
    for (int row = 0; row < 3; row++)
#pragma unroll
      for (int col = 0; col < 3; col++)
#pragma unroll
        for (int r = 0; r < 2; r++) {
          const long ic = 72 * i + 18 * mu + 2 * (3 * row + col) + r;  // [mu][row][col]
          const long iw = 72 * wil + 18 * mu + 2 * (row + 3 * col) + r;  // [mu][col][row]
          if (c2w) dst[iw] = src[ic];
          else dst[ic] = src[iw];
        }
}

// five: ls slices of v4 sites; the upper half of slice s_u and the lower
// half of slice s_l carry the 4D field, every other half is zero
__global__ void four2five_kernel(long v4, int ls, double2 *five, const double2 *four, int s_u, int s_l) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= v4 * ls) return;
  const int s = (int)(idx / v4);
  const long x = idx % v4;
#pragma unroll
  for (int k = 0; k < 6; k++) five[12 * idx + k] = (s == s_u) ? four[12 * x + k] : make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 6; k < 12; k++) five[12 * idx + k] = (s == s_l) ? four[12 * x + k] : make_double2(0.0, 0.0);
}

__global__ void five2four_kernel(long v4, double2 *four, const double2 *five, int s_u, int s_l) {
  const long x = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= v4) return;
#pragma unroll
  for (int k = 0; k < 6; k++) four[12 * x + k] = five[12 * ((long)s_u * v4 + x) + k];
#pragma unroll
  for (int k = 6; k < 12; k++) four[12 * x + k] = five[12 * ((long)s_l * v4 + x) + k];
}

unsigned blocks(long n) { return (unsigned)((n + 255) / 256); }

bool c2w_of(int to, int from) {
  const bool c2w = (from == CPSGPU_STR_CANONICAL && to == CPSGPU_STR_WILSON);
  const bool w2c = (from == CPSGPU_STR_WILSON && to == CPSGPU_STR_CANONICAL);
  if (!c2w && !w2c) throw Error(CPSGPU_ERR_ARG, "only CANONICAL <-> WILSON");
  return c2w;
}

void check_dev(const Lattice &lat, const void *a, const void *b) {
  if (!a || !b) throw Error(CPSGPU_ERR_ARG, "null field");
  if (a == b) throw Error(CPSGPU_ERR_ARG, "device conversions are out of place: dst and src must differ");
  if (lat.t_nodes != 1) throw Error(CPSGPU_ERR_ARG, "conversions of a whole lattice, not a t slab");
}

}  // namespace

void fconvert_device(const Lattice &lat, int ls, double *dst, const double *src, int to, int from) {
  check_dev(lat, dst, src);
  if (ls < 1) throw Error(CPSGPU_ERR_ARG, "ls must be >= 1");
  const DevGeom g = geom_of(lat);
  if (to == from) {
    CPSGPU_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * 24 * (size_t)ls * g.vol, cudaMemcpyDeviceToDevice,
                                lat.stream));
    return;
  }
  const int c2w = c2w_of(to, from) ? 1 : 0;
  fconvert_kernel<<<blocks(g.vol * ls), 256, 0, lat.stream>>>(g, ls, reinterpret_cast<double2 *>(dst),
                                                              reinterpret_cast<const double2 *>(src), c2w);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void gconvert_device(const Lattice &lat, double *dst, const double *src, int to, int from) {
  check_dev(lat, dst, src);
  const DevGeom g = geom_of(lat);
  if (to == from) {
    CPSGPU_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * 72 * (size_t)g.vol, cudaMemcpyDeviceToDevice, lat.stream));
    return;
  }
  const int c2w = c2w_of(to, from) ? 1 : 0;
  gconvert_kernel<<<blocks(g.vol), 256, 0, lat.stream>>>(g, dst, src, c2w);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void four2five_device(const Lattice &lat, int ls, double *five, const double *four, int s_u, int s_l, int ncb) {
  check_dev(lat, five, four);
  if (ncb != 1 && ncb != 2) throw Error(CPSGPU_ERR_ARG, "ncb must be 1 or 2");
  if (ls < 1 || s_u < 0 || s_u >= ls || s_l < 0 || s_l >= ls) throw Error(CPSGPU_ERR_ARG, "s_u and s_l must lie in [0, ls)");
  const long v4 = lat.vh * ncb;
  four2five_kernel<<<blocks(v4 * ls), 256, 0, lat.stream>>>(v4, ls, reinterpret_cast<double2 *>(five),
                                                            reinterpret_cast<const double2 *>(four), s_u, s_l);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

void five2four_device(const Lattice &lat, int ls, double *four, const double *five, int s_u, int s_l, int ncb) {
  check_dev(lat, four, five);
  if (ncb != 1 && ncb != 2) throw Error(CPSGPU_ERR_ARG, "ncb must be 1 or 2");
  if (ls < 1 || s_u < 0 || s_u >= ls || s_l < 0 || s_l >= ls) throw Error(CPSGPU_ERR_ARG, "s_u and s_l must lie in [0, ls)");
  const long v4 = lat.vh * ncb;
  five2four_kernel<<<blocks(v4), 256, 0, lat.stream>>>(v4, reinterpret_cast<double2 *>(four),
                                                       reinterpret_cast<const double2 *>(five), s_u, s_l);
  CPSGPU_CUDA(cudaGetLastError());
  launch_counter()++;
}

}  // namespace cpsgpu
