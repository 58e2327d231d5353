// Host-side storage-order conversions either side of the solve: the
// CANONICAL <-> WILSON orders of fermion and gauge fields and the 4D <-> 5D
// wall placement of DWF sources and solutions.  These are the reference's
// host routines (no device work): a caller that keeps its fields in
// CANONICAL order converts them here before the C ABI's WILSON-order calls.
//
//   fermion, 4D WILSON (convert_func.C:429-494): site (x,y,z,t) at
//     (x - x%2 + Lx*(y + Ly*(z + Lz*t)) + V*((x+y+z+t+1)%2)) / 2, so the odd
//     checkerboard comes first; the 24 reals of a site keep their order.
//   fermion, 5D WILSON (convert.C:639-1000): [odd part][even part], slice s of
//     the odd part holding the 4D sites of parity (s+1)%2 and of the even part
//     those of parity s%2, each in checkerboard order; CANONICAL is Ls 4D
//     CANONICAL volumes.
//   gauge WILSON (convert.C:258-336): [parity, even first][checkerboard site]
//     [mu][col][row][re, im]; CANONICAL [lexicographic site][mu][row][col].
//   Ffour2five / Ffive2four (f_dwf_base.C:961-1140): the upper spin half of
//     slice s_u and the lower one of slice s_l carry the 4D field.
#include <cstring>
#include <vector>

#include "../../include/cpsgpu.h"
#include "cpsgpu_impl.h"

namespace cpsgpu {

namespace {

struct Geom {
  int L[4];
  long vol, vh;
  explicit Geom(const int node_sites[4]) {
    for (int k = 0; k < 4; k++) L[k] = node_sites[k];
    vol = (long)L[0] * L[1] * L[2] * L[3];
    vh = vol / 2;
  }
  // lexicographic index of (x, y, z, t)
  long lex(int x, int y, int z, int t) const { return x + (long)L[0] * (y + (long)L[1] * (z + (long)L[2] * t)); }
  // checkerboard index within the site's parity
  long cb(int x, int y, int z, int t) const { return (long)(x / 2) + (long)(L[0] / 2) * (y + (long)L[1] * (z + (long)L[2] * t)); }
  template <typename F> void each(F &&f) const {
    for (int t = 0; t < L[3]; t++)
      for (int z = 0; z < L[2]; z++)
        for (int y = 0; y < L[1]; y++)
          for (int x = 0; x < L[0]; x++) f(x, y, z, t);
  }
};

void check_geom(const int node_sites[4]) {
  if (!node_sites) throw Error(CPSGPU_ERR_ARG, "null node_sites");
  for (int k = 0; k < 4; k++)
    if (node_sites[k] < 2 || node_sites[k] % 2) throw Error(CPSGPU_ERR_ARG, "node sites must be even and >= 2");
}

// position (in sites) of 4D site (x,y,z,t) of slice s in the WILSON order
long wilson_pos(const Geom &g, int ls, int x, int y, int z, int t, int s) {
  const int p = (x + y + z + t) & 1;
  const long c = g.cb(x, y, z, t);
  if (ls == 1) return c + g.vh * (1 - p);  // odd checkerboard first
  const bool odd_part = ((p + s) & 1) == 1;
  return (odd_part ? 0 : (long)ls * g.vh) + (long)s * g.vh + c;
}

}  // namespace

void fconvert(const int node_sites[4], int ls, double *f, int to, int from) {
  check_geom(node_sites);
  if (ls < 1) throw Error(CPSGPU_ERR_ARG, "ls must be >= 1");
  if (!f) throw Error(CPSGPU_ERR_ARG, "null field");
  if (to == from) return;
  const bool c2w = (from == CPSGPU_STR_CANONICAL && to == CPSGPU_STR_WILSON);
  const bool w2c = (from == CPSGPU_STR_WILSON && to == CPSGPU_STR_CANONICAL);
  if (!c2w && !w2c) throw Error(CPSGPU_ERR_ARG, "only CANONICAL <-> WILSON");
  const Geom g(node_sites);
  std::vector<double> tmp(f, f + 24 * (size_t)ls * g.vol);
  for (int s = 0; s < ls; s++)
    g.each([&](int x, int y, int z, int t) {
      const long canon = (long)s * g.vol + g.lex(x, y, z, t);
      const long wil = wilson_pos(g, ls, x, y, z, t, s);
      const long dst = c2w ? wil : canon, src = c2w ? canon : wil;
      std::memcpy(f + 24 * dst, tmp.data() + 24 * src, 24 * sizeof(double));
    });
}

void gconvert(const int node_sites[4], double *u, int to, int from) {
  check_geom(node_sites);
  if (!u) throw Error(CPSGPU_ERR_ARG, "null field");
  if (to == from) return;
  const bool c2w = (from == CPSGPU_STR_CANONICAL && to == CPSGPU_STR_WILSON);
  const bool w2c = (from == CPSGPU_STR_WILSON && to == CPSGPU_STR_CANONICAL);
  if (!c2w && !w2c) throw Error(CPSGPU_ERR_ARG, "only CANONICAL <-> WILSON");
  const Geom g(node_sites);
  std::vector<double> tmp(u, u + 72 * (size_t)g.vol);
  g.each([&](int x, int y, int z, int t) {
    const long canon = g.lex(x, y, z, t);
    const long wil = g.cb(x, y, z, t) + g.vh * ((x + y + z + t) & 1);  // even parity first
    for (int mu = 0; mu < 4; mu++)
      for (int row = 0; row < 3; row++)
        for (int col = 0; col < 3; col++)
          for (int r = 0; r < 2; r++) {
            const long ic = 72 * canon + 18 * mu + 2 * (3 * row + col) + r;
            const long iw = 72 * wil + 18 * mu + 2 * (row + 3 * col) + r;
            if (c2w) u[iw] = tmp[ic];
            else u[ic] = tmp[iw];
          }
  });
}

void four2five(const int node_sites[4], int ls, double *five, const double *four, int s_u, int s_l, int ncb) {
  check_geom(node_sites);
  if (!five || !four) throw Error(CPSGPU_ERR_ARG, "null field");
  if (ncb != 1 && ncb != 2) throw Error(CPSGPU_ERR_ARG, "ncb must be 1 or 2");
  if (ls < 1 || s_u < 0 || s_u >= ls || s_l < 0 || s_l >= ls) throw Error(CPSGPU_ERR_ARG, "s_u and s_l must lie in [0, ls)");
  const Geom g(node_sites);
  const long v4 = g.vol * ncb / 2;
  std::memset(five, 0, sizeof(double) * 24 * (size_t)ls * v4);
  for (long x = 0; x < v4; x++) {
    std::memcpy(five + 24 * ((long)s_u * v4 + x), four + 24 * x, 12 * sizeof(double));
    std::memcpy(five + 24 * ((long)s_l * v4 + x) + 12, four + 24 * x + 12, 12 * sizeof(double));
  }
}

void five2four(const int node_sites[4], int ls, double *four, const double *five, int s_u, int s_l, int ncb) {
  check_geom(node_sites);
  if (!five || !four) throw Error(CPSGPU_ERR_ARG, "null field");
  if (ncb != 1 && ncb != 2) throw Error(CPSGPU_ERR_ARG, "ncb must be 1 or 2");
  if (ls < 1 || s_u < 0 || s_u >= ls || s_l < 0 || s_l >= ls) throw Error(CPSGPU_ERR_ARG, "s_u and s_l must lie in [0, ls)");
  const Geom g(node_sites);
  const long v4 = g.vol * ncb / 2;
  for (long x = 0; x < v4; x++) {
    std::memcpy(four + 24 * x, five + 24 * ((long)s_u * v4 + x), 12 * sizeof(double));
    std::memcpy(four + 24 * x + 12, five + 24 * ((long)s_l * v4 + x) + 12, 12 * sizeof(double));
  }
}

}  // namespace cpsgpu
