// Seeded synthetic inputs: SU(3) gauge links and Gaussian fermion sources.
//
// Every random number is a pure function of (seed, stream, index) through
// a SplitMix64-style integer hash (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014), so results do not depend on
// thread count or traversal order.  Gaussians use the Box-Muller transform.
//
// Links: U = exp(i w H) with H = (A + A^+)/2 - tr(.)/3, A a 3x3 matrix of
// unit complex Gaussians; the exponential by scaling and squaring of a
// Taylor series, then Gram-Schmidt on rows 0 and 1 and row 2 = conj(r0 x r1)
// so det U = 1 to rounding (the 12-real compression relies on it).
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace cpsgpu {

using cd = std::complex<double>;

static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline double uniform(uint64_t seed, uint64_t stream, uint64_t idx) {
  uint64_t h = mix64(seed ^ mix64(stream * 0x632BE59BD9B4E019ull ^ mix64(idx)));
  return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);  // (0, 1)
}

// Gaussian number `idx` of a stream: Box-Muller pair (2k, 2k+1)
double gaussian(uint64_t seed, uint64_t stream, uint64_t idx) {
  uint64_t pair = idx >> 1;
  double u1 = uniform(seed, stream, 2 * pair), u2 = uniform(seed, stream, 2 * pair + 1);
  double r = std::sqrt(-2.0 * std::log(u1));
  double th = 6.283185307179586476925286766559 * u2;
  return (idx & 1) ? r * std::sin(th) : r * std::cos(th);
}

typedef cd M3[3][3];

static void mat_mul(const M3 a, const M3 b, M3 c) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      cd s = 0;
      for (int k = 0; k < 3; k++) s += a[i][k] * b[k][j];
      c[i][j] = s;
    }
}

static void su3_from_seed(uint64_t seed, uint64_t key, double width, M3 u) {
  M3 a, h;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      a[i][j] = cd(gaussian(seed, 1, key * 18 + 2 * (3 * i + j)), gaussian(seed, 1, key * 18 + 2 * (3 * i + j) + 1));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) h[i][j] = 0.5 * (a[i][j] + std::conj(a[j][i]));
  cd tr = (h[0][0] + h[1][1] + h[2][2]) / 3.0;
  for (int i = 0; i < 3; i++) h[i][i] -= tr;
  // X = i w H; exp(X) = exp(X / 2^k)^(2^k)
  M3 x;
  double nrm = 0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      x[i][j] = cd(0, width) * h[i][j];
      nrm += std::norm(x[i][j]);
    }
  nrm = std::sqrt(nrm);
  int k = 0;
  while (nrm > 0.25) {
    nrm *= 0.5;
    k++;
  }
  double sc = std::ldexp(1.0, -k);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) x[i][j] *= sc;
  M3 e, term, t2;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) e[i][j] = term[i][j] = (i == j) ? 1.0 : 0.0;
  for (int n = 1; n <= 18; n++) {
    mat_mul(term, x, t2);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        term[i][j] = t2[i][j] / double(n);
        e[i][j] += term[i][j];
      }
  }
  for (int s = 0; s < k; s++) {
    mat_mul(e, e, t2);
    std::memcpy(e, t2, sizeof(M3));
  }
  // reunitarise: Gram-Schmidt rows 0, 1; row 2 = conj(row0 x row1)
  double n0 = 0;
  for (int j = 0; j < 3; j++) n0 += std::norm(e[0][j]);
  n0 = 1.0 / std::sqrt(n0);
  for (int j = 0; j < 3; j++) u[0][j] = e[0][j] * n0;
  cd pr = 0;
  for (int j = 0; j < 3; j++) pr += std::conj(u[0][j]) * e[1][j];
  for (int j = 0; j < 3; j++) u[1][j] = e[1][j] - pr * u[0][j];
  double n1 = 0;
  for (int j = 0; j < 3; j++) n1 += std::norm(u[1][j]);
  n1 = 1.0 / std::sqrt(n1);
  for (int j = 0; j < 3; j++) u[1][j] *= n1;
  u[2][0] = std::conj(u[0][1] * u[1][2] - u[0][2] * u[1][1]);
  u[2][1] = std::conj(u[0][2] * u[1][0] - u[0][0] * u[1][2]);
  u[2][2] = std::conj(u[0][0] * u[1][1] - u[0][1] * u[1][0]);
}

// WILSON order: u[72 (i + vh p) + 18 mu + 2 (row + 3 col)], the RNG keyed by
// the canonical site x + Lx (y + Ly (z + Lz t)) and mu.
void gen_gauge(const int L[4], uint64_t seed, double width, double *out) {
  const long vol = (long)L[0] * L[1] * L[2] * L[3];
  const long vh = vol / 2;
  unsigned nth = std::thread::hardware_concurrency();
  if (nth == 0) nth = 1;
  if (nth > 64) nth = 64;
  auto work = [&](long begin, long end) {
    for (long site = begin; site < end; site++) {
      long r = site;
      int x = (int)(r % L[0]);
      r /= L[0];
      int y = (int)(r % L[1]);
      r /= L[1];
      int z = (int)(r % L[2]);
      int t = (int)(r / L[2]);
      int p = (x + y + z + t) & 1;
      long i = x / 2 + (long)(L[0] / 2) * (y + (long)L[1] * (z + (long)L[2] * t));
      for (int mu = 0; mu < 4; mu++) {
        M3 u;
        su3_from_seed(seed, (uint64_t)site * 4 + mu, width, u);
        double *m = out + 72 * (i + vh * p) + 18 * mu;
        for (int row = 0; row < 3; row++)
          for (int col = 0; col < 3; col++) {
            m[2 * (row + 3 * col)] = u[row][col].real();
            m[2 * (row + 3 * col) + 1] = u[row][col].imag();
          }
      }
    }
  };
  std::vector<std::thread> th;
  long per = (vol + nth - 1) / nth;
  for (unsigned k = 0; k < nth; k++) {
    long b = k * per, e = std::min(vol, b + per);
    if (b < e) th.emplace_back(work, b, e);
  }
  for (auto &t : th) t.join();
}

void gen_gaussian(double *out, long n, uint64_t seed, unsigned stream) {
  unsigned nth = std::thread::hardware_concurrency();
  if (nth == 0) nth = 1;
  if (nth > 64) nth = 64;
  if (n < (1 << 16)) nth = 1;
  auto work = [&](long b, long e) {
    for (long k = b; k < e; k++) out[k] = gaussian(seed, 1000 + stream, (uint64_t)k);
  };
  std::vector<std::thread> th;
  long per = (n + nth - 1) / nth;
  for (unsigned k = 0; k < nth; k++) {
    long b = k * per, e = std::min(n, b + per);
    if (b < e) th.emplace_back(work, b, e);
  }
  for (auto &t : th) t.join();
}

}  // namespace cpsgpu
