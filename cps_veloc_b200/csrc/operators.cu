// Even-odd preconditioned operators built from the fused hop kernel.
//
//   Wilson  MatPc  = 1 - kappa^2 D_oe D_eo              (wilson_m.C:49-93)
//   DWF     MatPc  = 1 - kappa_5^2 D D, D = 4D + 5D hop   (dwf_m.C:31-63)
//   Mobius  MatPc  = 1 - kappa_b D_4 M5^-1 kappa_b D_4 M5^-1   (SYM2,
//           zmobius_m-sym2.h:5-127) and its dagger (zmobius_mdag-sym2.h)
//
// For Mobius every s-local factor between two hops (M5^-1, the b/c
// mixing of zmobius_dslash_4, the kappa_b scalings) is folded into one Ls x
// Ls matrix per chirality, precomputed here in FP64, so MatPc is
//   out = in - kappa_b W0 ( Q W1 ( P in ) )        (3 kernels)
//   MatPcDag: out = in + S W0^+ ( R W1^+ in )       (2 kernels)
// where W is the plain Wilson hop of every slice.
#include <cmath>
#include <complex>
#include <cstring>

#include "cpsgpu_impl.h"
#include "hop.cuh"

namespace cpsgpu {

using cd = std::complex<double>;

// ---------------------------------------------------------------- lattice
Lattice::Lattice(const int L_[4], const double bc_[4]) {
  for (int k = 0; k < 4; k++) {
    if (L_[k] <= 0 || (L_[k] & 1)) throw Error(-1, "lattice extents must be positive and even");
    L[k] = L_[k];
    bc[k] = bc_[k];
  }
  vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
  // the kernels index the gauge field (8 x 9 x vh 16-byte elements at most)
  // and the sites of a slice with 32-bit offsets
  if (vh > 2147483647L / 72) throw Error(-1, "lattice too large: more than 29,826,161 sites per checkerboard");
  CPSGPU_CUDA(cudaGetDevice(&device));
  CPSGPU_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  own_stream = stream;
  CPSGPU_CUDA(cudaMallocHost(&pinned, 64 * sizeof(double)));
  scratch_st.alloc(sizeof(SolverScalars) * 4);
  CPSGPU_CUDA(cudaMemsetAsync(scratch_st.ptr, 0, scratch_st.bytes, stream));
}

Lattice::~Lattice() {
  if (stream && stream != own_stream) cudaStreamSynchronize(stream);
  if (own_stream) {
    cudaStreamSynchronize(own_stream);
    cudaStreamDestroy(own_stream);
  }
  if (pinned) cudaFreeHost(pinned);
}

GaugeView Lattice::gauge(int prec) const {
  GaugeView g;
  g.vh = vh;
  if (prec == PREC_DOUBLE)
    g.data = use_recon12 ? gD12.ptr : gD18.ptr;
  else if (prec == PREC_SINGLE || recon(prec) == LINK_F32_18 || recon(prec) == LINK_F32_12)
    g.data = (recon(prec) == 18 || recon(prec) == LINK_F32_18) ? gS18.ptr : gS12.ptr;
  else
    g.data = recon(prec) == 18 ? gH18.ptr : gH12.ptr;
  return g;
}

// ---------------------------------------------------------------- Mobius matrices
namespace {

// Dense M5^-1 as the reference's recurrences apply it (zmobius_m5inv.C
// :247-396 for dag 0, :534-679 for dag 1): the same scalar recurrence along
// s for every site and component, run here on the unit vectors.
void m5inv_columns(int ls, const std::vector<cd> &K, double mass, int dag, std::vector<cd> &up,
                   std::vector<cd> &dn) {
  up.assign((size_t)ls * ls, 0.0);
  dn.assign((size_t)ls * ls, 0.0);
  cd inv_d_last, prod = 1.0;
  if (!dag) {
    for (int s = 0; s < ls; s++) prod *= -K[s];
    inv_d_last = 1.0 / (1.0 + prod * mass);
  } else {
    for (int s = 0; s < ls; s++) prod *= K[s];
    inv_d_last = std::conj(1.0 / (1.0 + prod * mass));
  }
  std::vector<cd> v(ls), w(ls);
  for (int col = 0; col < ls; col++) {
    for (int s = 0; s < ls; s++) v[s] = w[s] = (s == col) ? 1.0 : 0.0;
    if (!dag) {
      w[ls - 1] *= inv_d_last;
      cd fl = K[ls - 1] * mass * inv_d_last;
      for (int s = 0; s + 1 < ls; s++) {
        v[s + 1] += -K[s + 1] * v[s];
        w[ls - 1] += fl * w[s];
        fl *= -K[s];
      }
      cd p = 1.0;
      for (int s = 0; s < ls - 1; s++) p *= -K[s];
      cd fr = -p * mass * inv_d_last;
      for (int s = ls - 2; s >= 0; s--) {
        v[s] += fr * v[ls - 1];
        w[s] += -K[s] * w[s + 1];
        fr /= -K[s];
      }
      v[ls - 1] *= inv_d_last;
    } else {
      v[ls - 1] *= inv_d_last;
      cd fr = std::conj(K[0]) * mass * inv_d_last;
      for (int s = 0; s + 1 < ls; s++) {
        v[ls - 1] += fr * v[s];
        w[s + 1] += -std::conj(K[s]) * w[s];
        fr *= -std::conj(K[s + 1]);
      }
      cd p = 1.0;
      for (int s = 0; s < ls - 2; s++) p *= -K[s];
      p *= -K[ls - 1];
      cd fl = -std::conj(p) * mass * inv_d_last;
      for (int s = ls - 2; s >= 0; s--) {
        v[s] += -std::conj(K[s + 1]) * v[s + 1];
        w[s] += fl * w[ls - 1];
        if (s > 0) fl /= -std::conj(K[s - 1]);
      }
      w[ls - 1] *= inv_d_last;
    }
    for (int s = 0; s < ls; s++) {
      up[(size_t)s * ls + col] = v[s];
      dn[(size_t)s * ls + col] = w[s];
    }
  }
}

// b/c mixing of zmobius_dslash_4 (dag 0): b_s psi(s) + c-weighted fifth-
// direction hop with -m_f at the walls (zmobius_dslash_5_plus.C:125-374).
void bmix(int ls, const std::vector<cd> &b, const std::vector<cd> &c, double mass, std::vector<cd> &up,
          std::vector<cd> &dn) {
  up.assign((size_t)ls * ls, 0.0);
  dn.assign((size_t)ls * ls, 0.0);
  for (int s = 0; s < ls; s++) {
    up[(size_t)s * ls + s] += b[s];
    dn[(size_t)s * ls + s] += b[s];
    if (s == 0) up[(size_t)s * ls + ls - 1] += -mass * c[0];
    else up[(size_t)s * ls + s - 1] += c[s];
    if (s == ls - 1) dn[(size_t)s * ls + 0] += -mass * c[ls - 1];
    else dn[(size_t)s * ls + s + 1] += c[s];
  }
}

std::vector<cd> matmul(int n, const std::vector<cd> &a, const std::vector<cd> &b) {
  std::vector<cd> r((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < n; k++)
      for (int j = 0; j < n; j++) r[(size_t)i * n + j] += a[(size_t)i * n + k] * b[(size_t)k * n + j];
  return r;
}
std::vector<cd> adjoint(int n, const std::vector<cd> &a) {
  std::vector<cd> r((size_t)n * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) r[(size_t)i * n + j] = std::conj(a[(size_t)j * n + i]);
  return r;
}
std::vector<cd> diag_left(int n, const std::vector<cd> &d, const std::vector<cd> &a) {
  std::vector<cd> r(a);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) r[(size_t)i * n + j] *= d[i];
  return r;
}
std::vector<cd> diag_right(int n, const std::vector<cd> &a, const std::vector<cd> &d) {
  std::vector<cd> r(a);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) r[(size_t)i * n + j] *= d[j];
  return r;
}

// pack [upper; lower] real parts (real b, c give real matrices)
std::vector<double> pack(int n, const std::vector<cd> &up, const std::vector<cd> &dn) {
  std::vector<double> r(2 * (size_t)n * n);
  for (size_t k = 0; k < (size_t)n * n; k++) {
    r[k] = up[k].real();
    r[(size_t)n * n + k] = dn[k].real();
  }
  return r;
}

// pack [upper; lower] as complex: [2][n][n][re, im]
std::vector<double> pack_complex(int n, const std::vector<cd> &up, const std::vector<cd> &dn) {
  std::vector<double> r(4 * (size_t)n * n);
  for (size_t k = 0; k < (size_t)n * n; k++) {
    r[2 * k] = up[k].real();
    r[2 * k + 1] = up[k].imag();
    r[2 * ((size_t)n * n + k)] = dn[k].real();
    r[2 * ((size_t)n * n + k) + 1] = dn[k].imag();
  }
  return r;
}

void upload(DeviceBuffer &buf, const std::vector<double> &h) {
  buf.alloc(h.size() * sizeof(double));
  CPSGPU_CUDA(cudaMemcpy(buf.ptr, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
}

}  // namespace

Dirac::Dirac(Lattice *l, int kind_, int ls_, double mass_, double m5_, double b_, double c_, double a5inv_)
    : lat(l), kind(kind_), ls(ls_), mass(mass_), m5(m5_), b(b_), c(c_), a5inv(a5inv_), kappa(0), kappa_c(0) {
  if (!(a5inv > 0.0)) throw Error(-1, "dwf_a5_inv must be positive");
  if (kind == KIND_WILSON) {
    ls = 1;
    kappa = 1.0 / (2.0 * (mass + 4.0));  // d_op_wilson.C:134-137
    return;
  }
  if (ls < 2 || ls > MAX_LS) throw Error(-1, "Ls must be in [2, 32]");
  if (kind == KIND_DWF) {
    kappa = 1.0 / (2.0 * (4.0 + a5inv - m5));  // dwf_init.C:97-98
    return;
  }
  // Mobius: d_op_mobius.C:112-131 (real b, c: the same for every slice)
  build_mobius(std::vector<cd>(ls, b), std::vector<cd>(ls, c));
}

// Per-slice kappa_b, kappa_c and K = kappa_b / kappa_c as the zMobius
// operator sets them (d_op_zmobius.C:246-292, with a5inv), and every s-local
// matrix the operators apply.
void Dirac::build_mobius(const std::vector<cd> &bs, const std::vector<cd> &cs) {
  std::vector<cd> kb(ls), kc(ls), K(ls);
  cplx = false;
  for (int s = 0; s < ls; s++) {
    kb[s] = 1.0 / (2.0 * (bs[s] * (4.0 - m5) + a5inv));
    kc[s] = 1.0 / (2.0 * (cs[s] * (4.0 - m5) - a5inv));
    K[s] = kb[s] / kc[s];
    cplx = cplx || bs[s].imag() != 0.0 || cs[s].imag() != 0.0;
  }
  uniform_bc = true;
  for (int s = 1; s < ls; s++) uniform_bc = uniform_bc && bs[s] == bs[0] && cs[s] == cs[0];
  b = bs[0].real();
  c = cs[0].real();
  kappa = kb[0].real();
  kappa_c = kc[0].real();
  std::vector<cd> m0u, m0d, m1u, m1d, bu, bd;
  m5inv_columns(ls, K, mass, 0, m0u, m0d);
  m5inv_columns(ls, K, mass, 1, m1u, m1d);
  bmix(ls, bs, cs, mass, bu, bd);
  std::vector<cd> bdu = adjoint(ls, bu), bdd = adjoint(ls, bd);
  std::vector<cd> mkb(ls);
  for (int s = 0; s < ls; s++) mkb[s] = -std::conj(kb[s]);
  std::vector<cd> ckb(ls);
  for (int s = 0; s < ls; s++) ckb[s] = std::conj(kb[s]);
  // P = B M5inv ; Q = B M5inv kappa_b
  std::vector<cd> Pu = matmul(ls, bu, m0u), Pd = matmul(ls, bd, m0d);
  std::vector<cd> Qu = diag_right(ls, Pu, kb), Qd = diag_right(ls, Pd, kb);
  // S = M5inv^+ B^+ ; R = conj(kappa_b) S (-conj(kappa_b))
  std::vector<cd> Su = matmul(ls, m1u, bdu), Sd = matmul(ls, m1d, bdd);
  std::vector<cd> Ru = diag_right(ls, diag_left(ls, ckb, Su), mkb), Rd = diag_right(ls, diag_left(ls, ckb, Sd), mkb);
  // M5 = 1 + K D5, what MatInv applies to the initial guess (the b/c mixing
  // form with b = 1, c = K)
  std::vector<cd> m5u, m5d, m5au, m5ad, Ka(ls);
  bmix(ls, std::vector<cd>(ls, 1.0), K, mass, m5u, m5d);
  for (int s = 0; s < ls; s++) Ka[s] = a5inv * K[s];
  bmix(ls, std::vector<cd>(ls, 1.0), Ka, mass, m5au, m5ad);
  // -kappa_b(s) on both chiralities (zmobius_m-sym2.h: the last step of MatPc)
  std::vector<cd> kbm((size_t)ls * ls, 0.0);
  for (int s = 0; s < ls; s++) kbm[(size_t)s * ls + s] = -kb[s];
  auto packm = [&](const std::vector<cd> &up, const std::vector<cd> &dn) {
    return cplx ? pack_complex(ls, up, dn) : pack(ls, up, dn);
  };
  // uploads keeping the host copy of a real matrix (launch_mix's parameter)
  mix_host.clear();
  auto upload = [&](DeviceBuffer &buf, const std::vector<double> &h) {
    cpsgpu::upload(buf, h);
    if (!cplx) mix_host[buf.ptr] = h;
  };
  hM5i = packm(m0u, m0d);
  hM5id = packm(m1u, m1d);
  hB = packm(bu, bd);
  hBd = packm(bdu, bdd);
  upload(mixP, packm(Pu, Pd));
  upload(mixQ, packm(Qu, Qd));
  upload(mixR, packm(Ru, Rd));
  upload(mixS, packm(Su, Sd));
  upload(mixB, hB);
  upload(mixBd, hBd);
  upload(mixM5i, hM5i);
  upload(mixM5id, hM5id);
  upload(mixM5, packm(m5u, m5d));
  upload(mixM5a, packm(m5au, m5ad));
  upload(mixKb, packm(kbm, kbm));
  set_pc_type((cplx || !uniform_bc) ? PC_SYM2 : pc_type);
}

// The plans of MatPc and MatPc^dagger for a preconditioning type, in the
// notation out = X + Last W_cb0(Mid W_cb1(Pre in)) with B the b/c mixing of
// zmobius_dslash_4 (B^+ after the hop for dag 1), M = M5^-1, K = kappa_b:
//   ORIG      (zmobius_m-orig.h, zmobius_mdag-orig.h)
//       dag 0: Pre B,            Mid B M K,  Last -K,            X = M5 in
//       dag 1: Pre -,            Mid K M^+ B^+ (-K), Last B^+,   X = M5^+ in
//   SYM1      (zmobius_m-sym1.h, zmobius_mdag-sym1.h)
//       dag 0: Pre B,            Mid B M K,  Last M (-K)
//       dag 1: Pre M^+,          Mid K M^+ B^+ (-K), Last B^+
//   SYM2      (zmobius_m-sym2.h, zmobius_mdag-sym2.h)
//       dag 0: Pre B M,          Mid B M K,  Last -K
//       dag 1: Pre -,            Mid K M^+ B^+ (-K), Last M^+ B^+
//   SYM1_MIT  (zmobius_m-sym1-MIT.h, zmobius_mdag-sym1-MIT.h)
//       dag 0: Pre B Binv,       Mid B M K,  Last Bm M (-K)
//       dag 1: Pre M^+ Bm^+,     Mid K M^+ B^+ (-K), Last Binv^+ B^+
//   SYM2_MIT  (zmobius_m-sym2-MIT.h, zmobius_mdag-sym2-MIT.h)
//       dag 0: Pre B M Binv,     Mid B M K,  Last Bm (-K)
//       dag 1: Pre Bm^+,         Mid K M^+ B^+ (-K), Last Binv^+ M^+ B^+
//   SYM3      (zmobius_m-sym3.h, zmobius_mdag-sym3.h)
//       dag 0: Pre B M,          Mid B M,    Last 1
//       dag 1: Pre -,            Mid M^+ B^+, Last M^+ B^+
// with Bm = b (1 + (c/b) D5) and Binv = M5^-1(K = c/b) / b the MIT matrices
// (zmobius_B_MIT / zmobius_Binv_MIT, d_op_zmobius.C:132-239), X = in unless
// stated, and diagonal factors moved through W (it acts slice by slice).
// SYM3 rescales GJP's b, c by i kappa_b around its hops, but
// zmobius_dslash_4 reads the operator's own copies of b, c
// (zmobius_dslash_4.C:61-62), so the hops see the plain B: reproduced as
// the reference computes it.  The forms other than SYM2 need real b, c.
void Dirac::set_pc_type(int pc) {
  if (kind != KIND_MOBIUS) throw Error(-1, "preconditioning type: Mobius operators only");
  if (pc < PC_ORIG || pc > PC_SYM3) throw Error(-1, "unknown Mobius preconditioning type");
  if (pc != PC_SYM2 && (cplx || !uniform_bc))
    throw Error(-1, "Mobius preconditioning other than SYM2: real b, c, the same on every slice");
  pc_type = pc;
  for (const DeviceBuffer &b : pc_bufs) mix_host.erase(b.ptr);
  pc_bufs.clear();
  pc_bufs.reserve(16);
  plan[0] = plan[1] = MobiusPlan();
  if (pc == PC_SYM2) {
    plan[0].pre = mixP.as<double>();
    plan[0].mid = mixQ.as<double>();
    if (cplx) plan[0].last = mixKb.as<double>();
    else plan[0].coef = -kappa;
    plan[1].mid = mixR.as<double>();
    plan[1].last = mixS.as<double>();
    return;
  }
  using V = std::vector<cd>;
  const V bs(ls, b), cs(ls, c), ones(ls, 1.0);
  V kb(ls), K(ls), fact(ls), mkb(ls), ckb(ls), invb(ls), invbc(ls);
  for (int s = 0; s < ls; s++) {
    kb[s] = 1.0 / (2.0 * (bs[s] * (4.0 - m5) + a5inv));
    const cd kc = 1.0 / (2.0 * (cs[s] * (4.0 - m5) - a5inv));
    K[s] = kb[s] / kc;
    fact[s] = cs[s] / bs[s];
    mkb[s] = -kb[s];
    ckb[s] = std::conj(kb[s]);
    invb[s] = 1.0 / bs[s];
    invbc[s] = 1.0 / std::conj(bs[s]);
  }
  V m0u, m0d, m1u, m1d, f0u, f0d, f1u, f1d, bu, bd, m5u, m5d, fbu, fbd;
  m5inv_columns(ls, K, mass, 0, m0u, m0d);
  m5inv_columns(ls, K, mass, 1, m1u, m1d);
  m5inv_columns(ls, fact, mass, 0, f0u, f0d);
  m5inv_columns(ls, fact, mass, 1, f1u, f1d);
  bmix(ls, bs, cs, mass, bu, bd);
  bmix(ls, ones, K, mass, m5u, m5d);
  bmix(ls, ones, fact, mass, fbu, fbd);
  struct Pair {
    V u, d;
  };
  auto mm = [&](const Pair &a, const Pair &b2) { return Pair{matmul(ls, a.u, b2.u), matmul(ls, a.d, b2.d)}; };
  auto adj = [&](const Pair &a) { return Pair{adjoint(ls, a.u), adjoint(ls, a.d)}; };
  auto dl = [&](const V &d, const Pair &a) { return Pair{diag_left(ls, d, a.u), diag_left(ls, d, a.d)}; };
  auto dr = [&](const Pair &a, const V &d) { return Pair{diag_right(ls, a.u, d), diag_right(ls, a.d, d)}; };
  const Pair B{bu, bd}, Bd = adj(B), M{m0u, m0d}, Md{m1u, m1d}, M5{m5u, m5d}, M5d = adj(M5);
  const Pair Bm = dl(bs, Pair{fbu, fbd}), Bmd = dr(adj(Pair{fbu, fbd}), V(ls, std::conj(bs[0])));
  const Pair Binv = dr(Pair{f0u, f0d}, invb), Binvd = dl(invbc, Pair{f1u, f1d});
  V diag_mk((size_t)ls * ls, 0.0);
  for (int s = 0; s < ls; s++) diag_mk[(size_t)s * ls + s] = mkb[s];
  const Pair negK{diag_mk, diag_mk};
  const Pair Q = dr(mm(B, M), kb);                 // B M K
  const Pair R = dr(dl(ckb, mm(Md, Bd)), mkb);     // K M^+ B^+ (-K)
  auto put = [&](const Pair &a) -> const double * {
    pc_bufs.emplace_back();
    const std::vector<double> h = pack(ls, a.u, a.d);
    upload(pc_bufs.back(), h);
    mix_host[pc_bufs.back().ptr] = h;
    return pc_bufs.back().as<double>();
  };
  switch (pc) {
    case PC_ORIG:
      plan[0].pre = put(B);
      plan[0].mid = put(Q);
      plan[0].coef = -kappa;
      plan[0].xmix = put(M5);
      plan[1].mid = put(R);
      plan[1].last = put(Bd);
      plan[1].xmix = put(M5d);
      break;
    case PC_SYM1:
      plan[0].pre = put(B);
      plan[0].mid = put(Q);
      plan[0].last = put(mm(M, negK));
      plan[1].pre = put(Md);
      plan[1].mid = put(R);
      plan[1].last = put(Bd);
      break;
    case PC_SYM1_MIT:
      plan[0].pre = put(mm(B, Binv));
      plan[0].mid = put(Q);
      plan[0].last = put(mm(Bm, mm(M, negK)));
      plan[1].pre = put(mm(Md, Bmd));
      plan[1].mid = put(R);
      plan[1].last = put(mm(Binvd, Bd));
      break;
    case PC_SYM2_MIT:
      plan[0].pre = put(mm(B, mm(M, Binv)));
      plan[0].mid = put(Q);
      plan[0].last = put(mm(Bm, negK));
      plan[1].pre = put(Bmd);
      plan[1].mid = put(R);
      plan[1].last = put(mm(Binvd, mm(Md, Bd)));
      break;
    default:  // PC_SYM3
      plan[0].pre = put(mm(B, M));
      plan[0].mid = put(mm(B, M));
      plan[0].coef = 1.0;
      plan[1].mid = put(mm(Md, Bd));
      plan[1].last = put(mm(Md, Bd));
      break;
  }
}

// ---------------------------------------------------------------- operators
static SpinorView none() { return SpinorView(); }

void op_dslash(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int cb, int dag) {
  HopLaunch L;
  L.prec = prec;
  L.ep = EP_STORE;
  L.cb = cb;
  L.dag = dag;
  launch_hop(D, L, in, out, none(), none(), none(), none(), none(), nullptr);
}

void op_mobius_dslash4(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int cb, int dag,
                       OpWork &w) {
  if (D.kind != KIND_MOBIUS) throw Error(-1, "dslash_4: not a Mobius operator");
  if (!dag) {
    ensure_field(w.t0, prec, D.lat->vh, D.ls, in.nrhs);
    launch_mix(D, prec, D.mixB.as<double>(), in, w.t0.view());
    op_dslash(D, prec, out, w.t0.view(), cb, 0);
  } else {
    HopLaunch L;
    L.prec = prec;
    L.ep = EP_MIX;
    L.cb = cb;
    L.dag = 1;
    L.mix = D.mixBd.as<double>();
    launch_hop(D, L, in, out, none(), none(), none(), none(), none(), nullptr);
  }
}

void op_mobius_m5inv(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int dag) {
  if (D.kind != KIND_MOBIUS) throw Error(-1, "m5inv: not a Mobius operator");
  launch_mix(D, prec, dag ? D.mixM5id.as<double>() : D.mixM5i.as<double>(), in, out);
}

// out = MatPc in (dag = 0) or MatPc^+ in (dag = 1).  With norm, the last
// kernel reduces |out|^2 and |in|^2 into st with red_op.
void op_matpc(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, int dag, OpWork &w,
              SolverScalars *st, int norm, int red_op) {
  const Lattice &lat = *D.lat;
  ensure_field(w.t1, prec, lat.vh, D.ls, in.nrhs);
  HopLaunch L;
  L.prec = prec;
  L.dag = dag;
  if (D.kind != KIND_MOBIUS) {
    L.ep = EP_STORE;
    L.cb = 1;
    launch_hop(D, L, in, w.t1.view(), none(), none(), none(), none(), none(), st);
    L.ep = EP_AXPY;
    L.cb = 0;
    L.coef.assign(D.ls, -D.kappa * D.kappa);
    L.norm = norm;
    L.red_op = red_op;
    launch_hop(D, L, w.t1.view(), out, in, none(), none(), none(), none(), st);
    return;
  }
  // the Mobius form of the preconditioning type (D.plan): SYM2 by default
  const MobiusTail t = mobius_head(D, prec, dag, in, w, L, st);
  L.cb = 0;
  if (t.mix) {
    L.ep = EP_MIX_AXPY;
    L.mix = t.mix;
  } else {
    L.ep = EP_AXPY;
    L.mix = nullptr;
    L.coef.assign(D.ls, t.coef);
  }
  L.norm = norm;
  L.red_op = red_op;
  launch_hop(D, L, t.hop_in, out, t.x, none(), none(), none(), none(), st);
}

MobiusTail mobius_head(const Dirac &D, int prec, int dag, const SpinorView &in, OpWork &w, HopLaunch Lh,
                       SolverScalars *st) {
  const Lattice &lat = *D.lat;
  const MobiusPlan &p = D.plan[dag ? 1 : 0];
  SpinorView src = in;
  if (p.pre) {
    ensure_field(w.t0, prec, lat.vh, D.ls, in.nrhs);
    launch_mix(D, prec, p.pre, in, w.t0.view(), st, Lh.gate);
    src = w.t0.view();
  }
  ensure_field(w.t1, prec, lat.vh, D.ls, in.nrhs);
  Lh.ep = EP_MIX;
  Lh.cb = 1;
  Lh.dag = dag;
  Lh.mix = p.mid;
  Lh.norm = 0;
  launch_hop(D, Lh, src, w.t1.view(), none(), none(), none(), none(), none(), st);
  MobiusTail t{w.t1.view(), in, p.last, p.coef};
  if (p.xmix) {
    ensure_field(w.t3, prec, lat.vh, D.ls, in.nrhs);
    launch_mix(D, prec, p.xmix, in, w.t3.view(), st, Lh.gate);
    t.x = w.t3.view();
  }
  return t;
}

// out = MatPc^+ MatPc in; st->sum[0] = |MatPc in|^2 (the reference's dot).
void op_mdagm(const Dirac &D, int prec, const SpinorView &out, const SpinorView &in, OpWork &w, SolverScalars *st,
              int red_op_dot) {
  ensure_field(w.t2, prec, D.lat->vh, D.ls, in.nrhs);
  op_matpc(D, prec, w.t2.view(), in, 0, w, st, st ? 1 : 0, red_op_dot);
  op_matpc(D, prec, out, w.t2.view(), 1, w, st, 0, 0);
}

}  // namespace cpsgpu
