/* Test infrastructure only: the CPU oracle (see oracle.h).
 *
 * Each function restates the arithmetic of the reference routine cited in
 * its comment; file:line citations are to the reference's cps_pp tree.
 * Written for clarity, not speed: plain loops, FP64, single thread.
 */
#include "oracle.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ---------------------------------------------------------------------- */
/* geometry                                                                */
/* ---------------------------------------------------------------------- */
static long vol_cb(const orc_geom *g) {
  return (long)g->L[0] * g->L[1] * g->L[2] * g->L[3] / 2;
}

/* the fifth-direction inverse spacing (DoArg.dwf_a5_inv; 0 reads as 1) */
static double a5inv(const orc_geom *g) { return g->a5_inv != 0.0 ? g->a5_inv : 1.0; }

/* checkerboard index of a site (wilson_dslash.C:288) */
static long cb_index(const orc_geom *g, const int x[4]) {
  return x[0] / 2 + (long)(g->L[0] / 2) * (x[1] + g->L[1] * (x[2] + (long)g->L[2] * x[3]));
}

/* coordinates of checkerboard site i on 4D parity p */
static void cb_coords(const orc_geom *g, long i, int p, int x[4]) {
  int hx = g->L[0] / 2;
  long r = i / hx;
  x[1] = (int)(r % g->L[1]);
  r /= g->L[1];
  x[2] = (int)(r % g->L[2]);
  x[3] = (int)(r / g->L[2]);
  x[0] = 2 * (int)(i % hx) + ((x[1] + x[2] + x[3] + p) & 1);
}

/* ---------------------------------------------------------------------- */
/* spin and colour algebra                                                 */
/* ---------------------------------------------------------------------- */
/* gamma_mu as (column, factor) for each row, in the basis the reference's
 * OneMinusPlusGammaTimesPsi expands (wilson_dslash.C:64-128); gamma_5 =
 * diag(1,1,-1,-1) (chiral halves are reals 0-11 and 12-23). */
static const int g_col[4][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}, {2, 3, 0, 1}};
static const cplx g_fac_tab[4][4] = {
    {I, I, -I, -I}, {-1, 1, 1, -1}, {I, -I, -I, I}, {1, 1, 1, 1}};

/* link element (row, col) of direction mu at gauge site gs
 * (UELEM, wilson_dslash.C:54): stored column-major within the matrix. */
static cplx link(const double *u, long gs, int mu, int row, int col) {
  const double *m = u + 72 * gs + 18 * mu + 2 * (row + 3 * col);
  return m[0] + I * m[1];
}

static cplx ferm(const double *f, long site, int spin, int col) {
  const double *p = f + 24 * site + 2 * (col + 3 * spin);
  return p[0] + I * p[1];
}

/* acc += sign * Ulink * (1 + k gamma_mu) psi, Ulink = U or U^dagger */
static void hop_term(cplx acc[4][3], const double *u, long gs, int mu, int herm,
                     const double *psi, long ns, double k, double sign) {
  cplx chi[4][3];
  for (int s = 0; s < 4; s++)
    for (int c = 0; c < 3; c++)
      chi[s][c] = ferm(psi, ns, s, c) + k * g_fac_tab[mu][s] * ferm(psi, ns, g_col[mu][s], c);
  for (int s = 0; s < 4; s++)
    for (int a = 0; a < 3; a++) {
      cplx v = 0;
      for (int b = 0; b < 3; b++)
        v += (herm ? conj(link(u, gs, mu, b, a)) : link(u, gs, mu, a, b)) * chi[s][b];
      acc[s][a] += sign * v;
    }
}

/* ---------------------------------------------------------------------- */
/* Wilson                                                                  */
/* ---------------------------------------------------------------------- */
/* wilson_dslash.C:173-515.  Output parity cbn = 1-cb.  Forward hop: link at
 * the output site, U (1 - sdag gamma) psi(x+mu); backward hop: link at x-mu,
 * U^dagger (1 + sdag gamma) psi(x-mu).  A hop that wraps in direction mu
 * picks up bc[mu]. */
void orc_wilson_dslash(const orc_geom *g, double *chi, const double *u,
                       const double *psi, int cb, int dag) {
  long vh = vol_cb(g);
  int cbn = 1 - cb;
  double sdag = dag ? -1.0 : 1.0;
  for (long i = 0; i < vh; i++) {
    int x[4];
    cb_coords(g, i, cbn, x);
    cplx acc[4][3] = {{0}};
    for (int mu = 0; mu < 4; mu++) {
      int xp[4] = {x[0], x[1], x[2], x[3]};
      int wrap = (x[mu] == g->L[mu] - 1);
      xp[mu] = wrap ? 0 : x[mu] + 1;
      hop_term(acc, u, i + vh * cbn, mu, 0, psi, cb_index(g, xp), -sdag,
               wrap ? g->bc[mu] : 1.0);
    }
    for (int mu = 0; mu < 4; mu++) {
      int xm[4] = {x[0], x[1], x[2], x[3]};
      int wrap = (x[mu] == 0);
      xm[mu] = wrap ? g->L[mu] - 1 : x[mu] - 1;
      long j = cb_index(g, xm);
      hop_term(acc, u, j + vh * cb, mu, 1, psi, j, sdag, wrap ? g->bc[mu] : 1.0);
    }
    double *o = chi + 24 * i;
    for (int s = 0; s < 4; s++)
      for (int c = 0; c < 3; c++) {
        o[2 * (c + 3 * s)] = creal(acc[s][c]);
        o[2 * (c + 3 * s) + 1] = cimag(acc[s][c]);
      }
  }
}

/* wilson_m.C:49-93 (dag=0) and wilson_mdag.C:50-96 (dag=1):
 * chi = psi - kappa^2 D_oe D_eo psi. */
void orc_wilson_m(const orc_geom *g, double *chi, const double *u,
                  const double *psi, double kappa, int dag) {
  long n = 24 * vol_cb(g);
  double *tmp = malloc(sizeof(double) * n);
  orc_wilson_dslash(g, tmp, u, psi, 1, dag);
  orc_wilson_dslash(g, chi, u, tmp, 0, dag);
  for (long k = 0; k < n; k++) chi[k] = psi[k] - kappa * kappa * chi[k];
  free(tmp);
}

/* wilson_mdagm.C:83-154 */
void orc_wilson_mdagm(const orc_geom *g, double *chi, const double *u,
                      const double *psi, double kappa, double *dot) {
  long n = 24 * vol_cb(g);
  double *t = malloc(sizeof(double) * n);
  orc_wilson_m(g, t, u, psi, kappa, 0);
  if (dot) {
    double s = 0;
    for (long k = 0; k < n; k++) s += t[k] * t[k];
    *dot = s;
  }
  orc_wilson_m(g, chi, u, t, kappa, 1);
  free(t);
}

/* ---------------------------------------------------------------------- */
/* Shamir DWF                                                              */
/* ---------------------------------------------------------------------- */
/* dwf_dslash.C:32-51 = dwf_dslash_4 (dwf_dslash_4.C:68-154: slice s uses 4D
 * parity (s+cb)%2) + dwf_dslash_5_plus (dwf_dslash_5_plus_omp.C:115-271:
 * out[s] += 2/a5 * P in[s-1] on one chiral half and P' in[s+1] on the other,
 * the walls weighted by -2 m_f / a5), 1/a5 = g->a5_inv. */
void orc_dwf_dslash(const orc_geom *g, double *out, const double *u,
                    const double *in, double mass, int cb, int dag) {
  long vh = vol_cb(g);
  int ls = g->ls;
  long slice = 24 * vh;
  for (int s = 0; s < ls; s++)
    orc_wilson_dslash(g, out + s * slice, u, in + s * slice, (s + cb) % 2, dag);
  const double two_a5 = 2.0 * a5inv(g), wall = -2.0 * mass * a5inv(g);
  /* half fed from s-1 is the upper one for D, the lower one for D^dagger */
  int from_below = dag ? 12 : 0, from_above = dag ? 0 : 12;
  for (int s = 0; s < ls; s++) {
    int sb = (s == 0) ? ls - 1 : s - 1;
    int sa = (s == ls - 1) ? 0 : s + 1;
    double fb = (s == 0) ? wall : two_a5;
    double fa = (s == ls - 1) ? wall : two_a5;
    for (long i = 0; i < vh; i++) {
      double *o = out + s * slice + 24 * i;
      const double *ib = in + sb * slice + 24 * i;
      const double *ia = in + sa * slice + 24 * i;
      for (int k = 0; k < 12; k++) {
        o[from_below + k] += fb * ib[from_below + k];
        o[from_above + k] += fa * ia[from_above + k];
      }
    }
  }
}

/* dwf_m.C:31-63 (dag 0), dwf_mdag.C:32-63 (dag 1): out = in - kappa5^2 D D in,
 * kappa5 = 1 / (2 (4 + a5inv - M5))  (dwf_init.C:97-98) */
void orc_dwf_m(const orc_geom *g, double *out, const double *u,
               const double *in, double mass, double m5, int dag) {
  long n = 24 * vol_cb(g) * g->ls;
  double kappa = 1.0 / (2.0 * (4.0 + a5inv(g) - m5));
  double *tmp = malloc(sizeof(double) * n);
  orc_dwf_dslash(g, tmp, u, in, mass, 1, dag);
  orc_dwf_dslash(g, out, u, tmp, mass, 0, dag);
  for (long k = 0; k < n; k++) out[k] = -kappa * kappa * out[k] + in[k];
  free(tmp);
}

/* dwf_mdagm.C:32-62 */
void orc_dwf_mdagm(const orc_geom *g, double *out, const double *u,
                   const double *in, double mass, double m5, double *dot) {
  long n = 24 * vol_cb(g) * g->ls;
  double *t = malloc(sizeof(double) * n);
  orc_dwf_m(g, t, u, in, mass, m5, 0);
  if (dot) {
    double s = 0;
    for (long k = 0; k < n; k++) s += t[k] * t[k];
    *dot = s;
  }
  orc_dwf_m(g, out, u, t, mass, m5, 1);
  free(t);
}

/* ---------------------------------------------------------------------- */
/* Mobius (zMobius kernels with real or complex per-s coefficients)        */
/* ---------------------------------------------------------------------- */
/* DiracOpMobius ctor, d_op_mobius.C:112-131 */
void orc_mobius_params(orc_mobius *mp, int ls, double b, double c, double m5) {
  orc_mobius_params_a5(mp, ls, b, c, m5, 1.0);
}

void orc_mobius_params_a5(orc_mobius *mp, int ls, double b, double c, double m5, double a5_inv) {
  double kb = 1.0 / (2.0 * (b * (4.0 - m5) + a5_inv));
  double kc = 1.0 / (2.0 * (c * (4.0 - m5) - a5_inv));
  for (int s = 0; s < ls; s++) {
    mp->b[s] = b;
    mp->c[s] = c;
    mp->kappa_b[s] = kb;
    mp->K[s] = kb / kc;
  }
}

static cplx fget(const double *f, long idx) { return f[2 * idx] + I * f[2 * idx + 1]; }
static void fset(double *f, long idx, cplx v) {
  f[2 * idx] = creal(v);
  f[2 * idx + 1] = cimag(v);
}

/* out[s] += fact-weighted fifth-direction hop of in, zmobius_dslash_5_plus.C
 * :125-374.  Complex index: 12 per site, 0-5 upper chiral half, 6-11 lower. */
static void mobius_hop5_acc(const orc_geom *g, int ls, const cplx *coef,
                            double *out, const double *in, double mass, int dag) {
  long vh = vol_cb(g);
  long slice = 12 * vh; /* complex numbers per s-slice */
  cplx f[64];
  for (int s = 0; s < ls; s++) f[s] = dag ? conj(coef[s]) : coef[s];
  for (int s = 0; s < ls; s++) {
    int sb = (s == 0) ? ls - 1 : s - 1;
    int sa = (s == ls - 1) ? 0 : s + 1;
    cplx fb, fa; /* weights of the terms from s-1 and s+1 */
    if (!dag) {
      fb = (s == 0) ? -mass * f[0] : f[s];
      fa = (s == ls - 1) ? -mass * f[ls - 1] : f[s];
    } else {
      fb = (s == 0) ? -mass * f[ls - 1] : f[s - 1];
      fa = (s == ls - 1) ? -mass * f[0] : f[s + 1];
    }
    int hb = dag ? 6 : 0, ha = dag ? 0 : 6;
    for (long i = 0; i < vh; i++)
      for (int k = 0; k < 6; k++) {
        long o1 = s * slice + 12 * i + hb + k, i1 = sb * slice + 12 * i + hb + k;
        long o2 = s * slice + 12 * i + ha + k, i2 = sa * slice + 12 * i + ha + k;
        fset(out, o1, fget(out, o1) + fb * fget(in, i1));
        fset(out, o2, fget(out, o2) + fa * fget(in, i2));
      }
  }
}

/* zmobius_dslash_4.C:34-221.  dag 0: tmp[s] = b_s in[s] + c-hop5(in), then
 * a Wilson hop of every slice from parity cb.  dag 1: Wilson hop^dagger of
 * every slice, then conj(b_s) tmp[s] + conj(c)-hop5^dagger(tmp). */
void orc_mobius_dslash_4(const orc_geom *g, const orc_mobius *mp, double *out,
                         const double *u, const double *in, int cb, int dag,
                         double mass) {
  int ls = g->ls;
  long vh = vol_cb(g), slice = 24 * vh;
  double *tmp = malloc(sizeof(double) * slice * ls);
  if (!dag) {
    for (int s = 0; s < ls; s++)
      for (long k = 0; k < 12 * vh; k++) fset(tmp, s * 12 * vh + k, mp->b[s] * fget(in, s * 12 * vh + k));
    mobius_hop5_acc(g, ls, mp->c, tmp, in, mass, 0);
    for (int s = 0; s < ls; s++)
      orc_wilson_dslash(g, out + s * slice, u, tmp + s * slice, cb, 0);
  } else {
    for (int s = 0; s < ls; s++)
      orc_wilson_dslash(g, tmp + s * slice, u, in + s * slice, cb, 1);
    for (int s = 0; s < ls; s++)
      for (long k = 0; k < 12 * vh; k++) fset(out, s * 12 * vh + k, conj(mp->b[s]) * fget(tmp, s * 12 * vh + k));
    mobius_hop5_acc(g, ls, mp->c, out, tmp, mass, 1);
  }
  free(tmp);
}

/* M5^-1 in place, zmobius_m5inv_cmplx_dag0 (zmobius_m5inv.C:247-396) and
 * _dag1 (:534-679).  For each site and each of the 6 complex components of a
 * chiral half the reference runs the same scalar recurrence along s; v is
 * the upper-half component, w the lower-half one. */
void orc_mobius_m5inv(const orc_geom *g, const orc_mobius *mp, double *inout,
                      double mass, int dag) {
  int ls = g->ls;
  long vh = vol_cb(g), slice = 12 * vh;
  const cplx *K = mp->K;
  cplx inv_d_last, prod = 1.0;
  if (!dag) {
    for (int s = 0; s < ls; s++) prod *= -K[s];
    inv_d_last = 1.0 / (1.0 + prod * mass);
  } else {
    for (int s = 0; s < ls; s++) prod *= K[s];
    inv_d_last = conj(1.0 / (1.0 + prod * mass));
  }
  cplx v[64], w[64];
  for (long i = 0; i < vh; i++)
    for (int k = 0; k < 6; k++) {
      for (int s = 0; s < ls; s++) {
        v[s] = fget(inout, s * slice + 12 * i + k);
        w[s] = fget(inout, s * slice + 12 * i + 6 + k);
      }
      if (!dag) {
        w[ls - 1] *= inv_d_last;
        cplx fl = K[ls - 1] * mass * inv_d_last;
        for (int s = 0; s <= ls - 2; s++) {
          v[s + 1] += -K[s + 1] * v[s];
          w[ls - 1] += fl * w[s];
          fl *= -K[s];
        }
        cplx p = 1.0;
        for (int s = 0; s < ls - 1; s++) p *= -K[s];
        cplx fr = -p * mass * inv_d_last;
        for (int s = ls - 2; s >= 0; s--) {
          v[s] += fr * v[ls - 1];
          w[s] += -K[s] * w[s + 1];
          fr /= -K[s];
        }
        v[ls - 1] *= inv_d_last;
      } else {
        v[ls - 1] *= inv_d_last;
        cplx fr = conj(K[0]) * mass * inv_d_last;
        for (int s = 0; s <= ls - 2; s++) {
          v[ls - 1] += fr * v[s];
          w[s + 1] += -conj(K[s]) * w[s];
          fr *= -conj(K[s + 1]);
        }
        cplx p = 1.0;
        for (int s = 0; s < ls - 2; s++) p *= -K[s];
        p *= -K[ls - 1];
        cplx fl = -conj(p) * mass * inv_d_last;
        for (int s = ls - 2; s >= 0; s--) {
          v[s] += -conj(K[s + 1]) * v[s + 1];
          w[s] += fl * w[ls - 1];
          if (s > 0) fl /= -conj(K[s - 1]);
        }
        w[ls - 1] *= inv_d_last;
      }
      for (int s = 0; s < ls; s++) {
        fset(inout, s * slice + 12 * i + k, v[s]);
        fset(inout, s * slice + 12 * i + 6 + k, w[s]);
      }
    }
}

static void scale_slices(double *f, long vh, int ls, const cplx *fac, double sign, int conjugate) {
  for (int s = 0; s < ls; s++) {
    cplx a = sign * (conjugate ? conj(fac[s]) : fac[s]);
    for (long k = 0; k < 12 * vh; k++) fset(f, s * 12 * vh + k, a * fget(f, s * 12 * vh + k));
  }
}

/* SYM2 preconditioned operator: zmobius_m-sym2.h:5-127 (dag 0) and
 * zmobius_mdag-sym2.h:4-109 (dag 1). */
void orc_mobius_m(const orc_geom *g, const orc_mobius *mp, double *out,
                  const double *u, const double *in, double mass, int dag) {
  int ls = g->ls;
  long vh = vol_cb(g), n = 24 * vh * ls;
  double *t2 = malloc(sizeof(double) * n);
  if (!dag) {
    memcpy(t2, in, sizeof(double) * n);
    orc_mobius_m5inv(g, mp, t2, mass, 0);
    orc_mobius_dslash_4(g, mp, out, u, t2, 1, 0, mass);
    scale_slices(out, vh, ls, mp->kappa_b, 1.0, 0);
    orc_mobius_m5inv(g, mp, out, mass, 0);
    orc_mobius_dslash_4(g, mp, t2, u, out, 0, 0, mass);
    scale_slices(t2, vh, ls, mp->kappa_b, -1.0, 0);
    for (long k = 0; k < n; k++) out[k] = in[k] + t2[k];
  } else {
    memcpy(out, in, sizeof(double) * n);
    scale_slices(out, vh, ls, mp->kappa_b, -1.0, 1);
    orc_mobius_dslash_4(g, mp, t2, u, out, 1, 1, mass);
    orc_mobius_m5inv(g, mp, t2, mass, 1);
    scale_slices(t2, vh, ls, mp->kappa_b, 1.0, 1);
    orc_mobius_dslash_4(g, mp, out, u, t2, 0, 1, mass);
    orc_mobius_m5inv(g, mp, out, mass, 1);
    for (long k = 0; k < n; k++) out[k] += in[k];
  }
  free(t2);
}

/* zmobius_B_MIT (d_op_zmobius.C:132-185), in place, fact = c/b:
 * dag 0: out = b_s (in + fact-hop5(in)); dag 1: t = conj(b_s) in, out = t + fact-hop5^dagger(t). */
static void mobius_b_mit(const orc_geom *g, const orc_mobius *mp, double *inout, double mass, int dag) {
  int ls = g->ls;
  long vh = vol_cb(g), n = 24 * vh * ls;
  cplx fact[64];
  for (int s = 0; s < ls; s++) fact[s] = mp->c[s] / mp->b[s];
  double *t = malloc(sizeof(double) * n);
  if (!dag) {
    memcpy(t, inout, sizeof(double) * n);
    mobius_hop5_acc(g, ls, fact, inout, t, mass, 0);
    scale_slices(inout, vh, ls, mp->b, 1.0, 0);
  } else {
    scale_slices(inout, vh, ls, mp->b, 1.0, 1);
    memcpy(t, inout, sizeof(double) * n);
    mobius_hop5_acc(g, ls, fact, inout, t, mass, 1);
  }
  free(t);
}

/* zmobius_Binv_MIT (d_op_zmobius.C:190-239), in place: dag 0: M5^-1(K = c/b) (in / b_s);
 * dag 1: M5^-1^dagger(K = c/b) in, then / conj(b_s). */
static void mobius_binv_mit(const orc_geom *g, const orc_mobius *mp, double *inout, double mass, int dag) {
  int ls = g->ls;
  long vh = vol_cb(g);
  orc_mobius q = *mp;
  cplx inv_b[64];
  for (int s = 0; s < ls; s++) q.K[s] = mp->c[s] / mp->b[s];
  if (!dag) {
    for (int s = 0; s < ls; s++) inv_b[s] = 1.0 / mp->b[s];
    scale_slices(inout, vh, ls, inv_b, 1.0, 0);
    orc_mobius_m5inv(g, &q, inout, mass, 0);
  } else {
    orc_mobius_m5inv(g, &q, inout, mass, 1);
    for (int s = 0; s < ls; s++) inv_b[s] = 1.0 / conj(mp->b[s]);
    scale_slices(inout, vh, ls, inv_b, 1.0, 0);
  }
}

/* The preconditioned operator of every type zmobius_m / zmobius_mdag
 * dispatch on (zmobius_m.C:40-74, zmobius_mdag.C:41-69), step by step as
 * zmobius_m-{orig,sym1,sym2,sym1-MIT,sym2-MIT,sym3}.h and their mdag
 * counterparts.  SYM3 rescales GJP's b, c around its hops, which read the
 * operator's own copies (zmobius_dslash_4.C:61-62): no effect, so none here. */
void orc_mobius_m_pc(const orc_geom *g, const orc_mobius *mp, double *out, const double *u, const double *in,
                     double mass, int dag, int pc) {
  if (pc == ORC_PC_SYM2) {
    orc_mobius_m(g, mp, out, u, in, mass, dag);
    return;
  }
  int ls = g->ls;
  long vh = vol_cb(g), n = 24 * vh * ls;
  double *t2 = malloc(sizeof(double) * n);
  if (!dag) {
    const double *src = in;
    if (pc == ORC_PC_SYM1_MIT || pc == ORC_PC_SYM2_MIT || pc == ORC_PC_SYM3) {
      memcpy(t2, in, sizeof(double) * n);
      if (pc != ORC_PC_SYM3) mobius_binv_mit(g, mp, t2, mass, 0);
      if (pc != ORC_PC_SYM1_MIT) orc_mobius_m5inv(g, mp, t2, mass, 0);
      src = t2;
    }
    orc_mobius_dslash_4(g, mp, out, u, src, 1, 0, mass);
    if (pc != ORC_PC_SYM3) scale_slices(out, vh, ls, mp->kappa_b, 1.0, 0);
    orc_mobius_m5inv(g, mp, out, mass, 0);
    orc_mobius_dslash_4(g, mp, t2, u, out, 0, 0, mass);
    if (pc != ORC_PC_SYM3) scale_slices(t2, vh, ls, mp->kappa_b, -1.0, 0);
    if (pc == ORC_PC_SYM1 || pc == ORC_PC_SYM1_MIT) orc_mobius_m5inv(g, mp, t2, mass, 0);
    if (pc == ORC_PC_SYM1_MIT || pc == ORC_PC_SYM2_MIT) mobius_b_mit(g, mp, t2, mass, 0);
    for (long k = 0; k < n; k++) out[k] = in[k] + t2[k];
    if (pc == ORC_PC_ORIG) mobius_hop5_acc(g, ls, mp->K, out, in, mass, 0);
  } else {
    memcpy(out, in, sizeof(double) * n);
    if (pc == ORC_PC_SYM1_MIT || pc == ORC_PC_SYM2_MIT) mobius_b_mit(g, mp, out, mass, 1);
    if (pc == ORC_PC_SYM1 || pc == ORC_PC_SYM1_MIT) orc_mobius_m5inv(g, mp, out, mass, 1);
    if (pc != ORC_PC_SYM3) scale_slices(out, vh, ls, mp->kappa_b, -1.0, 1);
    orc_mobius_dslash_4(g, mp, t2, u, out, 1, 1, mass);
    orc_mobius_m5inv(g, mp, t2, mass, 1);
    if (pc != ORC_PC_SYM3) scale_slices(t2, vh, ls, mp->kappa_b, 1.0, 1);
    orc_mobius_dslash_4(g, mp, out, u, t2, 0, 1, mass);
    if (pc == ORC_PC_SYM2_MIT || pc == ORC_PC_SYM3) orc_mobius_m5inv(g, mp, out, mass, 1);
    if (pc == ORC_PC_SYM1_MIT || pc == ORC_PC_SYM2_MIT) mobius_binv_mit(g, mp, out, mass, 1);
    for (long k = 0; k < n; k++) out[k] += in[k];
    if (pc == ORC_PC_ORIG) mobius_hop5_acc(g, ls, mp->K, out, in, mass, 1);
  }
  free(t2);
}

void orc_mobius_mdagm_pc(const orc_geom *g, const orc_mobius *mp, double *out, const double *u, const double *in,
                         double mass, double *dot, int pc) {
  long n = 24 * vol_cb(g) * g->ls;
  double *t = malloc(sizeof(double) * n);
  orc_mobius_m_pc(g, mp, t, u, in, mass, 0, pc);
  if (dot) {
    double s = 0;
    for (long k = 0; k < n; k++) s += t[k] * t[k];
    *dot = s;
  }
  orc_mobius_m_pc(g, mp, out, u, t, mass, 1, pc);
  free(t);
}

/* zmobius_mdagm.C:32-59 */
void orc_mobius_mdagm(const orc_geom *g, const orc_mobius *mp, double *out,
                      const double *u, const double *in, double mass,
                      double *dot) {
  long n = 24 * vol_cb(g) * g->ls;
  double *t = malloc(sizeof(double) * n);
  orc_mobius_m(g, mp, t, u, in, mass, 0);
  if (dot) {
    double s = 0;
    for (long k = 0; k < n; k++) s += t[k] * t[k];
    *dot = s;
  }
  orc_mobius_m(g, mp, out, u, t, mass, 1);
  free(t);
}

/* ---------------------------------------------------------------------- */
/* Krylov solvers                                                          */
/* ---------------------------------------------------------------------- */
static double norm2(const double *a, long n) {
  double s = 0;
  for (long k = 0; k < n; k++) s += a[k] * a[k];
  return s;
}

/* DiracOp::InvCgShift, inv_cg.C:84-448 */
int orc_invcg(orc_mdagm_fn op, void *ctx, long n, double *sol,
              const double *src, double src_norm_sq, double stop_rsd,
              int max_num_iter, double *true_res, const double *shift) {
  double *res = malloc(sizeof(double) * n), *dir = malloc(sizeof(double) * n),
         *mmp = malloc(sizeof(double) * n);
  if (src_norm_sq == 0) src_norm_sq = norm2(src, n);
  double stp_cnd = src_norm_sq * stop_rsd * stop_rsd;
  op(ctx, mmp, sol, 0);
  if (shift)
    for (long k = 0; k < n; k++) mmp[k] = *shift * sol[k] + mmp[k];
  for (long k = 0; k < n; k++) res[k] = src[k] - mmp[k];
  memcpy(dir, res, sizeof(double) * n);
  double rr = norm2(res, n), prv, d, a, b;
  int itr = 0, max_itr = max_num_iter - 1;
  if (rr <= stp_cnd) max_itr = 0;
  for (int i = 0; i < max_itr; i++) {
    itr++;
    prv = rr;
    op(ctx, mmp, dir, &d);
    if (shift) {
      for (long k = 0; k < n; k++) mmp[k] = *shift * dir[k] + mmp[k];
      d += *shift * norm2(dir, n);
    }
    if (d == 0.0) {
      fprintf(stderr, "orc_invcg: d = 0\n");
      break;
    }
    a = prv / d;
    for (long k = 0; k < n; k++) sol[k] = a * dir[k] + sol[k];
    for (long k = 0; k < n; k++) res[k] = -a * mmp[k] + res[k];
    rr = norm2(res, n);
    if (rr <= stp_cnd) break;
    b = rr / prv;
    for (long k = 0; k < n; k++) dir[k] = b * dir[k] + res[k];
  }
  op(ctx, mmp, sol, 0);
  if (shift)
    for (long k = 0; k < n; k++) mmp[k] = *shift * sol[k] + mmp[k];
  for (long k = 0; k < n; k++) res[k] = src[k] - mmp[k];
  if (true_res) *true_res = sqrt(norm2(res, n) / src_norm_sq);
  free(res);
  free(dir);
  free(mmp);
  return itr + 1;
}

/* DiracOp::MInvCG, minvcg.C:47-353 (Jegerlehner's shifted recurrences). */
int orc_minvcg(orc_mdagm_fn op, void *ctx, long n, double **psi,
               const double *chi, double chi_norm, const double *mass,
               int nmass, double *rsdcg, int type, const double *alpha,
               int max_num_iter) {
  double *r = malloc(sizeof(double) * n), *Ap = malloc(sizeof(double) * n);
  double **p = malloc(sizeof(double *) * nmass);
  for (int s = 0; s < nmass; s++) p[s] = malloc(sizeof(double) * n);
  int *conv = calloc(nmass, sizeof(int));
  double *bs = malloc(sizeof(double) * nmass), *z[2], *rsd_sq = malloc(sizeof(double) * nmass);
  z[0] = malloc(sizeof(double) * nmass);
  z[1] = malloc(sizeof(double) * nmass);
  double a, as, b, bp, c, cp, d, css = 0;
  if (type == 1)
    for (int s = 0; s < nmass; s++) memset(psi[s], 0, sizeof(double) * n);
  if (type == 0 || type == 1) {
    memcpy(r, chi, sizeof(double) * n);
    cp = chi_norm;
  } else {
    op(ctx, r, psi[0], 0);
    for (long k = 0; k < n; k++) r[k] = chi[k] - r[k];
    cp = norm2(r, n);
  }
  for (int s = 0; s < nmass; s++) memcpy(p[s], r, sizeof(double) * n);
  for (int s = 0; s < nmass; s++) rsd_sq[s] = cp * rsdcg[s] * rsdcg[s];

  /* d = <p, A p> */
  if (mass[0] > 0) {
    op(ctx, Ap, p[0], 0);
    for (long k = 0; k < n; k++) Ap[k] = mass[0] * p[0][k] + Ap[k];
    d = 0;
    for (long k = 0; k < n; k++) d += p[0][k] * Ap[k];
  } else {
    op(ctx, Ap, p[0], &d);
  }
  b = -cp / d;
  z[0][0] = z[1][0] = 1.0;
  bs[0] = b;
  int iz = 1;
  for (int s = 1; s < nmass; s++) {
    z[1 - iz][s] = 1.0;
    z[iz][s] = 1.0 / (1.0 - b * (mass[s] - mass[0]));
    bs[s] = b * z[iz][s];
  }
  for (long k = 0; k < n; k++) r[k] = b * Ap[k] + r[k];
  c = norm2(r, n);
  if (type == 0) {
    for (int s = 0; s < nmass; s++) {
      double bt = bs[s] * alpha[s];
      for (long k = 0; k < n; k++) psi[0][k] = -bt * chi[k] + psi[0][k];
    }
  } else {
    for (int s = 0; s < nmass; s++)
      for (long k = 0; k < n; k++) psi[s][k] = -bs[s] * chi[k] + psi[s][k];
  }
  int convP = (c < rsd_sq[0]) ? 1 : 0;
  int k;
  for (k = 1; k <= max_num_iter && !convP; k++) {
    a = c / cp;
    for (int s = 0; s < nmass; s++) {
      if (conv[s]) continue;
      if (s == 0) {
        for (long q = 0; q < n; q++) p[0][q] = a * p[0][q] + r[q];
      } else {
        as = a * (z[iz][s] * bs[s]) / (z[1 - iz][s] * b);
        for (long q = 0; q < n; q++) p[s][q] = z[iz][s] * r[q] + as * p[s][q];
      }
    }
    cp = c;
    if (mass[0] > 0) {
      op(ctx, Ap, p[0], 0);
      for (long q = 0; q < n; q++) Ap[q] = mass[0] * p[0][q] + Ap[q];
      d = 0;
      for (long q = 0; q < n; q++) d += p[0][q] * Ap[q];
    } else {
      op(ctx, Ap, p[0], &d);
    }
    bp = b;
    b = -cp / d;
    bs[0] = b;
    iz = 1 - iz;
    for (int s = 1; s < nmass; s++) {
      if (conv[s]) continue;
      double zt = z[1 - iz][s] * z[iz][s] * bp /
                  (b * a * (z[iz][s] - z[1 - iz][s]) +
                   z[iz][s] * bp * (1 - b * (mass[s] - mass[0])));
      bs[s] = b * zt / z[1 - iz][s];
      z[iz][s] = zt;
    }
    for (long q = 0; q < n; q++) r[q] = b * Ap[q] + r[q];
    c = norm2(r, n);
    if (type == 0) {
      for (int s = 0; s < nmass; s++) {
        if (conv[s]) continue;
        for (long q = 0; q < n; q++) psi[0][q] = -bs[s] * alpha[s] * p[s][q] + psi[0][q];
      }
    } else {
      for (int s = 0; s < nmass; s++) {
        if (conv[s]) continue;
        for (long q = 0; q < n; q++) psi[s][q] = -bs[s] * p[s][q] + psi[s][q];
      }
    }
    for (int s = 0; s < nmass; s++) {
      if (conv[s]) continue;
      css = c * z[iz][s] * z[iz][s];
      conv[s] = (css < rsd_sq[s]) ? 1 : 0;
      if (conv[s]) rsdcg[s] = css;
    }
    convP = conv[0];
    if (convP)
      for (int s = 0; s < nmass; s++)
        if (!conv[s]) convP = 0;
  }
  for (int s = nmass - 1; s >= 0; s--) {
    if (conv[s])
      rsdcg[s] = sqrt(rsdcg[s]);
    else
      rsdcg[s] = sqrt(c * z[iz][s] * z[iz][s]);
  }
  for (int s = 0; s < nmass; s++) free(p[s]);
  free(p);
  free(r);
  free(Ap);
  free(conv);
  free(bs);
  free(z[0]);
  free(z[1]);
  free(rsd_sq);
  return k;
}

/* ---------------------------------------------------------------------- */
/* Full-lattice solves (DiracOp*::MatInv with the CG inverter)             */
/* ---------------------------------------------------------------------- */
void orc_mobius_m5(const orc_geom *g, const orc_mobius *mp, double *inout, double mass) {
  long n = 24 * vol_cb(g) * g->ls;
  double *t = malloc(sizeof(double) * n);
  memcpy(t, inout, sizeof(double) * n);
  mobius_hop5_acc(g, g->ls, mp->K, inout, t, mass, 0);
  free(t);
}

typedef struct {
  const orc_geom *g;
  const orc_mobius *mp;
  const double *u;
  double mass, m5, kappa;
  int kind; /* 0 Wilson, 1 DWF, 2 Mobius */
  int pc;   /* Mobius preconditioning (ORC_PC_*) */
} matinv_ctx;

static void matinv_mdagm(void *vctx, double *out, const double *in, double *dot) {
  const matinv_ctx *c = (const matinv_ctx *)vctx;
  if (c->kind == 0) orc_wilson_mdagm(c->g, out, c->u, in, c->kappa, dot);
  else if (c->kind == 1) orc_dwf_mdagm(c->g, out, c->u, in, c->mass, c->m5, dot);
  else orc_mobius_mdagm_pc(c->g, c->mp, out, c->u, in, c->mass, dot, c->pc);
}

/* out[k] = a * x[k] + y[k] (fTimesV1PlusV2) */
static void axpy_to(double *out, double a, const double *x, const double *y, long n) {
  for (long k = 0; k < n; k++) out[k] = a * x[k] + y[k];
}

/* Wilson and DWF share the steps (d_op_wilson.C:257-334, d_op_dwf.C:316-492):
 * temp = kappa Dslash(in_even, CHKB_EVEN) + in_odd; b = MatPcDag temp;
 * CG on the odd checkerboard; out_even = kappa Dslash(out_odd, CHKB_ODD) + in_even. */
static int wilson_dwf_matinv(const matinv_ctx *c, double *out, const double *in, double stop_rsd,
                             int max_num_iter, double *true_res) {
  const orc_geom *g = c->g;
  long half = 24 * vol_cb(g) * g->ls;
  const double *in_odd = in, *in_even = in + half;
  double *out_odd = out, *out_even = out + half;
  double *temp = malloc(sizeof(double) * half), *b = malloc(sizeof(double) * half);
  if (c->kind == 0) orc_wilson_dslash(g, temp, c->u, in_even, 0, 0);
  else orc_dwf_dslash(g, temp, c->u, in_even, c->mass, 0, 0);
  axpy_to(temp, c->kappa, temp, in_odd, half);
  if (c->kind == 0) orc_wilson_m(g, b, c->u, temp, c->kappa, 1);
  else orc_dwf_m(g, b, c->u, temp, c->mass, c->m5, 1);
  int iter = orc_invcg(matinv_mdagm, (void *)c, half, out_odd, b, 0.0, stop_rsd, max_num_iter, true_res, 0);
  if (c->kind == 0) orc_wilson_dslash(g, temp, c->u, out_odd, 1, 0);
  else orc_dwf_dslash(g, temp, c->u, out_odd, c->mass, 1, 0);
  axpy_to(out_even, c->kappa, temp, in_even, half);
  free(temp);
  free(b);
  return iter;
}

int orc_wilson_matinv(const orc_geom *g, double *out, const double *u, const double *in, double kappa,
                      double stop_rsd, int max_num_iter, double *true_res) {
  matinv_ctx c = {g, 0, u, 0.0, 0.0, kappa, 0, ORC_PC_SYM2};
  return wilson_dwf_matinv(&c, out, in, stop_rsd, max_num_iter, true_res);
}

int orc_dwf_matinv(const orc_geom *g, double *out, const double *u, const double *in, double mass, double m5,
                   double stop_rsd, int max_num_iter, double *true_res) {
  matinv_ctx c = {g, 0, u, mass, m5, 1.0 / (2.0 * (4.0 + a5inv(g) - m5)), 1, ORC_PC_SYM2};  /* dwf_kappa */
  return wilson_dwf_matinv(&c, out, in, stop_rsd, max_num_iter, true_res);
}

/* d_op_mobius.C:407-700 for the preconditionings ORIG, SYM1, SYM2 and SYM3
 * (the MIT ones stop with an error there; -1 here), real b, c (kappa_b the
 * same for every s). */
int orc_mobius_matinv_pc(const orc_geom *g, const orc_mobius *mp, double *out, const double *u, const double *in,
                         double mass, double stop_rsd, int max_num_iter, double *true_res, int pc) {
  if (pc == ORC_PC_SYM1_MIT || pc == ORC_PC_SYM2_MIT) return -1;
  long half = 24 * vol_cb(g) * g->ls;
  const double *even_in = in, *odd_in = in + half;
  double *even_out = out, *odd_out = out + half;
  double *temp = malloc(sizeof(double) * half), *temp2 = malloc(sizeof(double) * half),
         *b = malloc(sizeof(double) * half);
  const double kb = creal(mp->kappa_b[0]);
  /* source: temp = kappa_b Dslash_4(M5^-1 in_even, CHKB_EVEN) + in_odd (:477-495) */
  memcpy(temp, even_in, sizeof(double) * half);
  orc_mobius_m5inv(g, mp, temp, mass, 0);
  orc_mobius_dslash_4(g, mp, temp2, u, temp, 0, 0, mass);
  axpy_to(temp, kb, temp2, odd_in, half);
  /* guess: odd_out <- M5 odd_out for SYM2 / SYM3 (:498-515) */
  if (pc == ORC_PC_SYM2 || pc == ORC_PC_SYM3) orc_mobius_m5(g, mp, odd_out, mass);
  /* SYM1: temp <- M5^-1 temp (:519-530) */
  if (pc == ORC_PC_SYM1) orc_mobius_m5inv(g, mp, temp, mass, 0);
  /* CG on MatPcDag temp (:540-548) */
  orc_mobius_m_pc(g, mp, b, u, temp, mass, 1, pc);
  matinv_ctx c = {g, mp, u, mass, 0.0, 0.0, 2, pc};
  int iter = orc_invcg(matinv_mdagm, &c, half, odd_out, b, 0.0, stop_rsd, max_num_iter, true_res, 0);
  /* SYM2 / SYM3: odd_out <- M5^-1 odd_out; then (every type)
   * even_out = M5^-1 (kappa_b Dslash_4(odd_out, CHKB_ODD)) + M5^-1 in_even (:627-663) */
  if (pc == ORC_PC_SYM2 || pc == ORC_PC_SYM3) orc_mobius_m5inv(g, mp, odd_out, mass, 0);
  orc_mobius_dslash_4(g, mp, temp, u, odd_out, 1, 0, mass);
  for (long k = 0; k < half; k++) temp[k] *= kb;
  memcpy(even_out, temp, sizeof(double) * half);
  orc_mobius_m5inv(g, mp, even_out, mass, 0);
  memcpy(temp, even_in, sizeof(double) * half);
  orc_mobius_m5inv(g, mp, temp, mass, 0);
  for (long k = 0; k < half; k++) even_out[k] += temp[k];
  /* out *= 2 kappa_b (:667-677) */
  for (long k = 0; k < 2 * half; k++) out[k] *= 2.0 * kb;
  free(temp);
  free(temp2);
  free(b);
  return iter;
}

int orc_mobius_matinv(const orc_geom *g, const orc_mobius *mp, double *out, const double *u, const double *in,
                      double mass, double stop_rsd, int max_num_iter, double *true_res) {
  return orc_mobius_matinv_pc(g, mp, out, u, in, mass, stop_rsd, max_num_iter, true_res, ORC_PC_SYM2);
}

/* ---------------------------------------------------------------------- */
/* BiCGstab(n): DiracOpWilsonTypes::BiCGstab, bicgstab.C:35-229             */
/* ---------------------------------------------------------------------- */
/* <a, b> = sum conj(a) b (compDotProduct, vector_util.C:889-903) */
static cplx cdot(const double *a, const double *b, long n) {
  double re = 0, im = 0;
  for (long k = 0; k < n; k += 2) {
    re += a[k] * b[k] + a[k + 1] * b[k + 1];
    im += a[k] * b[k + 1] - a[k + 1] * b[k];
  }
  return re + I * im;
}
/* a = f c + d (cTimesV1PlusV2, vector_util.C:912-922) */
static void caxpy(double *a, cplx f, const double *c, const double *d, long n) {
  const double re = creal(f), im = cimag(f);
  for (long k = 0; k < n; k += 2) {
    const double cr = c[k], ci = c[k + 1];
    a[k] = re * cr - im * ci + d[k];
    a[k + 1] = re * ci + im * cr + d[k + 1];
  }
}

int orc_bicgstab(orc_matpc_fn matpc, void *ctx, long f_size, double *psi, const double *chi, double chi_norm,
                 int nn, double stop_rsd, int max_num_iter, double *true_res) {
  enum { NMAX = 10 };
  if (nn <= 0 || nn > NMAX) return -1;
  double *r[NMAX + 1], *u[NMAX + 1];
  for (int i = 0; i <= nn; i++) {
    r[i] = calloc(f_size, sizeof(double));
    u[i] = calloc(f_size, sizeof(double));
  }
  double *r0 = calloc(f_size, sizeof(double));
  cplx rho0 = 1.0, rho1, alpha = 0.0, omega = 1.0, beta;
  double sigma[NMAX + 1];
  cplx gamma[NMAX + 1], gamma_p[NMAX + 1], gamma_pp[NMAX + 1], tau[NMAX + 1][NMAX + 1];
  int converged = 0, k;
  if (chi_norm == 0.0) chi_norm = norm2(chi, f_size);
  if (chi_norm == 0.0) {
    memset(psi, 0, sizeof(double) * f_size);
    for (int i = 0; i <= nn; i++) { free(r[i]); free(u[i]); }
    free(r0);
    return 0;
  }
  const double rsd_sq = chi_norm * stop_rsd * stop_rsd;
  matpc(ctx, r[0], psi);
  for (long q = 0; q < f_size; q++) r[0][q] = chi[q] - r[0][q];
  sigma[0] = norm2(r[0], f_size);
  memcpy(r0, r[0], sizeof(double) * f_size);
  memset(u[0], 0, sizeof(double) * f_size);
  for (k = 1; k <= max_num_iter && !converged; k += nn) {
    rho0 *= -omega;
    for (int j = 0; j < nn; j++) { /* BiCG part */
      rho1 = cdot(r0, r[j], f_size);
      beta = alpha * rho1 / rho0;
      rho0 = rho1;
      for (int i = 0; i <= j; i++) caxpy(u[i], -beta, u[i], r[i], f_size);
      matpc(ctx, u[j + 1], u[j]);
      alpha = rho0 / cdot(r0, u[j + 1], f_size);
      for (int i = 0; i <= j; i++) caxpy(r[i], -alpha, u[i + 1], r[i], f_size);
      matpc(ctx, r[j + 1], r[j]);
      caxpy(psi, alpha, u[0], psi, f_size);
    }
    for (int j = 1; j <= nn; j++) { /* MR part */
      for (int i = 1; i < j; i++) {
        tau[i][j] = cdot(r[i], r[j], f_size) / sigma[i];
        caxpy(r[j], -tau[i][j], r[i], r[j], f_size);
      }
      sigma[j] = norm2(r[j], f_size);
      gamma_p[j] = cdot(r[j], r[0], f_size) / sigma[j];
    }
    gamma[nn] = gamma_p[nn];
    omega = gamma[nn];
    for (int j = nn - 1; j > 0; j--) {
      gamma[j] = gamma_p[j];
      for (int i = j + 1; i <= nn; i++) gamma[j] -= tau[j][i] * gamma[i];
    }
    for (int j = 1; j < nn; j++) {
      gamma_pp[j] = gamma[j + 1];
      for (int i = j + 1; i < nn; i++) gamma_pp[j] += tau[j][i] * gamma[i + 1];
    }
    caxpy(u[0], -gamma[nn], u[nn], u[0], f_size);
    caxpy(psi, gamma[1], r[0], psi, f_size);
    caxpy(r[0], -gamma_p[nn], r[nn], r[0], f_size);
    for (int j = 1; j < nn; j++) {
      caxpy(u[0], -gamma[j], u[j], u[0], f_size);
      caxpy(psi, gamma_pp[j], r[j], psi, f_size);
      caxpy(r[0], -gamma_p[j], r[j], r[0], f_size);
    }
    sigma[0] = norm2(r[0], f_size);
    if (sigma[0] < rsd_sq) converged = 1;
  }
  if (converged && true_res) *true_res = sqrt(sigma[0]);
  for (int i = 0; i <= nn; i++) { free(r[i]); free(u[i]); }
  free(r0);
  return k;
}

/* ---------------------------------------------------------------------- */
/* HMC fermion force                                                       */
/* ---------------------------------------------------------------------- */
/* f_(i,j) = sum over blocks and spins of [(1 + sign gamma_mu) v]_(s,i)
 * conj(w_(s,j)) (sprojTr{X,Y,Z,T}{p,m}, f_wilson_types/noarch/sproj_tr.C):
 * blocks of 24 reals, v_stride / w_stride extra reals between blocks. */
void orc_sproj_tr(int mu, int sign, double *f, const double *v, const double *w, int nblk, int v_stride,
                  int w_stride) {
  cplx acc[3][3] = {{0}};
  for (int b = 0; b < nblk; b++) {
    const double *vb = v + (long)b * (24 + v_stride), *wb = w + (long)b * (24 + w_stride);
    for (int s = 0; s < 4; s++) {
      cplx a[3];
      for (int c = 0; c < 3; c++)
        a[c] = ferm(vb, 0, s, c) + sign * g_fac_tab[mu][s] * ferm(vb, 0, g_col[mu][s], c);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) acc[i][j] += a[i] * conj(ferm(wb, 0, s, j));
    }
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      f[2 * (3 * i + j)] = creal(acc[i][j]);
      f[2 * (3 * i + j) + 1] = cimag(acc[i][j]);
    }
}

/* The per-link matrix steps of the force loop (f_wilson.C:642-656,
 * f_dwf_base_force.C:268-285) on row-major 3x3 matrices: F = U T;
 * F <- 1/2 (F - F^dag) - 1/3 i Im tr(...) (Matrix::TrLessAntiHermMatrix,
 * su3_util.C:79-91); F *= coeff; norm = -2 Re tr(F F) (Matrix::norm). */
void orc_force_matrix(double *f, double *norm, const double *U, const double *T, double coeff) {
  cplx F[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      cplx s = 0;
      for (int k = 0; k < 3; k++)
        s += (U[2 * (3 * i + k)] + I * U[2 * (3 * i + k) + 1]) * (T[2 * (3 * k + j)] + I * T[2 * (3 * k + j) + 1]);
      F[i][j] = s;
    }
  cplx A[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) A[i][j] = 0.5 * (F[i][j] - conj(F[j][i]));
  const double c = (cimag(A[0][0]) + cimag(A[1][1]) + cimag(A[2][2])) / 3.0;
  for (int i = 0; i < 3; i++) A[i][i] -= I * c;
  double tr = 0.0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      A[i][j] *= coeff;
    }
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) tr += creal(A[i][k] * A[k][i]);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      f[2 * (3 * i + j)] = creal(A[i][j]);
      f[2 * (3 * i + j) + 1] = cimag(A[i][j]);
    }
  *norm = -2.0 * tr;
}

/* position (in sites) of 4D site x, slice s in a full WILSON-order fermion
 * (convert_func.C:429-494 for ls = 1: odd checkerboard first; convert.C:
 * 704-760 for ls > 1: [odd part][even part], slice s of the odd part
 * holding 4D parity (s+1)%2) */
static long wilson_site(const orc_geom *g, const int x[4], int s) {
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
  const long vh = vol_cb(g), c = cb_index(g, x);
  if (g->ls == 1) return c + vh * (1 - p);
  return (((p + s) & 1) ? 0 : (long)g->ls * vh) + (long)s * vh + c;
}

/* The force loop of FdwfBase::EvolveMomFforce (f_dwf_base_force.C:41-300;
 * ls = 1 is Fwilson::EvolveMomFforce, f_wilson.C:470-687) after
 * CalcHmdForceVecs: v1 = (chi, D chi), v2 = (-kappa^2 MatPc chi, D^dag of
 * it) as full fermion fields in WILSON order (the reference converts them to
 * CANONICAL first; indexing the WILSON order directly reads the same values).
 * Per site x and direction mu, with the sum over slices s:
 *   T = sproj(1 - g_mu)[v1(x+mu), v2(x)] + sproj(1 + g_mu)[v2(x+mu), v1(x)],
 *   mom(x, mu) += coeff TrLessAntiHerm(U_mu(x) T)  in the reference's step
 * order (orc_force_matrix), coeff = -2 dt, negated where x+mu wraps an
 * antiperiodic direction.  mom is CANONICAL: [lexicographic site][mu][row][col][re,im].
 * out = {L1, L2, Linf} as the reference's ForceArg(L1/(4V), sqrt(L2/(4V)), Linf). */
void orc_fforce(const orc_geom *g, double *mom, const double *u, const double *v1, const double *v2, double dt,
                double out[3]) {
  const long vol = 2 * vol_cb(g);
  double L1 = 0.0, L2 = 0.0, Linf = 0.0;
  for (int mu = 0; mu < 4; mu++)
    for (int t = 0; t < g->L[3]; t++)
      for (int z = 0; z < g->L[2]; z++)
        for (int y = 0; y < g->L[1]; y++)
          for (int xx = 0; xx < g->L[0]; xx++) {
            const int x[4] = {xx, y, z, t};
            int xp[4] = {xx, y, z, t};
            double coeff = -2.0 * dt;
            xp[mu] = (x[mu] + 1) % g->L[mu];
            if (x[mu] + 1 == g->L[mu] && g->bc[mu] < 0) coeff = -coeff;
            double T1[18] = {0}, T2[18] = {0}, tmp[18];
            for (int s = 0; s < g->ls; s++) {
              const long o = wilson_site(g, x, s), op = wilson_site(g, xp, s);
              orc_sproj_tr(mu, -1, tmp, v1 + 24 * op, v2 + 24 * o, 1, 0, 0);
              for (int k = 0; k < 18; k++) T1[k] += tmp[k];
              orc_sproj_tr(mu, +1, tmp, v2 + 24 * op, v1 + 24 * o, 1, 0, 0);
              for (int k = 0; k < 18; k++) T2[k] += tmp[k];
            }
            for (int k = 0; k < 18; k++) T1[k] += T2[k];
            /* U_mu(x) as a row-major matrix */
            const int p = (xx + y + z + t) & 1;
            const long gs = cb_index(g, x) + vol_cb(g) * p;
            double U[18];
            for (int i = 0; i < 3; i++)
              for (int j = 0; j < 3; j++) {
                const cplx e = link(u, gs, mu, i, j);
                U[2 * (3 * i + j)] = creal(e);
                U[2 * (3 * i + j) + 1] = cimag(e);
              }
            double F[18], n;
            orc_force_matrix(F, &n, U, T1, coeff);
            double *m = mom + 18 * (4 * (xx + (long)g->L[0] * (y + (long)g->L[1] * (z + (long)g->L[2] * t))) + mu);
            for (int k = 0; k < 18; k++) m[k] += F[k];
            const double a = sqrt(n);
            L1 += a;
            L2 += n;
            if (a > Linf) Linf = a;
          }
  out[0] = L1 / (4.0 * vol);
  out[1] = sqrt(L2 / (4.0 * vol));
  out[2] = Linf;
}

/* ---------------------------------------------------------------------- */
/* chronological initial guess                                             */
/* ---------------------------------------------------------------------- */
/* DiracOp::MinResExt (d_op_base/comsrc/minresext.C:30-150), step for step:
 * orthonormalise the previous solutions v[] in place, vm[i] = A v[i] with
 * A = MatPcDagMatPc, G = v^dag A v, b = v^dag phi, Gauss-Jordan with the
 * reference's diagonal pivoting, then psi = sum a_i v_i; *error =
 * |phi - A psi| / |phi|.  degree 0: psi = 0. */
void orc_minresext(orc_mdagm_fn op, void *ctx, long n, double *psi, const double *phi, double **v, double **vm,
                   int degree, double *error) {
  if (degree <= 0) {
    memset(psi, 0, sizeof(double) * n);
    if (error) *error = 1.0;
    return;
  }
  cplx G[16][16], a[16], b[16], xp;
  for (int i = 0; i < degree; i++) {
    const double s = 1.0 / sqrt(norm2(v[i], n));
    for (long k = 0; k < n; k++) v[i][k] *= s;
    for (int j = i + 1; j < degree; j++) {
      xp = cdot(v[i], v[j], n);
      caxpy(v[j], -xp, v[i], v[j], n);
    }
  }
  for (int i = 0; i < degree; i++) {
    double dot = 0.0;
    b[i] = cdot(v[i], phi, n);
    op(ctx, vm[i], v[i], &dot);
    G[i][i] = dot;
  }
  for (int j = 0; j < degree; j++)
    for (int k = j + 1; k < degree; k++) {
      G[j][k] = cdot(v[j], vm[k], n);
      G[k][j] = conj(G[j][k]);
    }
  for (int i = 0; i < degree; i++) {
    int k = i;
    for (int j = i + 1; j < degree; j++)
      if (cabs(G[j][j]) > cabs(G[k][k])) k = j;
    if (k != i) {
      xp = b[k];
      b[k] = b[i];
      b[i] = xp;
      for (int j = 0; j < degree; j++) {
        xp = G[k][j];
        G[k][j] = G[i][j];
        G[i][j] = xp;
      }
    }
    for (int j = i + 1; j < degree; j++) {
      xp = G[j][i] / G[i][i];
      b[j] -= xp * b[i];
      for (int kk = 0; kk < degree; kk++) G[j][kk] -= xp * G[i][kk];
    }
  }
  double *r = malloc(sizeof(double) * n);
  memset(psi, 0, sizeof(double) * n);
  memcpy(r, phi, sizeof(double) * n);
  for (int i = degree - 1; i >= 0; i--) {
    a[i] = 0.0;
    for (int j = i + 1; j < degree; j++) a[i] += G[i][j] * a[j];
    a[i] = (b[i] - a[i]) / G[i][i];
    caxpy(psi, a[i], v[i], psi, n);
    caxpy(r, -a[i], vm[i], r, n);
  }
  if (error) *error = sqrt(norm2(r, n) / norm2(phi, n));
  free(r);
}

/* mobius_Booee (d_op_mobius/noarch/mobius_dslash_4.C:40-88), dag 0:
 * out(s) = b_s in(s) + the c-weighted fifth-direction hop of in (with the
 * -mass wall terms, mobius_kappa_dslash_5_plus). */
void orc_mobius_booee(const orc_geom *g, const orc_mobius *mp, double *out, const double *in, double mass) {
  const long vh = vol_cb(g), slice = 12 * vh;
  for (int s = 0; s < g->ls; s++)
    for (long k = 0; k < slice; k++) fset(out, s * slice + k, mp->b[s] * fget(in, s * slice + k));
  mobius_hop5_acc(g, g->ls, mp->c, out, in, mass, 0);
}

/* The force loop of FforceWilsonType::run (f_wilson_types/fforce_wilson_type.C,
 * do_internal / do_surface with do_site_force), which Fmobius::EvolveMomFforce
 * (f_mobius.C:749-846) calls on the Mobius force vectors: per link,
 *   T = sum_s sprojTr(1 - g_mu)[v2(x+mu), v1(x)] + sprojTr(1 + g_mu)[v1(x+mu), v2(x)],
 *   mom(x, mu) += -coef TrLessAntiHerm(U_mu(x) T),
 * U carrying the boundary signs (Fmobius applies BondCond around it; here
 * the sign is applied where x+mu wraps an antiperiodic direction).  v1, v2
 * are full Mobius fields in their WILSON order: [even half][odd half], every
 * slice holding the same 4D parity (convert.C:797-851).  out = ForceArg. */
void orc_fforce_wilson_type(const orc_geom *g, double *mom, const double *u, const double *v1, const double *v2,
                            double coef, double out[3]) {
  const long vh = vol_cb(g), vol = 2 * vh;
  double L1 = 0.0, L2 = 0.0, Linf = 0.0;
  for (int mu = 0; mu < 4; mu++)
    for (int t = 0; t < g->L[3]; t++)
      for (int z = 0; z < g->L[2]; z++)
        for (int y = 0; y < g->L[1]; y++)
          for (int xx = 0; xx < g->L[0]; xx++) {
            const int x[4] = {xx, y, z, t};
            int xp[4] = {xx, y, z, t};
            xp[mu] = (x[mu] + 1) % g->L[mu];
            const double sign = (x[mu] + 1 == g->L[mu] && g->bc[mu] < 0) ? -1.0 : 1.0;
            const int p = (xx + y + z + t) & 1, pp = 1 - p;
            const long o0 = (p ? (long)g->ls * vh : 0) + cb_index(g, x);
            const long p0 = (pp ? (long)g->ls * vh : 0) + cb_index(g, xp);
            double T1[18] = {0}, T2[18] = {0}, tmp[18];
            for (int s = 0; s < g->ls; s++) {
              const long o = o0 + (long)s * vh, op = p0 + (long)s * vh;
              orc_sproj_tr(mu, -1, tmp, v2 + 24 * op, v1 + 24 * o, 1, 0, 0);
              for (int k = 0; k < 18; k++) T1[k] += tmp[k];
              orc_sproj_tr(mu, +1, tmp, v1 + 24 * op, v2 + 24 * o, 1, 0, 0);
              for (int k = 0; k < 18; k++) T2[k] += tmp[k];
            }
            for (int k = 0; k < 18; k++) T1[k] += T2[k];
            const long gs = cb_index(g, x) + vh * p;
            double U[18];
            for (int i = 0; i < 3; i++)
              for (int j = 0; j < 3; j++) {
                const cplx e = sign * link(u, gs, mu, i, j);
                U[2 * (3 * i + j)] = creal(e);
                U[2 * (3 * i + j) + 1] = cimag(e);
              }
            double F[18], n;
            orc_force_matrix(F, &n, U, T1, -coef);
            double *m = mom + 18 * (4 * (xx + (long)g->L[0] * (y + (long)g->L[1] * (z + (long)g->L[2] * t))) + mu);
            for (int k = 0; k < 18; k++) m[k] += F[k];
            const double a = sqrt(n);
            L1 += a;
            L2 += n;
            if (a > Linf) Linf = a;
          }
  out[0] = L1 / (4.0 * vol);
  out[1] = sqrt(L2 / (4.0 * vol));
  out[2] = Linf;
}

/* ---------------------------------------------------------------------- */
/* eigCG                                                                   */
/* ---------------------------------------------------------------------- */
/* Real symmetric eigenproblem by cyclic Jacobi rotations (Golub and Van
 * Loan, Matrix Computations, section 8.5): Ap is the packed lower triangle
 * (element (i, j), j <= i, at i(i+1)/2 + j); on return Evec[k n + i] is
 * component k of eigenvector i and Eval[i] its eigenvalue (unsorted), the
 * layout the reference's eigen_solver (eigen_solver.C:40) fills. */
void orc_sym_eigen(const double *Ap, double *Evec, double *Eval, int n) {
  double *a = malloc(sizeof(double) * n * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j <= i; j++) a[i * n + j] = a[j * n + i] = Ap[i * (i + 1) / 2 + j];
  for (int i = 0; i < n * n; i++) Evec[i] = 0.0;
  for (int i = 0; i < n; i++) Evec[i * n + i] = 1.0;
  double fro = 0.0;
  for (int i = 0; i < n * n; i++) fro += a[i] * a[i];
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) off += 2.0 * a[p * n + q] * a[p * n + q];
    if (off <= 1e-30 * fro) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = a[p * n + q];
        if (apq == 0.0) continue;
        const double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; k++) { /* columns p, q */
          const double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) { /* rows p, q */
          const double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = Evec[k * n + p], vkq = Evec[k * n + q];
          Evec[k * n + p] = c * vkp - s * vkq;
          Evec[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; i++) Eval[i] = a[i * n + i];
  free(a);
}

/* indices of the nev smallest of EIG[0..n) (min_eig_index, inv_eig_cg.C:37-51) */
static void min_eig_index(int *index, int nev, const double *eig, int n) {
  for (int i = 0; i < nev; i++) index[i] = i;
  for (int i = nev; i < n; i++) {
    int mx = 0;
    for (int j = 1; j < nev; j++)
      if (eig[index[j]] > eig[index[mx]]) mx = j;
    if (eig[i] < eig[index[mx]]) index[mx] = i;
  }
}

/* DiracOp::InvEigCg (d_op_base/comsrc/inv_eig_cg.C:129-635), step for step:
 * CG on A = MatPcDagMatPc from a zero guess (or the deflated guess
 * U invH U^dag src when def_len > 0), with the eigCG bookkeeping when
 * nev > 0: the Lanczos matrix T of the CG coefficients (packed lower
 * triangle), the normalised residuals kept in V[0..m), and at i_eig == m the
 * restart to the 2 nev Ritz vectors of T (lowest nev of T(m) and T(m-1),
 * orthonormalised, H = Q^T T Q diagonalised, V <- V Q Z, T <- diag(M) plus
 * the coupling row from A r).  Deflated restarts at the residuals
 * restart[i] |src|.  M receives the 2 nev Ritz values (0 past the rank).
 * U holds def_len deflation vectors, invH their inverse projected matrix
 * (complex, row-major, as (re, im) pairs).  Returns the reference's iter
 * (the loop index it stopped at); *true_res = |src - A sol| / |src|. */
int orc_inveigcg(orc_mdagm_fn op, void *ctx, long n, double *sol, const double *src, double stop_rsd, int max_iter,
                 int nev, int m, double **V, double *M, int def_len, double **U, const double *invH,
                 const double *restart, int restart_len, double *true_res) {
  const double src_norm_sq = norm2(src, n);
  const double stp = src_norm_sq * stop_rsd * stop_rsd;
  double *r = malloc(sizeof(double) * n), *dir = malloc(sizeof(double) * n), *mmp = malloc(sizeof(double) * n);
  double *mmp_prev = nev > 0 ? malloc(sizeof(double) * n) : NULL;
  cplx *Ub = def_len > 0 ? malloc(sizeof(cplx) * def_len) : NULL;
  cplx *invHUb = def_len > 0 ? malloc(sizeof(cplx) * def_len) : NULL;
  double dummy;
  memset(sol, 0, sizeof(double) * n);
  if (def_len > 0) {
    for (int ii = 0; ii < def_len; ii++) Ub[ii] = cdot(U[ii], src, n);
    for (int ii = 0; ii < def_len; ii++) {
      invHUb[ii] = 0.0;
      for (int jj = 0; jj < def_len; jj++)
        invHUb[ii] += (invH[2 * (ii * def_len + jj)] + I * invH[2 * (ii * def_len + jj) + 1]) * Ub[jj];
    }
    for (int ii = 0; ii < def_len; ii++) caxpy(sol, invHUb[ii], U[ii], sol, n);
  }
  op(ctx, mmp, sol, &dummy);
  for (long q = 0; q < n; q++) r[q] = dir[q] = src[q] - mmp[q];
  double res_cur = norm2(r, n), res_prv;
  int i_eig = 0, iter;
  double alpha = 1.0, beta = 0.0, alpha_old = 0.0, beta_old = 0.0, pAp;
  const int nev2 = 2 * nev;
  double *T = NULL, *Tt = NULL, *Y = NULL, *Q = NULL, *QZ = NULL, *H = NULL, *EIG = NULL, **Vn = NULL;
  int *INDEX = NULL;
  if (nev > 0) {
    T = calloc(m * (m + 1) / 2, sizeof(double));
    Tt = calloc(m * (m + 1) / 2, sizeof(double));
    Y = calloc(m * m, sizeof(double));
    Q = calloc(m * nev2, sizeof(double));
    QZ = calloc(m * nev2, sizeof(double));
    H = calloc(nev2 * (nev2 + 1) / 2, sizeof(double));
    EIG = calloc(m, sizeof(double));
    INDEX = calloc(nev, sizeof(int));
    Vn = malloc(sizeof(double *) * nev2);
    for (int j = 0; j < nev2; j++) Vn[j] = malloc(sizeof(double) * n);
  }
  int restarted = 0;
  for (iter = 0; iter < max_iter; iter++) {
    if (nev > 0 && i_eig == m) memcpy(mmp_prev, mmp, sizeof(double) * n);
    res_prv = res_cur;
    op(ctx, mmp, dir, &pAp);
    if (pAp == 0) break;
    if (nev > 0) {
      if (i_eig != 0) T[(i_eig - 1) * i_eig / 2 + i_eig - 1] = 1.0 / alpha + beta_old / alpha_old;
      if (i_eig == m) {
        for (int i = 0; i < m * (m - 1) / 2; i++) Tt[i] = T[i];
        orc_sym_eigen(Tt, Y, EIG, m - 1);
        min_eig_index(INDEX, nev, EIG, m - 1);
        for (int i = nev; i < nev2; i++) {
          for (int j = 0; j < m - 1; j++) Q[j * nev2 + i] = Y[j * (m - 1) + INDEX[i - nev]];
          Q[(m - 1) * nev2 + i] = 0.0;
        }
        for (int i = 0; i < m * (m + 1) / 2; i++) Tt[i] = T[i];
        orc_sym_eigen(Tt, Y, EIG, m);
        min_eig_index(INDEX, nev, EIG, m);
        for (int i = 0; i < nev; i++)
          for (int j = 0; j < m; j++) Q[j * nev2 + i] = Y[j * m + INDEX[i]];
        int rank = nev;
        for (int i = nev; i < nev2; i++) {
          for (int j = 0; j < rank; j++) {
            double xy = 0.0;
            for (int k = 0; k < m; k++) xy += Q[k * nev2 + i] * Q[k * nev2 + j];
            for (int k = 0; k < m; k++) Q[k * nev2 + i] -= xy * Q[k * nev2 + j];
          }
          double xx = 0.0;
          for (int k = 0; k < m; k++) xx += Q[k * nev2 + i] * Q[k * nev2 + i];
          if (xx > 1e-16) {
            xx = 1.0 / sqrt(xx);
            for (int k = 0; k < m; k++) Q[k * nev2 + rank] = xx * Q[k * nev2 + i];
            rank++;
          }
        }
        for (int i = 0; i < rank; i++)
          for (int j = 0; j <= i; j++) {
            double h = 0.0;
            for (int l = 0; l < m; l++)
              for (int k = 0; k < m; k++) {
                const double tlk = (k <= l) ? T[l * (l + 1) / 2 + k] : T[k * (k + 1) / 2 + l];
                h += Q[l * nev2 + i] * tlk * Q[k * nev2 + j];
              }
            H[i * (i + 1) / 2 + j] = h;
          }
        orc_sym_eigen(H, Y, M, rank);
        for (int i = rank; i < nev2; i++) M[i] = 0.0;
        for (int j = 0; j < rank; j++)
          for (int i = 0; i < m; i++) {
            double z = 0.0;
            for (int k = 0; k < rank; k++) z += Q[i * nev2 + k] * Y[j + k * rank];
            QZ[i + m * j] = z;
          }
        /* V[j] <- sum_i V[i] QZ[i + m j], j < rank (eigcg_vec_mult) */
        for (int j = 0; j < rank; j++)
          for (long q = 0; q < n; q++) {
            double z = 0.0;
            for (int i = 0; i < m; i++) z += V[i][q] * QZ[i + m * j];
            Vn[j][q] = z;
          }
        for (int j = 0; j < rank; j++) memcpy(V[j], Vn[j], sizeof(double) * n);
        for (int i = 0; i < m * (m + 1) / 2; i++) T[i] = 0.0;
        for (int i = 0; i < rank; i++) T[i * (i + 1) / 2 + i] = M[i];
        i_eig = rank;
        for (long q = 0; q < n; q++) mmp_prev[q] = -beta * mmp_prev[q] + mmp[q];
        for (int ii = 0; ii < i_eig; ii++) {
          double d = 0.0;
          for (long q = 0; q < n; q++) d += mmp_prev[q] * V[ii][q];
          T[i_eig * (i_eig + 1) / 2 + ii] = d / sqrt(res_cur);
        }
      } else if (i_eig != 0) {
        T[i_eig * (i_eig + 1) / 2 + i_eig - 1] = -sqrt(beta) / alpha;
      }
      const double sc = 1.0 / sqrt(res_cur);
      for (long q = 0; q < n; q++) V[i_eig][q] = sc * r[q];
      i_eig++;
    }
    alpha_old = alpha;
    alpha = -res_prv / pAp;
    res_cur = 0.0;
    for (long q = 0; q < n; q++) {
      r[q] = alpha * mmp[q] + r[q];
      res_cur += r[q] * r[q];
    }
    alpha = -alpha;
    beta_old = beta;
    beta = res_cur / res_prv;
    for (long q = 0; q < n; q++) {
      sol[q] = alpha * dir[q] + sol[q];
      dir[q] = beta * dir[q] + r[q];
    }
    if (restarted < restart_len && def_len > 0 && res_cur < restart[restarted] * restart[restarted] * src_norm_sq) {
      restarted++;
      for (int ii = 0; ii < def_len; ii++) Ub[ii] = cdot(U[ii], r, n);
      for (int ii = 0; ii < def_len; ii++) {
        invHUb[ii] = 0.0;
        for (int jj = 0; jj < def_len; jj++)
          invHUb[ii] += (invH[2 * (ii * def_len + jj)] + I * invH[2 * (ii * def_len + jj) + 1]) * Ub[jj];
      }
      memset(dir, 0, sizeof(double) * n);
      for (int ii = 0; ii < def_len; ii++) caxpy(dir, invHUb[ii], U[ii], dir, n);
      for (long q = 0; q < n; q++) sol[q] += dir[q];
      op(ctx, mmp, dir, &dummy);
      for (long q = 0; q < n; q++) r[q] -= mmp[q];
      res_cur = norm2(r, n);
      memcpy(dir, r, sizeof(double) * n);
    }
    if (res_cur <= stp) break;
  }
  op(ctx, mmp, sol, &dummy);
  double tr = 0.0;
  for (long q = 0; q < n; q++) tr += (src[q] - mmp[q]) * (src[q] - mmp[q]);
  if (true_res) *true_res = sqrt(tr / src_norm_sq);
  free(r);
  free(dir);
  free(mmp);
  free(mmp_prev);
  free(Ub);
  free(invHUb);
  if (nev > 0) {
    for (int j = 0; j < nev2; j++) free(Vn[j]);
    free(Vn);
    free(T);
    free(Tt);
    free(Y);
    free(Q);
    free(QZ);
    free(H);
    free(EIG);
    free(INDEX);
  }
  return iter;
}

/* ---------------------------------------------------------------------- */
/* Ritz eigensolver                                                        */
/* ---------------------------------------------------------------------- */
/* psi -= <vec[i], psi> vec[i] for i < nvec (DiracOp::GramSchm, ritz.C:117-150) */
static void gram_schm(double *psi, double **vec, int nvec, long n) {
  for (int i = 0; i < nvec; i++) {
    const cplx xp = cdot(vec[i], psi, n);
    caxpy(psi, -xp, vec[i], psi, n);
  }
}

static double re_dot(const double *a, const double *b, long n) {
  double s = 0.0;
  for (long k = 0; k < n; k++) s += a[k] * b[k];
  return s;
}

/* DiracOp::Ritz (d_op_base/comsrc/ritz.C:152-532), step for step: the
 * N_eig-th lowest eigenvector of A = RitzMat (MatPcDagMatPc, negated when
 * neg: RitzMatOper NEG_MATPCDAG_MATPC) by conjugate-gradient minimisation
 * of the Ritz functional orthogonal to psi_all[0..N_eig-1), starting from
 * psi_all[N_eig-1], which receives the eigenvector; *lambda its eigenvalue.
 * Returns the iteration count k (0 when the start already satisfies the
 * test); -1 after MaxCG iterations (the reference then exits). */
int orc_ritz(orc_mdagm_fn op, void *ctx, int neg, long n, double **psi_all, int N_eig, double RsdR_a,
             double RsdR_r, double Rsdlam, double Cutl_zero, int n_renorm, int Kalk_Sim, int N_min, int N_max,
             double Cv_fact, int MaxCG, int ProjApsiP, double *lambda_out) {
  double *psi = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
  double *Apsi = malloc(sizeof(double) * n), *Ap = malloc(sizeof(double) * n);
  double dummy;
#define RITZMAT(out, in)                                  \
  do {                                                    \
    op(ctx, out, in, &dummy);                             \
    if (neg)                                              \
      for (long q_ = 0; q_ < n; q_++) (out)[q_] = -(out)[q_]; \
  } while (0)
  double acc = 2.0e-24;
  acc *= acc;
  double rsda_sq = RsdR_a * RsdR_a;
  const double rsdr_sq = RsdR_r * RsdR_r;
  rsda_sq = (rsda_sq > acc) ? rsda_sq : acc;
  const int nn = N_eig - 1;
  int result = -1;
  memcpy(psi, psi_all[nn], sizeof(double) * n);
  gram_schm(psi, psi_all, nn, n);
  double d = sqrt(norm2(psi, n)), ct = 1.0 / d, st, mu, lambda, g2, p2, g2_0, del_lam, rsd, s1, s2, s3, a, b;
  for (long q = 0; q < n; q++) psi[q] *= ct;
  RITZMAT(Apsi, psi);
  if (ProjApsiP == 1) gram_schm(Apsi, psi_all, nn, n);
  mu = re_dot(psi, Apsi, n);
  lambda = mu;
  for (long q = 0; q < n; q++) p[q] = -lambda * psi[q] + Apsi[q];
  g2 = norm2(p, n);
  p2 = g2;
  g2_0 = g2 * Cv_fact;
  g2_0 = (g2_0 > acc) ? g2_0 : acc;
  rsd = rsdr_sq * lambda * lambda;
  rsd = (rsda_sq > rsd) ? rsda_sq : rsd;
  if (Kalk_Sim == 0 && N_min <= 0 && g2 <= rsd) {
    memcpy(psi_all[nn], psi, sizeof(double) * n);
    result = 0;
    goto done;
  }
  del_lam = mu;
  for (int k = 1; k <= MaxCG; ++k) {
    RITZMAT(Ap, p);
    if (ProjApsiP == 1) gram_schm(Ap, psi_all, nn, n);
    d = re_dot(p, Ap, n) / p2;
    s1 = 0.5 * (mu + d);
    s2 = 0.5 * (mu - d);
    p2 = 1.0 / sqrt(p2);
    s3 = g2 * p2;
    a = (s2 > 0.0) ? s2 : -s2;
    if (a >= s3) {
      d = s3 / s2;
      d = sqrt(1.0 + d * d);
      a = a * d;
    } else {
      d = s2 / s3;
      d = sqrt(1.0 + d * d);
      a = s3 * d;
    }
    s2 /= a; /* cos(delta) */
    s3 /= a; /* sin(delta) */
    if (s2 > 0) {
      s2 = 0.5 * (1.0 + s2);
      d = -sqrt(s2);       /* sin(theta) */
      s2 = -0.5 * s3 / d;  /* cos(theta) */
    } else {
      s2 = 0.5 * (1.0 - s2);
      s2 = sqrt(s2);       /* cos(theta) */
      d = -0.5 * s3 / s2;  /* sin(theta) */
    }
    s1 = 2.0 * a * d * d;
    mu -= s1;
    lambda = mu;
    del_lam = s1;
    st = d * p2;
    ct = s2;
    for (long q = 0; q < n; q++) {
      psi[q] = st * p[q] + ct * psi[q];
      Apsi[q] = st * Ap[q] + ct * Apsi[q];
    }
    for (long q = 0; q < n; q++) Ap[q] = -lambda * psi[q] + Apsi[q];
    s1 = g2;
    g2 = norm2(Ap, n);
    rsd = rsdr_sq * lambda * lambda;
    rsd = (rsda_sq > rsd) ? rsda_sq : rsd;
    st = Rsdlam * fabs(mu);
    if ((Kalk_Sim == 0 && k >= N_min && (fabs(mu) < Cutl_zero || (g2 <= rsd && del_lam <= st))) ||
        (Kalk_Sim == 1 && (del_lam <= st || fabs(mu) < Cutl_zero || (k >= N_min && (g2 < g2_0 || k >= N_max))))) {
      gram_schm(psi, psi_all, nn, n);
      d = sqrt(norm2(psi, n));
      ct = 1.0 / d;
      for (long q = 0; q < n; q++) psi[q] *= ct;
      RITZMAT(Apsi, psi);
      mu = re_dot(psi, Apsi, n);
      lambda = mu;
      memcpy(psi_all[nn], psi, sizeof(double) * n);
      result = k;
      goto done;
    }
    b = ct * g2 / s1;
    ct *= 0.05 * b;
    d = sqrt(g2);
    ct /= (p2 * d);
    if (ct > 1.0) {
      memcpy(p, Ap, sizeof(double) * n); /* restart: p = g */
    } else {
      const cplx xp = cdot(psi, p, n);
      caxpy(p, -xp, psi, p, n);
      for (long q = 0; q < n; q++) p[q] = b * p[q] + Ap[q];
    }
    if (k % n_renorm == 0) {
      gram_schm(psi, psi_all, nn, n);
      d = sqrt(norm2(psi, n));
      ct = 1.0 / d;
      for (long q = 0; q < n; q++) psi[q] *= ct;
      RITZMAT(Apsi, psi);
      if (ProjApsiP == 1) gram_schm(Apsi, psi_all, nn, n);
      mu = re_dot(psi, Apsi, n);
      lambda = mu;
      for (long q = 0; q < n; q++) Ap[q] = -lambda * psi[q] + Apsi[q];
      g2 = norm2(Ap, n);
      gram_schm(p, psi_all, nn, n);
      double *pp[1] = {psi};
      gram_schm(p, pp, 1, n);
      cplx xq = g2 - cdot(Ap, p, n);
      xq *= 1.0 / g2;
      caxpy(p, xq, Ap, p, n);
    } else if (ProjApsiP == 1 && nn > 0) {
      gram_schm(psi, psi_all, nn, n);
      gram_schm(p, psi_all, nn, n);
    }
    p2 = norm2(p, n);
  }
  memcpy(psi_all[nn], psi, sizeof(double) * n);
done:
#undef RITZMAT
  if (lambda_out) *lambda_out = lambda;
  free(psi);
  free(p);
  free(Apsi);
  free(Ap);
  return result;
}

/* DiracOp::Jacobi (d_op_base/comsrc/jacobi.C:48-268), step for step: Jacobi
 * rotations of the vectors psi[0..N) that zero the complex off-diagonal
 * elements off_diag[j(j-1)/2 + i] = <psi_i, A psi_j> (i < j) of the small
 * matrix with diagonal lambda, until no element exceeds
 * |lambda_i lambda_j| Toler^2; then the pairs sorted by |lambda|.  Returns
 * the sweep count, -1 after N_max sweeps (the reference exits). */
int orc_jacobi(double **psi, long n, int N_eig, double *lambda, double *off_diag_ri, double Toler, int N_max) {
  cplx *off = (cplx *)off_diag_ri; /* (re, im) pairs */
  const double tol_sq = Toler * Toler;
  double *t1 = malloc(sizeof(double) * n), *t2 = malloc(sizeof(double) * n);
  int result = -1;
  for (int k = 0; k <= N_max; k++) {
    int i_rot = 0, ij = 0;
    for (int j = 1; j < N_eig; j++)
      for (int i = 0; i < j; i++) {
        double dd = creal(off[ij]) * creal(off[ij]) + cimag(off[ij]) * cimag(off[ij]);
        double ftmp = fabs(lambda[i] * lambda[j] * tol_sq);
        if (dd > ftmp) {
          i_rot++;
          dd = sqrt(dd);
          const double acc = 100.0 * dd;
          const double diff_l = lambda[j] - lambda[i];
          double t, c, s;
          ftmp = fabs(diff_l);
          if ((ftmp + acc) == ftmp) {
            t = dd / diff_l;
          } else {
            const double theta = 0.5 * diff_l / dd;
            t = sqrt(1.0 + theta * theta);
            t = 1.0 / (fabs(theta) + t);
            if (theta < 0.0) t = -t;
          }
          if (diff_l >= 0) {
            c = 1.0 / sqrt(1.0 + t * t);
            s = -t * c;
          } else {
            s = 1.0 / sqrt(1.0 + t * t);
            c = t * s;
          }
          double al1 = c * c * lambda[i], al2 = c * c * lambda[j];
          al1 += s * s * lambda[j];
          al2 += s * s * lambda[i];
          ftmp = 2.0 * dd * s * c;
          al1 += ftmp;
          al2 -= ftmp;
          lambda[i] = al1;
          lambda[j] = al2;
          const double v11 = c;
          const cplx v12 = (s / dd) * off[ij];
          const cplx v21 = -conj(v12);
          off[ij] = 0.0;
          for (long q = 0; q < n; q += 2) {
            const cplx pi = psi[i][q] + I * psi[i][q + 1], pj = psi[j][q] + I * psi[j][q + 1];
            const cplx a = v11 * pi - v21 * pj, b = v11 * pj - v12 * pi;
            t1[q] = creal(a);
            t1[q + 1] = cimag(a);
            t2[q] = creal(b);
            t2[q + 1] = cimag(b);
          }
          memcpy(psi[i], t1, sizeof(double) * n);
          memcpy(psi[j], t2, sizeof(double) * n);
          for (int m = 0; m < N_eig; m++) {
            if (m == i || m == j) continue;
            if (m < i) {
              const int mi = i * (i - 1) / 2 + m, mj = j * (j - 1) / 2 + m;
              const cplx c1 = off[mi] * v11 - off[mj] * v21, c2 = off[mj] * v11 - off[mi] * v12;
              off[mi] = c1;
              off[mj] = c2;
            } else if (m < j) {
              const int mi = m * (m - 1) / 2 + i, mj = j * (j - 1) / 2 + m;
              const cplx c1 = conj(off[mi]) * v11 - off[mj] * v21, c2 = off[mj] * v11 - conj(off[mi]) * v12;
              off[mi] = conj(c1);
              off[mj] = c2;
            } else {
              const int mi = m * (m - 1) / 2 + i, mj = m * (m - 1) / 2 + j;
              const cplx c1 = conj(off[mi]) * v11 - conj(off[mj]) * v21;
              const cplx c2 = conj(off[mj]) * v11 - conj(off[mi]) * v12;
              off[mi] = conj(c1);
              off[mj] = conj(c2);
            }
          }
        }
        ij++;
      }
    if (i_rot == 0) {
      for (int j = 1; j < N_eig; j++)
        for (int i = 0; i < j; i++)
          if (fabs(lambda[j]) < fabs(lambda[i])) {
            const double f = lambda[i];
            lambda[i] = lambda[j];
            lambda[j] = f;
            memcpy(t1, psi[i], sizeof(double) * n);
            memcpy(psi[i], psi[j], sizeof(double) * n);
            memcpy(psi[j], t1, sizeof(double) * n);
          }
      result = k;
      break;
    }
  }
  free(t1);
  free(t2);
  return result;
}

/* RitzEigMat for RitzMatOper MATPCDAG_MATPC / NEG_MATPCDAG_MATPC
 * (d_op_wilson_types/d_op_wilson_types.C:189-215) */
static void ritz_eig_mat(orc_mdagm_fn op, void *ctx, int neg, double *out, const double *in, long n) {
  double dummy;
  op(ctx, out, in, &dummy);
  if (neg)
    for (long q = 0; q < n; q++) out[q] = -out[q];
}

/* MatHermElements (eigen_wilson.C:708-740): diag[i] = Re <psi_i, A psi_i>,
 * off[i(i-1)/2 + j] = <psi_j, A psi_i> for j < i */
static void mat_herm_elements(orc_mdagm_fn op, void *ctx, int neg, long n, double **psi, int n_vec, double *diag,
                              cplx *off, double *tmp) {
  int ij = 0;
  for (int i = 0; i < n_vec; i++) {
    ritz_eig_mat(op, ctx, neg, tmp, psi[i], n);
    diag[i] = creal(cdot(psi[i], tmp, n));
    for (int j = 0; j < i; j++) off[ij++] = cdot(psi[j], tmp, n);
  }
}

static void normalise(double *x, long n) {
  const double f = 1.0 / sqrt(norm2(x, n));
  for (long q = 0; q < n; q++) x[q] *= f;
}

/* DiracOpWilsonTypes::RitzEig (d_op_wilson_types/eigen_wilson.C:89-586),
 * step for step, with RitzEigMat = (-)MatPcDagMatPc.
 *  1. Kalkreuter-Simma (lines 187-300): sweeps of Ritz on each vector in
 *     turn (Kalk_Sim stopping rules), the off-diagonal elements
 *     <psi_j, A psi_i> and Jacobi rotations (tolerance RsdR_a), until the
 *     largest relative change of an eigenvalue between sweeps is <= Rsdlam,
 *     at most N_KS_max sweeps; with N_eig = 1 or Kalk_Sim = 0 successive
 *     Ritz calls (lines 321-330).
 *  2. Projection (lines 354-583): the matrix elements of RitzEigMat, the
 *     eigenvectors whose row of that matrix has a squared norm below 0.98
 *     lambda_old marked invalid (iterated), every vector from the first
 *     invalid one on replaced by (1 +- A / sqrt|lambda_old|) psi (the sign
 *     of <A psi, psi>; of the two the one with the larger overlap with the
 *     valid vectors), normalised; a normalised Gram-Schmidt pass over all;
 *     the matrix elements again and Jacobi with tolerance 1e-5.
 * lambda_H[0..N_eig): the eigenvalues of the last Jacobi;
 * lambda_H[N_eig..2 N_eig): lambda_old (the Ritz / KS eigenvalues);
 * valid_eig[0..N_eig).  Returns the total Ritz iteration count; -1 if a
 * Ritz call hit MaxCG, -2 if the sweeps ran out (the reference's codes,
 * including its test n_KS >= N_KS_max after the loop), -3 if a Jacobi call
 * ran out (the reference exits).  The reference's text dump of the matrix
 * to eig_arg->fname is not reproduced. */
int orc_ritz_eig(orc_mdagm_fn op, void *ctx, int neg, long n, double **psi, int N_eig, double RsdR_a,
                 double RsdR_r, double Rsdlam, double Cv_fact, int n_renorm, int Kalk_Sim, int N_min, int N_max,
                 int MaxCG, int ProjApsiP, int N_KS_max, double *lambda_H, int *valid_eig) {
  if (N_eig == 1) Kalk_Sim = 0;
  if (Kalk_Sim == 0) N_KS_max = 0;
  double *lambda = lambda_H, *lambda_old = lambda_H + N_eig, lambda_t;
  cplx *off = calloc(N_eig > 1 ? (size_t)N_eig * (N_eig - 1) / 2 : 1, sizeof(cplx));
  double *tmp = malloc(sizeof(double) * n), *tmp2 = malloc(sizeof(double) * n);
  int ncg_tot = 0, result;
  for (int k = 0; k < N_eig; k++) {
    lambda_old[k] = 1.0;
    valid_eig[k] = 0;
  }
  double del_lamb = 1.0;
  if (Kalk_Sim == 1) {
    int n_KS;
    for (n_KS = 1; n_KS <= N_KS_max && del_lamb > Rsdlam; n_KS++) {
      int ij = 0;
      for (int nn = 1, i = 0; nn <= N_eig; nn++, i++) {
        const int ncnt = orc_ritz(op, ctx, neg, n, psi, nn, RsdR_a, RsdR_r, Rsdlam, 0.0, n_renorm, Kalk_Sim, N_min,
                                  N_max, Cv_fact, MaxCG, ProjApsiP, &lambda_t);
        if (ncnt < 0) {
          result = ncnt;
          goto done;
        }
        ncg_tot += ncnt;
        lambda[i] = lambda_t;
        ritz_eig_mat(op, ctx, neg, tmp, psi[i], n);
        for (int j = 0; j < i; j++) off[ij++] = cdot(psi[j], tmp, n);
      }
      if (orc_jacobi(psi, n, N_eig, lambda, (double *)off, RsdR_a, 50) < 0) {
        result = -3;
        goto done;
      }
      if (n_KS == 1) {
        for (int i = 0; i < N_eig; i++) lambda_old[i] = lambda[i];
      } else {
        del_lamb = 0.0;
        for (int i = 0; i < N_eig; i++) {
          lambda_t = fabs((lambda_old[i] - lambda[i]) / lambda[i]);
          if (lambda_t > del_lamb) del_lamb = lambda_t;
          lambda_old[i] = lambda[i];
        }
      }
    }
    if (n_KS >= N_KS_max) {
      result = -2;
      goto done;
    }
  } else {
    for (int nn = 1, i = 0; nn <= N_eig; nn++, i++) {
      ncg_tot += orc_ritz(op, ctx, neg, n, psi, nn, RsdR_a, RsdR_r, Rsdlam, 0.0, n_renorm, 0, 0, 0, Cv_fact, MaxCG,
                          ProjApsiP, &lambda_t);
      lambda_old[i] = lambda_t;
    }
  }
  /* projection onto the eigenvectors of RitzEigMat itself */
  mat_herm_elements(op, ctx, neg, n, psi, N_eig, lambda, off, tmp);
  for (int i = 0; i < N_eig; i++) valid_eig[i] = 1;
  for (int looping = 1; looping;) {
    looping = 0;
    for (int i = 0; i < N_eig; i++) {
      if (!valid_eig[i]) continue;
      const double rEig2 = 1.0 / lambda_old[i];
      double sum = lambda[i] * lambda[i] * rEig2;
      int xy = 0;
      for (int x = 0; x < N_eig; x++)
        for (int y = 0; y < x; y++) {
          if ((x == i && valid_eig[y]) || (y == i && valid_eig[x])) {
            const double v = cabs(off[xy]);
            sum += v * v * rEig2;
          }
          xy++;
        }
      if (sum < 0.98) {
        valid_eig[i] = 0;
        looping = 1;
      }
    }
  }
  int N_dp = 0, i;
  for (i = 0; i < N_eig; i++) {
    if (valid_eig[i] == 1) N_dp++;
    else break;
  }
  for (i++; i < N_eig; i++) valid_eig[i] = 0;
  while (N_dp < N_eig) {
    valid_eig[N_dp] = 1;
    const double lam = sqrt(fabs(lambda_old[N_dp]));
    ritz_eig_mat(op, ctx, neg, tmp, psi[N_dp], n);
    const double proj = creal(cdot(tmp, psi[N_dp], n));
    const double sign = proj < 0 ? -1.0 : 1.0;
    for (long q = 0; q < n; q++) tmp2[q] = sign / lam * tmp[q] + psi[N_dp][q];
    cplx snorm = 0.0, onorm = 0.0;
    for (int k = 0; k < N_dp; k++) snorm += cdot(tmp2, psi[k], n);
    for (long q = 0; q < n; q++) tmp[q] = -sign / lam * tmp[q] + psi[N_dp][q];
    for (int k = 0; k < N_dp; k++) onorm += cdot(tmp, psi[k], n);
    const double on = creal(onorm) * creal(onorm) + cimag(onorm) * cimag(onorm);
    const double sn = creal(snorm) * creal(snorm) + cimag(snorm) * cimag(snorm);
    memcpy(psi[N_dp], on > sn ? tmp2 : tmp, sizeof(double) * n);
    normalise(psi[N_dp], n);
    N_dp++;
  }
  /* GramSchmNorm(psi[j], psi[i]) (eigen_wilson.C:78-85) for every i < j */
  for (int a = 0; a < N_eig; a++)
    for (int b = a + 1; b < N_eig; b++) {
      const cplx xp = cdot(psi[a], psi[b], n);
      caxpy(psi[b], -xp, psi[a], psi[b], n);
      normalise(psi[b], n);
    }
  int min_dim = 0;
  for (int k = 0; k < N_eig; k++)
    if (valid_eig[k]) min_dim++;
  mat_herm_elements(op, ctx, neg, n, psi, min_dim, lambda, off, tmp);
  if (orc_jacobi(psi, n, min_dim, lambda, (double *)off, 1.0e-5, 50) < 0) {
    result = -3;
    goto done;
  }
  result = ncg_tot;
done:
  free(off);
  free(tmp);
  free(tmp2);
  return result;
}

/* ---- implicitly restarted Lanczos (DiracOp::ImpResLanczos) ---- */

/* sqrt(a^2 + b^2) without overflow (Numerical Recipes' pythag; the form
 * eigen_solver.C:199-203 uses) */
static double lz_pythag(double a, double b) {
  const double aa = fabs(a), ab = fabs(b);
  if (aa > ab) return aa * sqrt(1.0 + (ab / aa) * (ab / aa));
  return ab == 0.0 ? 0.0 : ab * sqrt(1.0 + (aa / ab) * (aa / ab));
}

/* One implicitly shifted QR step on the symmetric tridiagonal (d, e) over
 * rows kmin..kmax, shift dsh, Givens bulge chase; the rotations are applied
 * to columns k, k+1 of the rows 0..nk-1 of Q (Q[i * ld + k]).
 * QRtrf (eigen_solver.C:248-305), step for step. */
void orc_qrtrf(double *d, double *e, int nk, double *Q, int ld, double dsh, int kmin, int kmax) {
  int k = kmin;
  double den = 1.0 / lz_pythag(d[k] - dsh, e[k]);
  double c = (d[k] - dsh) * den, s = -e[k] * den;
  double t1 = d[k], t2 = d[k + 1], tb = e[k];
  d[k] = c * c * t1 + s * s * t2 - 2.0 * c * s * tb;
  d[k + 1] = s * s * t1 + c * c * t2 + 2.0 * c * s * tb;
  e[k] = c * s * (t1 - t2) + (c * c - s * s) * tb;
  double x = -s * e[k + 1];
  e[k + 1] *= c;
  for (int i = 0; i < nk; i++) {
    const double q1 = Q[i * ld + k], q2 = Q[i * ld + k + 1];
    Q[i * ld + k] = c * q1 - s * q2;
    Q[i * ld + k + 1] = s * q1 + c * q2;
  }
  for (k = kmin + 1; k < kmax; k++) {
    den = 1.0 / lz_pythag(x, e[k - 1]);
    c = e[k - 1] * den;
    s = -x * den;
    t1 = d[k];
    t2 = d[k + 1];
    tb = e[k];
    d[k] = c * c * t1 + s * s * t2 - 2.0 * c * s * tb;
    d[k + 1] = s * s * t1 + c * c * t2 + 2.0 * c * s * tb;
    e[k] = c * s * (t1 - t2) + (c * c - s * s) * tb;
    e[k - 1] = c * e[k - 1] - s * x;
    if (k != kmax - 1) {
      x = -s * e[k + 1];
      e[k + 1] *= c;
    }
    for (int i = 0; i < nk; i++) {
      const double q1 = Q[i * ld + k], q2 = Q[i * ld + k + 1];
      Q[i * ld + k] = c * q1 - s * q2;
      Q[i * ld + k + 1] = s * q1 + c * q2;
    }
  }
}

/* Eigenvalues of the leading nk x nk block of the tridiagonal (d, e) by
 * QR steps with the Wilkinson-type shift of the trailing 2 x 2 block and
 * deflation from both ends; Q accumulates the rotations.  Returns the
 * step count (at most 100 n).  tqri (eigen_solver.C:206-246). */
int orc_tqri(double *d, double *e, int nk, int n, double *Q, int ld) {
  int kmin = 0, kmax = nk - 1, iter = 0;
  const int maxiter = n * 100;
  while (iter < maxiter) {
    const double dsub = d[kmax] - d[kmax - 1];
    double dd = lz_pythag(dsub, 2.0 * e[kmax - 1]);
    const double dsh = 0.5 * (d[kmax - 1] + d[kmax] + (dsub < 0 ? -fabs(dd) : fabs(dd)));
    orc_qrtrf(d, e, nk, Q, ld, dsh, kmin, kmax);
    int j;
    for (j = kmax; j >= kmin + 1; j--) {
      dd = fabs(d[j - 1]) + fabs(d[j]);
      if (fabs(e[j - 1]) + dd > dd) {
        kmax = j;
        break;
      }
    }
    if (j == kmin) return iter;
    for (j = 0; j < kmax; j++) {
      dd = fabs(d[j]) + fabs(d[j + 1]);
      if (fabs(e[j]) + dd > dd) {
        kmin = j;
        break;
      }
    }
    iter++;
  }
  return iter;
}

/* selection sort into descending order; with Q (Q != NULL) the columns of
 * its n rows follow.  eigsrt(d, n) / eigsrt(d, v, n) (eigen_solver.C:1442-1498;
 * the vector-free one keeps the last of equal values, >=) */
void orc_eigsrt(double *d, double *Q, int ld, int n) {
  for (int i = 0; i < n - 1; i++) {
    int k = i;
    double p = d[i];
    for (int j = i + 1; j < n; j++)
      if (Q ? d[j] > p : d[j] >= p) {
        p = d[j];
        k = j;
      }
    if (k != i) {
      d[k] = d[i];
      d[i] = p;
      if (Q)
        for (int j = 0; j < n; j++) {
          const double t = Q[j * ld + i];
          Q[j * ld + i] = Q[j * ld + k];
          Q[j * ld + k] = t;
        }
    }
  }
}

typedef struct {
  orc_mdagm_fn op;
  void *ctx;
  long n;
  int neg_lanczos, neg_conv; /* RitzMatOper NEG_MATPCDAG_MATPC for the filter / the check */
  int Npol;
  double c0, c1;
  double *tmp1, *tmp2; /* the filter's work vectors (cheby_arg->tmp1/tmp2) */
} LzCtx;

/* RitzMat(out, in) for MATPCDAG_MATPC / NEG_MATPCDAG_MATPC (d_op_dwf.C:787-840) */
static void lz_ritz(const LzCtx *z, int neg, double *out, const double *in) {
  double dummy;
  z->op(z->ctx, out, in, &dummy);
  if (neg)
    for (long q = 0; q < z->n; q++) out[q] = -out[q];
}

/* out = T_Npol(Q) in with Q = (2 A - (a + b)) / ... as the reference writes
 * it: 2Q = c1 (c0 A - 1); T_0 = 1, T_1 = Q, T_{k+1} = 2 Q T_k - T_{k-1}.
 * DiracOpDwf::RitzMat(out, in, cheby_arg) (d_op_dwf.C:852-960), Npol >= 2. */
static void lz_cheby(const LzCtx *z, double *out, const double *in) {
  const long n = z->n;
  double *tmp = z->tmp1, *tmp2 = z->tmp2;
  memcpy(tmp2, in, sizeof(double) * n);
  lz_ritz(z, z->neg_lanczos, tmp, in);
  for (long q = 0; q < n; q++) tmp[q] *= 0.5 * z->c1 * z->c0;
  for (long q = 0; q < n; q++) tmp[q] += -0.5 * z->c1 * in[q];
  for (int i = 2; i <= z->Npol; i++) {
    lz_ritz(z, z->neg_lanczos, out, tmp);
    for (long q = 0; q < n; q++) out[q] *= z->c1 * z->c0;
    for (long q = 0; q < n; q++) out[q] += -z->c1 * tmp[q];
    for (long q = 0; q < n; q++) out[q] += -1.0 * tmp2[q];
    if (i != z->Npol) {
      double *sw = tmp2;
      tmp2 = tmp;
      tmp = sw;
      memcpy(tmp, out, sizeof(double) * n);
    }
  }
}

static double lz_ddot(const double *a, const double *b, long n) {
  double s = 0.0;
  for (long q = 0; q < n; q++) s += a[q] * b[q];
  return s;
}

/* lanczos_GramSchm_test, float form (eigen_solver.C:1341-1390): r rounded to
 * float, then for each V_i: xp = <V_i, r> (rounded to float), r -= xp V_i in
 * float; r back to double.  The reference accumulates each dot product in
 * float; here it is accumulated in double and rounded. */
static void lz_gram_schm_f(double *r, float **V, int nvec, long n) {
  float *rf = malloc(sizeof(float) * n);
  for (long q = 0; q < n; q++) rf[q] = (float)r[q];
  for (int i = 0; i < nvec; i++) {
    double sr = 0.0, si = 0.0;
    for (long q = 0; q < n; q += 2) {
      sr += (double)V[i][q] * rf[q] + (double)V[i][q + 1] * rf[q + 1];
      si += (double)V[i][q] * rf[q + 1] - (double)V[i][q + 1] * rf[q];
    }
    const float xr = -(float)sr, xi = -(float)si;
    for (long q = 0; q < n; q += 2) {
      const float vr = V[i][q], vi = V[i][q + 1];
      rf[q] += xr * vr - xi * vi;
      rf[q + 1] += xr * vi + xi * vr;
    }
  }
  for (long q = 0; q < n; q++) r[q] = rf[q];
  free(rf);
}

/* Lanczos steps k0..m-1 on the filtered operator: V[k0] = r / |r| and the
 * three-term recurrence with a float Gram-Schmidt pass against V[0..k]
 * after each step; alpha, beta: the tridiagonal.  DiracOp::lanczos
 * (lanczos.C:756-883). */
static void lz_steps(const LzCtx *z, int k0, int m, double *Apsi, double *r, float **V, double *alpha, double *beta,
                     double *vtmp, double *vtmp2) {
  const long n = z->n;
  (void)Apsi;
  const double ff = sqrt(lz_ddot(r, r, n));
  for (long q = 0; q < n; q++) vtmp[q] = r[q] * (1.0 / ff);
  for (long q = 0; q < n; q++) V[k0][q] = (float)vtmp[q];
  for (int k = k0; k < m; k++) {
    for (long q = 0; q < n; q++) vtmp[q] = V[k][q];
    lz_cheby(z, r, vtmp);
    if (k > 0) {
      for (long q = 0; q < n; q++) vtmp2[q] = V[k - 1][q];
      for (long q = 0; q < n; q++) r[q] += -beta[k - 1] * vtmp2[q];
    }
    alpha[k] = lz_ddot(vtmp, r, n);
    for (long q = 0; q < n; q++) r[q] += -alpha[k] * vtmp[q];
    beta[k] = sqrt(lz_ddot(r, r, n));
    if (k > 0) lz_gram_schm_f(r, V, k + 1, n);
    if (k == 0 || k + 1 < m) {
      for (long q = 0; q < n; q++) vtmp[q] = r[q] * (1.0 / beta[k]);
      for (long q = 0; q < n; q++) V[k + 1][q] = (float)vtmp[q];
    }
  }
}

/* V[k] <- sum_j V[j] Q[j][k] for every k < m (double sums, float store),
 * the j order increasing; entries of Q with |Q| <= qmin left out */
static void lz_rotate(float **V, const double *Q, int m, long n, double qmin) {
  double *acc = malloc(sizeof(double) * m);
  for (long q = 0; q < n; q++) {
    for (int k = 0; k < m; k++) acc[k] = 0.0;
    for (int k = 0; k < m; k++)
      for (int j = 0; j < m; j++) {
        const double w = Q[j * m + k];
        if (fabs(w) > qmin || (qmin < 0 && w != 0.0)) acc[k] += (double)V[j][q] * w;
      }
    for (int k = 0; k < m; k++) V[k][q] = (float)acc[k];
  }
  free(acc);
}

/* DiracOp::ImpResLanczos (d_op_base/comsrc/lanczos.C:193-745), step for
 * step, for the DWF / Mobius Chebyshev-filtered RitzMat: m = nk + np float
 * Lanczos vectors V (V[0] the start vector); the initial m-step
 * factorisation; per restart the np unwanted Ritz values of the m x m
 * tridiagonal (tqri, sorted descending) as exact shifts of np implicit QR
 * steps (QRtrf), V rotated by Q (its band structure: Q[j][k] = 0 for
 * j > k + np), the residual r = Q[m-1][nk-1] r + beta[nk-1] V[nk]; every
 * conv_check restarts the Ritz vectors of the leading nk block checked
 * against the unfiltered RitzMat (|A v - (v.Av/|v|) v| / |v| < stop_res
 * for the first nt); then np more Lanczos steps.  At the end V[0..m) are
 * the Ritz vectors of the leading nk block (entries |Q| <= 1e-16 skipped,
 * as the reference does) and alpha[0..nt) their Rayleigh quotients on
 * the unfiltered operator (alpha[nt..m): the tridiagonal's diagonal, as the
 * reference leaves it).
 * Returns the restart count; -1 on a NaN residual (the reference exits).
 * The filter: c1 = 2 (a+b)/(a-b), c0 = 2/(a+b), a = p0^2,
 * b = (p1 + |eigen_shift|)^2. */
int orc_lanczos(orc_mdagm_fn op, void *ctx, int neg_lanczos, int neg_conv, long n, float **V, double *alpha, int nk,
                int nt, int np, int maxiters, double stop_res, int conv_check, int Npol, double p0, double p1,
                double eigen_shift) {
  const int m = nk + np;
  LzCtx z;
  z.op = op;
  z.ctx = ctx;
  z.n = n;
  z.neg_lanczos = neg_lanczos;
  z.neg_conv = neg_conv;
  z.Npol = Npol;
  const double a = p0 * p0, b = (p1 + fabs(eigen_shift)) * (p1 + fabs(eigen_shift));
  z.c1 = 2.0 * (a + b) / (a - b);
  z.c0 = 2.0 / (a + b);
  z.tmp1 = malloc(sizeof(double) * n);
  z.tmp2 = malloc(sizeof(double) * n);
  double *r = malloc(sizeof(double) * n), *Apsi = malloc(sizeof(double) * n);
  double *vtmp = malloc(sizeof(double) * n), *vtmp2 = malloc(sizeof(double) * n);
  double *beta = calloc(m, sizeof(double)), *ttbeta = malloc(sizeof(double) * m);
  double *shifts = malloc(sizeof(double) * m), *Q = malloc(sizeof(double) * m * m);
  int result = 0;
  for (long q = 0; q < n; q++) r[q] = V[0][q];
  for (int j = 0; j < m; j++) alpha[j] = 0.0;
  lz_steps(&z, 0, m, Apsi, r, V, alpha, beta, vtmp, vtmp2);
  int it = 1;
  while (it <= maxiters) {
    memcpy(shifts, alpha, sizeof(double) * m);
    memcpy(ttbeta, beta, sizeof(double) * m);
    for (int j = 0; j < m * m; j++) Q[j] = 0.0;
    for (int j = 0; j < m; j++) Q[j * m + j] = 1.0;
    orc_tqri(shifts, ttbeta, m, m, Q, m);
    orc_eigsrt(shifts, NULL, m, m);
    for (int j = 0; j < m * m; j++) Q[j] = 0.0;
    for (int j = 0; j < m; j++) Q[j * m + j] = 1.0;
    for (int i = 0; i < np; i++) orc_qrtrf(alpha, beta, m, Q, m, shifts[nk + i], 0, m - 1);
    lz_rotate(V, Q, m, n, -1.0);
    for (long q = 0; q < n; q++) r[q] *= Q[(m - 1) * m + nk - 1];
    if (nk < m) {
      for (long q = 0; q < n; q++) Apsi[q] = V[nk][q];
      for (long q = 0; q < n; q++) Apsi[q] *= beta[nk - 1];
      for (long q = 0; q < n; q++) r[q] += Apsi[q];
    }
    beta[nk - 1] = sqrt(lz_ddot(r, r, n));
    if (it % conv_check == 0) {
      int Ndone = 0;
      memcpy(shifts, alpha, sizeof(double) * m);
      memcpy(ttbeta, beta, sizeof(double) * m);
      for (int j = 0; j < m * m; j++) Q[j] = 0.0;
      for (int j = 0; j < m; j++) Q[j * m + j] = 1.0;
      orc_tqri(shifts, ttbeta, nk, m, Q, m);
      orc_eigsrt(shifts, Q, m, m);
      for (int k = 0; k < nk; k++) {
        for (long q = 0; q < n; q++) vtmp[q] = 0.0;
        for (int j = 0; j < nk; j++) {
          for (long q = 0; q < n; q++) vtmp2[q] = V[j][q];
          for (long q = 0; q < n; q++) vtmp[q] = Q[j * m + k] * vtmp2[q] + vtmp[q];
        }
        lz_ritz(&z, z.neg_conv, Apsi, vtmp);
        const double bt = sqrt(lz_ddot(vtmp, vtmp, n));
        const double alp = lz_ddot(Apsi, vtmp, n) / bt;
        for (long q = 0; q < n; q++) Apsi[q] = -alp * vtmp[q] + Apsi[q];
        const double rnorm = sqrt(lz_ddot(Apsi, Apsi, n)) / bt;
        if (rnorm < stop_res && k < nt) Ndone++;
        if (isnan(rnorm)) {
          result = -1;
          goto done;
        }
      }
      if (Ndone == nt) break;
    }
    lz_steps(&z, nk, m, Apsi, r, V, alpha, beta, vtmp, vtmp2);
    it++;
  }
  if (it == maxiters + 1) it--;
  memcpy(shifts, alpha, sizeof(double) * m);
  memcpy(ttbeta, beta, sizeof(double) * m);
  for (int j = 0; j < m * m; j++) Q[j] = 0.0;
  for (int j = 0; j < m; j++) Q[j * m + j] = 1.0;
  orc_tqri(shifts, ttbeta, nk, m, Q, m);
  orc_eigsrt(shifts, Q, m, m);
  lz_rotate(V, Q, m, n, 1e-16);
  for (int i = 0; i < nt; i++) {
    for (long q = 0; q < n; q++) vtmp[q] = V[i][q];
    lz_ritz(&z, z.neg_conv, Apsi, vtmp);
    alpha[i] = lz_ddot(Apsi, vtmp, n);
  }
  result = it;
done:
  free(z.tmp1);
  free(z.tmp2);
  free(r);
  free(Apsi);
  free(vtmp);
  free(vtmp2);
  free(beta);
  free(ttbeta);
  free(shifts);
  free(Q);
  return result;
}

/* DiracOp::InvLowModeApprox (d_op_base/comsrc/inv_lowmode_approx.C:272-512,
 * the plain cache path at :450-500): out[i] = 0, then for k = 0..neig-1
 * z_i = <v_k, in_i> / eval_k (v_k float, widened) and out_i = z_i v_k + out_i.
 * square: the cached eigenvalues are squared first (MAT_HERM, MATPC_HERM). */
void orc_inv_lowmode_approx(double **out, double **in, int len, float **evecs, const double *evals, int neig,
                            long n, int square) {
  double *v = malloc(sizeof(double) * n);
  for (int i = 0; i < len; i++) memset(out[i], 0, sizeof(double) * n);
  for (int k = 0; k < neig; k++) {
    for (long q = 0; q < n; q++) v[q] = evecs[k][q];
    const double ev = square ? evals[k] * evals[k] : evals[k];
    for (int i = 0; i < len; i++) {
      const cplx z = cdot(v, in[i], n) / ev;
      caxpy(out[i], z, v, out[i], n);
    }
  }
  free(v);
}
