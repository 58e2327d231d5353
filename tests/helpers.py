"""Shared helpers for the tests: seeded inputs and oracle wrappers."""
from __future__ import annotations

import ctypes as C

import numpy as np

from oracle.loader import MATPC_FN, MDAGM_FN, OracleGeom, OracleMobius, p


def rel(a, b) -> float:
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def vh_of(L) -> int:
    return int(np.prod(L)) // 2


def s_inner(v, L, ls, layout):
    """A full WILSON-order fermion field in the S_INNER CANONICAL order
    [lexicographic site][s][24] that FforceWilsonType reads
    (Fconvert(S_INNER, CANONICAL)); layout "dwf" (Wilson/DWF halves [odd][even],
    slice s of the odd half holding 4D parity (s+1)%2) or "mobius" ([even][odd],
    one 4D parity per half)."""
    lx, ly, lz, lt = L
    vh = lx * ly * lz * lt // 2
    t, z, y, x = np.meshgrid(*(np.arange(n) for n in (lt, lz, ly, lx)), indexing="ij")
    x, y, z, t = (a.ravel() for a in (x, y, z, t))
    par = (x + y + z + t) & 1
    cb = x // 2 + (lx // 2) * (y + ly * (z + lz * t))
    pos = np.empty((x.size, ls), dtype=np.int64)
    for s in range(ls):
        if layout == "dwf":
            pos[:, s] = np.where(((par + s) & 1) == 1, 0, ls * vh) + s * vh + cb
        else:
            pos[:, s] = np.where(par == 1, ls * vh, 0) + s * vh + cb
    return np.asarray(v).reshape(-1, 24)[pos.ravel()].ravel()


class OracleOps:
    """The oracle's operators on one geometry (gauge field without signs)."""

    def __init__(self, O, L, u, ls=1, bc=(1, 1, 1, -1), m5=1.8, b=1.5, c=0.5, a5_inv=1.0):
        self.O = O
        self.L = tuple(L)
        self.u = np.ascontiguousarray(u)
        self.ls = ls
        self.a5_inv = a5_inv
        self.g = OracleGeom.make(L, ls, bc, a5_inv)
        self.g1 = OracleGeom.make(L, 1, bc)
        self.m5 = m5
        self.mp = OracleMobius()
        if ls > 1:
            O.orc_mobius_params_a5(C.byref(self.mp), ls, b, c, m5, a5_inv)
        self.n = 24 * ls * vh_of(L)

    def set_zmobius(self, b, c):
        """complex per-slice b_s, c_s with kappa_b, K as DiracOpZMobius sets them
        (d_op_zmobius.C:246-292, a5inv = 1)"""
        for s in range(self.ls):
            kb = 1 / (2 * (b[s] * (4 - self.m5) + self.a5_inv))
            kc = 1 / (2 * (c[s] * (4 - self.m5) - self.a5_inv))
            for name, v in (("b", b[s]), ("c", c[s]), ("kappa_b", kb), ("K", kb / kc)):
                arr = getattr(self.mp, name)
                arr[2 * s], arr[2 * s + 1] = complex(v).real, complex(v).imag

    def z(self):
        return np.zeros(self.n)

    def wilson_dslash(self, x, cb, dag):
        y = self.z()
        self.O.orc_wilson_dslash(C.byref(self.g1), p(y), p(self.u), p(x), cb, dag)
        return y

    def wilson_mdagm(self, x, kappa):
        y = self.z()
        d = C.c_double()
        self.O.orc_wilson_mdagm(C.byref(self.g1), p(y), p(self.u), p(x), kappa, C.byref(d))
        return y, d.value

    def wilson_m(self, x, kappa, dag):
        y = self.z()
        self.O.orc_wilson_m(C.byref(self.g1), p(y), p(self.u), p(x), kappa, dag)
        return y

    def dwf_dslash(self, x, mass, cb, dag):
        y = self.z()
        self.O.orc_dwf_dslash(C.byref(self.g), p(y), p(self.u), p(x), mass, cb, dag)
        return y

    def dwf_m(self, x, mass, dag):
        y = self.z()
        self.O.orc_dwf_m(C.byref(self.g), p(y), p(self.u), p(x), mass, self.m5, dag)
        return y

    def dwf_mdagm(self, x, mass):
        y = self.z()
        d = C.c_double()
        self.O.orc_dwf_mdagm(C.byref(self.g), p(y), p(self.u), p(x), mass, self.m5, C.byref(d))
        return y, d.value

    def mobius_dslash_4(self, x, mass, cb, dag):
        y = self.z()
        self.O.orc_mobius_dslash_4(C.byref(self.g), C.byref(self.mp), p(y), p(self.u), p(x), cb, dag, mass)
        return y

    def mobius_m5inv(self, x, mass, dag):
        y = np.ascontiguousarray(x).copy()
        self.O.orc_mobius_m5inv(C.byref(self.g), C.byref(self.mp), p(y), mass, dag)
        return y

    def mobius_m5(self, x, mass):
        y = np.ascontiguousarray(x).copy()
        self.O.orc_mobius_m5(C.byref(self.g), C.byref(self.mp), p(y), mass)
        return y

    def matinv(self, kind, src, out0=None, mass=0.0, kappa=0.0, stop_rsd=1e-8, max_num_iter=10000):
        """DiracOp*::MatInv on both checkerboards (see oracle.h for the halves' order)"""
        out = np.zeros(2 * self.n) if out0 is None else np.ascontiguousarray(out0).copy()
        src = np.ascontiguousarray(src)
        tr = C.c_double()
        if kind == "wilson":
            it = self.O.orc_wilson_matinv(C.byref(self.g1), p(out), p(self.u), p(src), kappa, stop_rsd,
                                          max_num_iter, C.byref(tr))
        elif kind == "dwf":
            it = self.O.orc_dwf_matinv(C.byref(self.g), p(out), p(self.u), p(src), mass, self.m5, stop_rsd,
                                       max_num_iter, C.byref(tr))
        else:
            it = self.O.orc_mobius_matinv(C.byref(self.g), C.byref(self.mp), p(out), p(self.u), p(src), mass,
                                          stop_rsd, max_num_iter, C.byref(tr))
        return out, it, tr.value

    def mobius_m(self, x, mass, dag):
        y = self.z()
        self.O.orc_mobius_m(C.byref(self.g), C.byref(self.mp), p(y), p(self.u), p(x), mass, dag)
        return y

    def mobius_mdagm(self, x, mass):
        y = self.z()
        d = C.c_double()
        self.O.orc_mobius_mdagm(C.byref(self.g), C.byref(self.mp), p(y), p(self.u), p(x), mass, C.byref(d))
        return y, d.value

    def mobius_m_pc(self, x, mass, dag, pc):
        """MatPc / MatPcDag under the preconditioning pc (zmobius_m.C:40-74)"""
        y = self.z()
        self.O.orc_mobius_m_pc(C.byref(self.g), C.byref(self.mp), p(y), p(self.u), p(np.ascontiguousarray(x)), mass,
                               dag, pc)
        return y

    def mobius_mdagm_pc(self, x, mass, pc):
        y = self.z()
        d = C.c_double()
        self.O.orc_mobius_mdagm_pc(C.byref(self.g), C.byref(self.mp), p(y), p(self.u), p(np.ascontiguousarray(x)),
                                   mass, C.byref(d), pc)
        return y, d.value

    def mobius_matinv_pc(self, src, mass, pc, stop_rsd=1e-8, max_num_iter=10000):
        """DiracOpMobius::MatInv under the preconditioning pc, zero guess"""
        out = np.zeros(2 * self.n)
        tr = C.c_double()
        it = self.O.orc_mobius_matinv_pc(C.byref(self.g), C.byref(self.mp), p(out), p(self.u),
                                         p(np.ascontiguousarray(src)), mass, stop_rsd, max_num_iter, C.byref(tr), pc)
        return out, it, tr.value

    # ---- solvers over an operator callback
    def _op(self, kind, mass, kappa, pc=2):
        O, u, g = self.O, self.u, self.g

        def fn(ctx, out, inp, dot):
            if kind == "wilson":
                O.orc_wilson_mdagm(C.byref(self.g1), out, p(u), inp, kappa, dot)
            elif kind == "dwf":
                O.orc_dwf_mdagm(C.byref(g), out, p(u), inp, mass, self.m5, dot)
            elif pc == 2:
                O.orc_mobius_mdagm(C.byref(g), C.byref(self.mp), out, p(u), inp, mass, dot)
            else:
                O.orc_mobius_mdagm_pc(C.byref(g), C.byref(self.mp), out, p(u), inp, mass, dot, pc)

        return MDAGM_FN(fn)

    def invcg(self, kind, src, sol0=None, mass=0.0, kappa=0.0, stop_rsd=1e-8, max_num_iter=10000, shift=None, pc=2):
        sol = np.zeros(self.n) if sol0 is None else np.ascontiguousarray(sol0).copy()
        tr = C.c_double()
        fn = self._op(kind, mass, kappa, pc)
        sh = C.c_double(shift) if shift is not None else None
        it = self.O.orc_invcg(fn, None, self.n, p(sol), p(src), 0.0, stop_rsd, max_num_iter, C.byref(tr),
                              C.byref(sh) if sh is not None else None)
        return sol, it, tr.value

    def minresext(self, kind, phi, v, mass=0.0, kappa=0.0):
        """DiracOp::MinResExt: returns (psi, v orthonormalised, vm, error)"""
        v = [np.ascontiguousarray(x).copy() for x in v]
        vm = [np.zeros(self.n) for _ in v]
        psi = np.zeros(self.n)
        err = C.c_double()
        pv = (C.POINTER(C.c_double) * max(1, len(v)))(*[p(x) for x in v])
        pm = (C.POINTER(C.c_double) * max(1, len(v)))(*[p(x) for x in vm])
        self.O.orc_minresext(self._op(kind, mass, kappa), None, self.n, p(psi), p(np.ascontiguousarray(phi)), pv,
                             pm, len(v), C.byref(err))
        return psi, v, vm, err.value

    def inveigcg(self, kind, src, nev, m, mass=0.0, kappa=0.0, stop_rsd=1e-8, max_num_iter=10000, U=None,
                 invH=None, restart=()):
        """DiracOp::InvEigCg (inv_eig_cg.C:129-635): returns (sol, iter,
        true_res, V, M)"""
        sol = np.zeros(self.n)
        V = [np.zeros(self.n) for _ in range(max(m, 1))]
        M = np.zeros(max(2 * nev, 1))
        U = [np.ascontiguousarray(u, dtype=np.float64) for u in (U or [])]
        def_len = len(U)
        ih = np.ascontiguousarray(invH if invH is not None else np.zeros(1), dtype=np.complex128).view(np.float64)
        rs = np.ascontiguousarray(list(restart) or [0.0], dtype=np.float64)
        tr = C.c_double()
        pv = (C.POINTER(C.c_double) * len(V))(*[p(x) for x in V])
        pu = (C.POINTER(C.c_double) * max(1, def_len))(*([p(x) for x in U] or [None]))
        it = self.O.orc_inveigcg(self._op(kind, mass, kappa), None, self.n, p(sol), p(np.ascontiguousarray(src)),
                                 stop_rsd, max_num_iter, nev, m, pv, p(M), def_len, pu, p(np.ascontiguousarray(ih)),
                                 p(rs), len(restart), C.byref(tr))
        return sol, it, tr.value, V, M

    def ritz(self, kind, psi_all, mass=0.0, kappa=0.0, neg=False, RsdR_a=1e-10, RsdR_r=1e-8, Rsdlam=1e-10,
             Cutl_zero=0.0, n_renorm=10, Kalk_Sim=0, N_min=0, N_max=1000, Cv_fact=0.0, MaxCG=10000, ProjApsiP=0):
        """DiracOp::Ritz (ritz.C:152-532) on the last of psi_all (updated in
        place): returns (iterations, lambda)"""
        lam = C.c_double()
        pv = (C.POINTER(C.c_double) * len(psi_all))(*[p(x) for x in psi_all])
        k = self.O.orc_ritz(self._op(kind, mass, kappa), None, 1 if neg else 0, self.n, pv, len(psi_all), RsdR_a,
                            RsdR_r, Rsdlam, Cutl_zero, n_renorm, Kalk_Sim, N_min, N_max, Cv_fact, MaxCG, ProjApsiP,
                            C.byref(lam))
        return k, lam.value

    def ritz_eig(self, kind, psi, mass=0.0, kappa=0.0, neg=False, RsdR_a=1e-10, RsdR_r=1e-8, Rsdlam=1e-10,
                 Cv_fact=0.1, n_renorm=10, Kalk_Sim=1, N_min=5, N_max=50, MaxCG=10000, ProjApsiP=0, N_KS_max=50):
        """DiracOpWilsonTypes::RitzEig (eigen_wilson.C:89-586) on the vectors
        psi (updated in place): returns (total Ritz iterations or the
        reference's negative code, lambda_H (2 len(psi)), valid_eig)"""
        lam = np.zeros(2 * len(psi))
        valid = (C.c_int * len(psi))()
        pv = (C.POINTER(C.c_double) * len(psi))(*[p(x) for x in psi])
        r = self.O.orc_ritz_eig(self._op(kind, mass, kappa), None, 1 if neg else 0, self.n, pv, len(psi), RsdR_a,
                                RsdR_r, Rsdlam, Cv_fact, n_renorm, Kalk_Sim, N_min, N_max, MaxCG, ProjApsiP, N_KS_max,
                                p(lam), valid)
        return r, lam, np.array(valid[:])

    def force_vecs(self, kind, chi, mass=0.0, kappa=0.0):
        """DiracOpWilson / DiracOpDwf::CalcHmdForceVecs (d_op_wilson.C:466-507,
        d_op_dwf.C:682-733): v1 = (chi, D chi), v2 = (psi, D^dag psi) with
        psi = -kappa^2 MatPc chi, full fields in WILSON order"""
        if kind == "wilson":
            psi = -kappa * kappa * self.wilson_m(chi, kappa, 0)
            rho, sigma = self.wilson_dslash(chi, 1, 0), self.wilson_dslash(psi, 1, 1)
        else:
            k5 = 1 / (2 * (4 + self.a5_inv - self.m5))
            psi = -k5 * k5 * self.dwf_m(chi, mass, 0)
            rho, sigma = self.dwf_dslash(chi, mass, 1, 0), self.dwf_dslash(psi, mass, 1, 1)
        return np.concatenate([chi, rho]), np.concatenate([psi, sigma])

    def mobius_booee(self, x, mass):
        y = self.z()
        self.O.orc_mobius_booee(C.byref(self.g), C.byref(self.mp), p(y), p(np.ascontiguousarray(x)), mass)
        return y

    # ---- unpreconditioned operators on full vectors [half 0][half 1] in
    # the reference's storage order (Wilson, DWF: [odd][even]; Mobius
    # [even][odd]), composed from the pinned kernels
    def _hop(self, kind, x, mass, cb, dag):
        if kind == "wilson":
            return self.wilson_dslash(x, cb, dag)
        return self.dwf_dslash(x, mass, cb, dag)

    def mat(self, kind, x, mass=0.0, kappa=0.0, dag=0):
        """DiracOpWilson / DiracOpDwf::Mat, MatDag (d_op_wilson.C:362-424,
        d_op_dwf.C:541-627): out_0 = in_0 - kappa D(in_1, CHKB_EVEN),
        out_1 = in_1 - kappa D(in_0, CHKB_ODD); DiracOpMobius::Mat
        (d_op_mobius.C:735-795): out_0 = (1 + a5inv K D5) in_0 - kappa_b
        Dslash_4(in_1, CHKB_ODD), out_1 = (1 + a5inv K D5) in_1 - kappa_b
        Dslash_4(in_0, CHKB_EVEN)"""
        x = np.ascontiguousarray(x)
        h = x.size // 2
        x0, x1 = x[:h], x[h:]
        if kind != "mobius":
            k = kappa if kind == "wilson" else 1 / (2 * (4 + self.a5_inv - self.m5))
            return np.concatenate([x0 - k * self._hop(kind, x1, mass, 0, dag), x1 - k * self._hop(kind, x0, mass, 1, dag)])
        if dag:
            raise ValueError("the reference's DiracOpMobius::MatDag stops with an error")
        kb = self.mp.kappa_b[0]  # real part of kappa_b(s = 0) (the array holds re, im pairs)

        def m5(v):
            return v + self.a5_inv * (self.mobius_m5(v, mass) - v)
        return np.concatenate([m5(x0) - kb * self.mobius_dslash_4(x1, mass, 1, 0),
                               m5(x1) - kb * self.mobius_dslash_4(x0, mass, 0, 0)])

    def gamma5_reflect(self, kind, y):
        """MatHerm's left factor: gamma_5 (reals 12-23 negated,
        DiracOpWilsonTypes::MultGamma 15) after, for DWF and Mobius, the
        reflection s -> Ls-1-s of FdwfBase::Freflex (f_dwf_base.C:1693-1790),
        which for even Ls takes each slice from the other half"""
        y = np.ascontiguousarray(y).reshape(2, max(self.ls, 1), -1, 24).copy()
        if kind != "wilson":
            y = y[::-1, ::-1] if self.ls % 2 == 0 else y[:, ::-1]
        y = y.copy()
        y[..., 12:] *= -1
        return y.reshape(-1)

    def matherm(self, kind, x, mass=0.0, kappa=0.0):
        return self.gamma5_reflect(kind, self.mat(kind, x, mass, kappa, 0))

    def mobius_mdagm_shift(self, x, mass, mu):
        """zmobius_mdagm_shift (zmobius_mdagm.C:79-135): out = M^+ M x - 2 mu
        R g5 M x + mu^2 x with R g5 = ReflectAndMultGamma5 (slice s from
        Ls-1-s within the checkerboard, reals 12-23 negated); dot = |M x|^2"""
        mx = self.mobius_m(x, mass, 0)
        out = self.mobius_m(mx, mass, 1)
        r = np.ascontiguousarray(mx).reshape(self.ls, -1, 24)[::-1].copy()
        r[..., 12:] *= -1
        return out - 2 * mu * r.reshape(-1) + mu * mu * np.asarray(x), float(mx @ mx)

    def mobius_force_vecs(self, phi1, phi2, mass):
        """DiracOpMobius::CalcHmdForceVecs(v1, v2, phi1, phi2), SYM2
        (d_op_mobius.C:1015-1100): full fields [even half][odd half]"""
        phi2 = self.mobius_m5inv(phi2, mass, 0)  # the reference overwrites phi2 with this
        v2_e = self.mobius_booee(self.mobius_m5inv(self.mobius_dslash_4(phi2, mass, 1, 0), mass, 0), mass)
        v2_o = self.mobius_booee(phi2, mass)
        v1_e = self.mobius_m5inv(self.mobius_dslash_4(phi1, mass, 1, 1), mass, 1)
        return np.concatenate([v1_e, phi1]), np.concatenate([v2_e, v2_o])

    def mobius_fforce(self, frm, step, mass, mom=None):
        """Fmobius::EvolveMomFforce(mom, frm, mass, step) (f_mobius.C:847-887):
        phi1 = MatPc frm, phi2 = frm, FforceWilsonType with coef = -step"""
        v1, v2 = self.mobius_force_vecs(self.mobius_m(frm, mass, 0), frm, mass)
        vol = int(np.prod(self.L))
        m = np.zeros(4 * vol * 18) if mom is None else np.ascontiguousarray(mom).copy()
        out = np.zeros(3)
        self.O.orc_fforce_wilson_type(C.byref(self.g), p(m), p(self.u), p(v1), p(v2), -step, p(out))
        return m, tuple(out)

    def fforce(self, kind, chi, dt, mass=0.0, kappa=0.0, mom=None):
        """Fwilson / FdwfBase::EvolveMomFforce: returns (mom + force, (L1, L2, Linf))"""
        v1, v2 = self.force_vecs(kind, chi, mass, kappa)
        vol = int(np.prod(self.L))
        m = np.zeros(4 * vol * 18) if mom is None else np.ascontiguousarray(mom).copy()
        out = np.zeros(3)
        g = self.g1 if kind == "wilson" else self.g
        self.O.orc_fforce(C.byref(g), p(m), p(self.u), p(v1), p(v2), dt, p(out))
        return m, tuple(out)

    def bicgstab(self, kind, chi, n=1, mass=0.0, kappa=0.0, stop_rsd=1e-8, max_num_iter=10000, psi0=None):
        """BiCGstab(n) on MatPc (bicgstab.C:35-229): returns psi, k, true_res"""
        O, u = self.O, self.u

        def fn(ctx, out, inp):
            if kind == "wilson":
                O.orc_wilson_m(C.byref(self.g1), out, p(u), inp, kappa, 0)
            elif kind == "dwf":
                O.orc_dwf_m(C.byref(self.g), out, p(u), inp, mass, self.m5, 0)
            else:
                O.orc_mobius_m(C.byref(self.g), C.byref(self.mp), out, p(u), inp, mass, 0)

        cb = MATPC_FN(fn)
        psi = np.zeros(self.n) if psi0 is None else np.ascontiguousarray(psi0).copy()
        tr = C.c_double()
        k = self.O.orc_bicgstab(cb, None, self.n, p(psi), p(np.ascontiguousarray(chi)), 0.0, n, stop_rsd,
                                max_num_iter, C.byref(tr))
        return psi, k, tr.value

    def minvcg(self, kind, chi, shifts, rsd, mass=0.0, kappa=0.0, type=1, alpha=None, max_num_iter=10000,
               psi0=None):
        n = len(shifts)
        npsi = 1 if type == 0 else n
        psi = [np.zeros(self.n) if psi0 is None else np.ascontiguousarray(psi0[k]).copy() for k in range(npsi)]
        arr = (C.POINTER(C.c_double) * npsi)(*[p(x) for x in psi])
        rs = np.ascontiguousarray(rsd, dtype=np.float64).copy()
        sh = np.ascontiguousarray(shifts, dtype=np.float64)
        al = np.ascontiguousarray(alpha if alpha is not None else np.ones(n), dtype=np.float64)
        fn = self._op(kind, mass, kappa)
        chi = np.ascontiguousarray(chi)
        k = self.O.orc_minvcg(fn, None, self.n, arr, p(chi), float(chi @ chi), p(sh), n, p(rs), type, p(al),
                              max_num_iter)
        return psi, k, rs


def mix_pairs(V, seed):
    """rotate pairs of vectors by random 2 x 2 unitaries (complex vectors as re/im pairs)"""
    rng = np.random.default_rng(seed)
    Wc = [v[0::2] + 1j * v[1::2] for v in V]
    out = []
    for k in range(0, len(Wc), 2):
        a, b = rng.normal(size=2) + 1j * rng.normal(size=2)
        u = np.array([[a, -np.conj(b)], [b, np.conj(a)]]) / np.sqrt(abs(a) ** 2 + abs(b) ** 2)
        out += [u[0, 0] * Wc[k] + u[0, 1] * Wc[k + 1], u[1, 0] * Wc[k] + u[1, 1] * Wc[k + 1]]
    res = []
    for w in out:
        r = np.empty(2 * w.size)
        r[0::2], r[1::2] = w.real, w.imag
        res.append(r)
    return res
