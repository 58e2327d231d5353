"""Device-resident solvers against the oracle's CG / multishift CG:
FP64 CG with the reference's bookkeeping, mixed-precision (FP32 and FP16
inner) reliable-update CG to a true residual of 1e-10, batched
right-hand sides, multishift CG, host-side failure injection, and the
BiCGstab, MinResExt, eigCG, Ritz, RitzEig and Jacobi routines."""
import ctypes as C

import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpMobius, DiracOpWilson, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, mix_pairs, rel
from oracle.loader import p

pytestmark = pytest.mark.gpu


def _wilson(oracle, L=(8, 8, 8, 8), seed=71):
    u = gen_gauge(L, seed=seed)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpWilson(lat, mass=1 / (2 * 0.12) - 4)
    return D, OracleOps(oracle, L, u, ls=1)


def test_wilson_cg_matches_oracle(oracle):
    """8^4 Wilson, kappa 0.12, stop 1e-8 (the plain CPU-runnable case)."""
    D, ops = _wilson(oracle)
    b = gen_gaussian(ops.n, seed=72)
    xo, ito, tro = ops.invcg("wilson", b, kappa=D.kappa, stop_rsd=1e-8)
    x = np.zeros(ops.n)
    r = D.InvCg(x, b, stop_rsd=1e-8)
    assert r.status == A.CONVERGED
    assert abs(r.iterations - ito) <= 1
    assert r.true_res < 1e-8
    assert rel(x, xo) < 1e-9


def test_cg_bookkeeping_and_graph_equivalence(oracle):
    D, ops = _wilson(oracle, L=(4, 4, 4, 8))
    b = gen_gaussian(ops.n, seed=73)
    x = np.zeros(ops.n)
    r = D.InvCg(x, b, stop_rsd=1e-14, max_num_iter=7)
    _, ito, _ = ops.invcg("wilson", b, kappa=D.kappa, stop_rsd=1e-14, max_num_iter=7)
    assert r.iterations == ito == 7 and r.status == A.MAX_ITER
    x1, x2 = np.zeros(ops.n), np.zeros(ops.n)
    r1 = D.InvCg(x1, b, stop_rsd=1e-10, use_graph=True, chunk=5)
    r2 = D.InvCg(x2, b, stop_rsd=1e-10, use_graph=False, chunk=3)
    assert r1.iterations == r2.iterations and np.array_equal(x1, x2)


@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE, A.HALF])
def test_dwf_cg_true_residual(oracle, prec):
    L, ls, mass = (4, 4, 4, 8), 8, 0.05
    u = gen_gauge(L, seed=81)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls)
    b = gen_gaussian(ops.n, seed=82)
    xo, ito, _ = ops.invcg("dwf", b, mass=mass, stop_rsd=1e-11)
    x = np.zeros(ops.n)
    r = D.InvCg(x, b, stop_rsd=1e-10, precision=prec)
    assert r.status == A.CONVERGED and r.true_res <= 1e-10
    assert rel(x, xo) < 1e-8
    if prec != A.DOUBLE:
        assert r.reliable_updates >= 1
        assert r.iterations < 2.0 * ito


@pytest.mark.parametrize("prec", [A.DOUBLE, A.HALF])
def test_mobius_cg_true_residual(oracle, prec):
    L, ls, mass = (4, 4, 4, 4), 8, 0.05
    u = gen_gauge(L, seed=91)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
    ops = OracleOps(oracle, L, u, ls=ls)
    b = gen_gaussian(ops.n, seed=92)
    xo, _, _ = ops.invcg("mobius", b, mass=mass, stop_rsd=1e-11)
    x = np.zeros(ops.n)
    r = D.InvCg(x, b, stop_rsd=1e-10, precision=prec)
    assert r.status == A.CONVERGED and r.true_res <= 1e-10
    assert rel(x, xo) < 1e-8


def test_multi_rhs_matches_single(oracle):
    L, ls = (4, 4, 4, 8), 4
    u = gen_gauge(L, seed=101)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=0.1, ls=ls)
    srcs = [gen_gaussian(D.f_size, seed=102 + k) for k in range(3)]
    sols = [np.zeros(D.f_size) for _ in srcs]
    res = D.InvCgMulti(sols, srcs, stop_rsd=1e-10, precision=A.SINGLE)
    for s, x, r in zip(srcs, sols, res):
        y = np.zeros(D.f_size)
        r1 = D.InvCg(y, s, stop_rsd=1e-10, precision=A.SINGLE)
        assert r.status == A.CONVERGED and r.true_res <= 1e-10
        assert r.iterations == r1.iterations
        assert rel(x, y) < 1e-12


def test_minvcg_fp64_matches_oracle(oracle):
    D, ops = _wilson(oracle, L=(4, 4, 4, 8))
    chi = gen_gaussian(ops.n, seed=111)
    shifts = [0.02, 0.2, 1.0, 5.0]
    psi_o, ko, rso = ops.minvcg("wilson", chi, shifts, [1e-10] * 4, kappa=D.kappa, type=1)
    psi = [np.zeros(ops.n) for _ in shifts]
    rs = np.full(4, 1e-10)
    k = D.MInvCG(psi, chi, float(chi @ chi), shifts, rs, type=A.MS_MULTI)
    assert abs(k - ko) <= 1
    for s in range(4):
        assert rel(psi[s], psi_o[s]) < 1e-9
        assert rs[s] / np.linalg.norm(chi) < 1e-10


def test_minvcg_single_type_and_sloppy_refine(oracle):
    D, ops = _wilson(oracle, L=(4, 4, 4, 8))
    chi = gen_gaussian(ops.n, seed=112)
    shifts = [0.01, 0.1, 1.0]
    alpha = [0.5, -1.0, 2.0]
    psi_o, _, _ = ops.minvcg("wilson", chi, shifts, [1e-10] * 3, kappa=D.kappa, type=0, alpha=alpha)
    psi = [np.zeros(ops.n)]
    rs = np.full(3, 1e-10)
    D.MInvCG(psi, chi, float(chi @ chi), shifts, rs, type=A.MS_SINGLE, alpha=alpha)
    assert rel(psi[0], psi_o[0]) < 1e-9
    # FP32 multishift + FP64 refinement of each shift
    psi2 = [np.zeros(ops.n) for _ in shifts]
    rs2 = np.full(3, 1e-10)
    D.MInvCG(psi2, chi, float(chi @ chi), shifts, rs2, type=A.MS_MULTI, precision=A.SINGLE)
    for s, sh in enumerate(shifts):
        Ax, _ = ops.wilson_mdagm(psi2[s], D.kappa)
        assert rel(Ax + sh * psi2[s], chi) <= 1e-10


@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE])
def test_minvcg_graph_reuse_and_recapture(oracle, prec):
    """The recurrences run as one graph launch (a WHILE node over chunks of
    iterations), instantiated on the first call and kept on the operator:
    a second call replays it and gives the first call's result bit for bit;
    a change of launch shape or of the number of shifts captures it again
    and gives the same solve within rounding, with the oracle's iteration
    count."""
    D, ops = _wilson(oracle, L=(4, 4, 4, 8))
    chi = gen_gaussian(ops.n, seed=113)
    shifts = [0.05, 0.5, 2.0]
    _, ko, _ = ops.minvcg("wilson", chi, shifts, [1e-10] * 3, kappa=D.kappa, type=1)

    def run(sh):
        psi = [np.zeros(ops.n) for _ in sh]
        rs = np.full(len(sh), 1e-10)
        k = D.MInvCG(psi, chi, float(chi @ chi), sh, rs, type=A.MS_MULTI, precision=prec)
        return k, psi, rs

    k1, psi1, rs1 = run(shifts)
    if prec == A.DOUBLE:
        assert abs(k1 - ko) <= 1
    for again in range(2):
        if again:
            sites = D.hop_shape(prec)[0]
            D.set_hop_shape(prec, 64 if sites != 64 else 32, 1, 1, D.ORDER_SITES)
        k2, psi2, rs2 = run(shifts)
        assert abs(k2 - k1) <= again
        for a, b in zip(psi2, psi1):
            if again:  # other block partials: the reductions round differently
                assert rel(a, b) < 1e-9
            else:
                np.testing.assert_array_equal(a, b)
    k4, psi4, _ = run(shifts + [8.0])  # another number of shifts
    assert abs(k4 - k1) <= 1
    assert rel(psi4[0], psi1[0]) < 1e-9


def test_failure_injection_nonfinite_source(oracle):
    """A NaN planted in the host source must come back as a status, not a fault."""
    D, ops = _wilson(oracle, L=(4, 4, 4, 4))
    b = gen_gaussian(ops.n, seed=121)
    b[17] = np.nan
    x = np.zeros(ops.n)
    r = D.InvCg(x, b, stop_rsd=1e-10, max_num_iter=50)
    assert r.status == A.NONFINITE


@pytest.mark.parametrize("kind,L,ls,mass", [("wilson", (4, 4, 4, 8), 1, 0.1), ("dwf", (4, 4, 4, 8), 8, 0.05),
                                           ("mobius", (4, 4, 4, 4), 8, 0.05)])
@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE])
def test_matinv_matches_oracle(oracle, kind, L, ls, mass, prec):
    """DiracOp*::MatInv on both checkerboards against the oracle's
    restatement (d_op_wilson.C:257, d_op_dwf.C:316, d_op_mobius.C:407)."""
    u = gen_gauge(L, seed=131)
    lat = Lattice(L)
    lat.import_gauge(u)
    if kind == "wilson":
        D = DiracOpWilson(lat, mass=mass)
    elif kind == "dwf":
        D = DiracOpDwf(lat, mass=mass, ls=ls)
    else:
        D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
    ops = OracleOps(oracle, L, u, ls=ls, b=1.5, c=0.5)
    src = gen_gaussian(2 * D.f_size, seed=132)
    guess = gen_gaussian(2 * D.f_size, seed=133) * 1e-3  # a non-zero initial guess
    xo, ito, tro = ops.matinv(kind, src, out0=guess, mass=mass, kappa=D.kappa, stop_rsd=1e-12)
    x = guess.copy()
    src0 = src.copy()
    r = D.MatInv(x, src, stop_rsd=1e-12, precision=prec)
    assert np.array_equal(src, src0)  # the source is preserved
    assert r.status == A.CONVERGED and r.true_res <= 1e-12
    assert rel(x, xo) < 1e-9
    if prec == A.DOUBLE:
        assert abs(r.iterations - ito) <= 1


def test_dwf_propagator_flow_from_canonical_fields(oracle):
    """What a propagator job does around the solve: a CANONICAL gauge field and
    4D source, Ffour2five onto the walls, Fconvert to WILSON, MatInv,
    Fconvert back and Ffive2four, against the same steps on the oracle."""
    from cps_veloc_b200.dirac import StrOrd, fconvert, five2four, four2five, gconvert

    L, ls, mass = (4, 4, 4, 8), 8, 0.05
    u_w = gen_gauge(L, seed=141)
    u_c = u_w.copy()
    gconvert(L, u_c, StrOrd.CANONICAL, StrOrd.WILSON)  # as a reader would deliver it
    u = u_c.copy()
    gconvert(L, u, StrOrd.WILSON, StrOrd.CANONICAL)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls)
    src4 = gen_gaussian(24 * int(np.prod(L)), seed=142)
    src5 = four2five(L, ls, src4, 0, ls - 1)
    fconvert(L, ls, src5, StrOrd.WILSON, StrOrd.CANONICAL)
    x = np.zeros_like(src5)
    r = D.MatInv(x, src5, stop_rsd=1e-12)
    xo, _, _ = ops.matinv("dwf", src5, mass=mass, stop_rsd=1e-12)
    assert r.status == A.CONVERGED and rel(x, xo) < 1e-9
    fconvert(L, ls, x, StrOrd.CANONICAL, StrOrd.WILSON)
    prop = five2four(L, ls, x, ls - 1, 0)
    fconvert(L, ls, xo, StrOrd.CANONICAL, StrOrd.WILSON)
    assert rel(prop, five2four(L, ls, xo, ls - 1, 0)) < 1e-9


@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE])
def test_zmobius_cg_true_residual(oracle, prec):
    L, ls, mass = (4, 4, 4, 4), 8, 0.05
    u = gen_gauge(L, seed=151)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
    zb = np.array([1.5 + 0.25j * np.sin(1.0 + s) for s in range(ls)])
    D.set_zmobius(zb, zb - 1.0)
    ops = OracleOps(oracle, L, u, ls=ls)
    ops.set_zmobius(zb, zb - 1.0)
    b = gen_gaussian(ops.n, seed=152)
    xo, _, _ = ops.invcg("mobius", b, mass=mass, stop_rsd=1e-11)
    x = np.zeros(ops.n)
    r = D.InvCg(x, b, stop_rsd=1e-10, precision=prec)
    assert r.status == A.CONVERGED and r.true_res <= 1e-10
    assert rel(x, xo) < 1e-8
    with pytest.raises(A.CpsGpuError):  # MatInv stays real-only, as the reference's scaling is
        D.MatInv(np.zeros(2 * D.f_size), gen_gaussian(2 * D.f_size, seed=153))


@pytest.mark.parametrize("kind,L,ls,n,iters", [
    ("wilson", (4, 4, 4, 8), 1, 1, None), ("wilson", (4, 4, 4, 8), 1, 3, None), ("dwf", (4, 4, 4, 4), 4, 3, None),
    ("dwf", (4, 4, 4, 8), 8, 1, 6), ("mobius", (4, 4, 4, 4), 8, 2, 6), ("zmobius", (4, 4, 4, 4), 8, 1, 6)])
def test_bicgstab_matches_oracle(oracle, kind, L, ls, n, iters):
    """DiracOpWilsonTypes::BiCGstab(n) (bicgstab.C:35-229) on MatPc against the
    oracle's restatement.  Converging cases: the same k (to one sweep), the
    same solution and a true residual below stop_rsd.  On the 5D operators at
    these sizes BiCGstab(n) does not converge (in the oracle alike) and its
    iterates are chaotic: in the oracle itself a 1e-15 relative change of chi
    grows to 1e-10 by iteration 8 and to O(1) by iteration 16.  Those cases
    stop after max_num_iter = 6 and compare the iterate itself."""
    mass = 0.1
    u = gen_gauge(L, seed=161)
    lat = Lattice(L)
    lat.import_gauge(u)
    ops = OracleOps(oracle, L, u, ls=ls, b=1.5, c=0.5)
    if kind == "wilson":
        D = DiracOpWilson(lat, mass=mass)
    elif kind == "dwf":
        D = DiracOpDwf(lat, mass=mass, ls=ls)
    else:
        D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
        if kind == "zmobius":
            zb = np.array([1.5 + 0.25j * np.cos(0.5 + s) for s in range(ls)])
            D.set_zmobius(zb, zb - 1.0)
            ops.set_zmobius(zb, zb - 1.0)
    chi = gen_gaussian(D.f_size, seed=162)
    guess = gen_gaussian(D.f_size, seed=163) * 1e-3 if kind == "wilson" else np.zeros(D.f_size)
    okind = "mobius" if kind == "zmobius" else kind
    mx = iters if iters else 2000
    xo, ko, tro = ops.bicgstab(okind, chi, n=n, mass=mass, kappa=D.kappa, stop_rsd=1e-12, psi0=guess,
                               max_num_iter=mx)
    x = guess.copy()
    k, tr = D.BiCGstab(x, chi, n=n, stop_rsd=1e-12, max_num_iter=mx)
    if iters:
        assert k == ko == 1 + n * ((iters + n - 1) // n) and tr == tro == 0.0
        assert rel(x, xo) < 1e-9
        return
    assert 1 < ko < mx and abs(k - ko) <= n
    assert 0 < tr < 1e-12 * np.linalg.norm(chi)
    assert rel(x, xo) < 1e-9
    r = chi - D.MatPc(x)
    assert np.linalg.norm(r) < 2e-12 * np.linalg.norm(chi)


def test_bicgstab_zero_source_and_argument_checks(oracle):
    lat = Lattice((4, 4, 4, 4))
    lat.import_gauge(gen_gauge((4, 4, 4, 4), seed=164))
    D = DiracOpWilson(lat, mass=0.1)
    x = np.ones(D.f_size)
    k, tr = D.BiCGstab(x, np.zeros(D.f_size), n=2)
    assert k == 0 and tr == 0.0 and not x.any()
    with pytest.raises(A.CpsGpuError):
        D.BiCGstab(x, np.ones(D.f_size), n=11)  # n_max = 10 (bicgstab.C:67-70)
    k, tr = D.BiCGstab(x, gen_gaussian(D.f_size, seed=165), n=2, stop_rsd=1e-14, max_num_iter=4)
    assert k == 5 and tr == 0.0


@pytest.mark.parametrize("kind,L,ls,degree", [("wilson", (4, 4, 4, 8), 1, 4), ("dwf", (4, 4, 4, 8), 8, 3),
                                              ("mobius", (4, 4, 4, 4), 8, 2), ("dwf", (4, 4, 4, 4), 4, 0)])
def test_minresext_matches_oracle(oracle, kind, L, ls, degree):
    """DiracOp::MinResExt (minresext.C:30-150) against the oracle: the same
    guess, the same orthonormalised basis and A v, the same residual."""
    mass = 0.1
    u = gen_gauge(L, seed=171)
    lat = Lattice(L)
    lat.import_gauge(u)
    if kind == "wilson":
        D = DiracOpWilson(lat, mass=mass)
    elif kind == "dwf":
        D = DiracOpDwf(lat, mass=mass, ls=ls)
    else:
        D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
    ops = OracleOps(oracle, L, u, ls=ls, b=1.5, c=0.5)
    phi = gen_gaussian(D.f_size, seed=172)
    basis = [gen_gaussian(D.f_size, seed=173 + k) for k in range(degree)]
    po, vo, vmo, eo = ops.minresext(kind, phi, basis, mass=mass, kappa=D.kappa)
    psi = np.ones(D.f_size)
    v = [b.copy() for b in basis]
    vm = [np.zeros(D.f_size) for _ in basis]
    err = D.MinResExt(psi, phi, v, vm)
    if degree == 0:
        assert not psi.any()
        return
    assert rel(psi, po) < 1e-11 and abs(err - eo) < 1e-11 * eo
    for k in range(degree):
        assert rel(v[k], vo[k]) < 1e-12 and rel(vm[k], vmo[k]) < 1e-12


def test_fmatevl_wrappers(oracle):
    """FmatEvlInv / FmatEvlMInv (f_dwf_base.C:189-275): the Lattice-level
    entries the HMC calls, over InvCg and MInvCG."""
    L, ls, mass = (4, 4, 4, 8), 8, 0.1
    u = gen_gauge(L, seed=181)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls)
    b = gen_gaussian(D.f_size, seed=182)
    x = np.zeros(D.f_size)
    it, tr = D.FmatEvlInv(x, b, stop_rsd=1e-11)
    xo, ito, _ = ops.invcg("dwf", b, mass=mass, stop_rsd=1e-11)
    assert abs(it - ito) <= 1 and tr <= 1e-11 and rel(x, xo) < 1e-9
    shifts = [0.0, 0.05, 0.5]
    outs = [np.zeros(D.f_size) for _ in shifts]
    k, rs = D.FmatEvlMInv(outs, b, shifts, [1e-10] * 3)
    for s_, o in zip(shifts, outs):
        y, _ = ops.dwf_mdagm(o, mass)
        assert rel(y + s_ * o, b) < 1e-9
    assert k > 1 and len(rs) == 3


def _ritz_match(V, M, Vo, Mo):
    """Ritz values equal after sorting, Ritz vectors equal up to sign"""
    r = int(np.count_nonzero(Mo))
    oi, gi = np.argsort(Mo[:r]), np.argsort(M[:r])
    assert np.allclose(M[:r][gi], Mo[:r][oi], rtol=1e-8, atol=0)
    for a, b in zip(gi, oi):
        c = abs(np.dot(V[a], Vo[b])) / (np.linalg.norm(V[a]) * np.linalg.norm(Vo[b]))
        assert abs(c - 1.0) < 1e-6


@pytest.mark.parametrize("kind,L,ls,nev,m", [("wilson", (4, 4, 4, 8), 1, 4, 24), ("dwf", (4, 4, 4, 4), 4, 3, 16)])
def test_inveigcg_matches_oracle(oracle, kind, L, ls, nev, m):
    """DiracOp::InvEigCg (inv_eig_cg.C:129-635) against the oracle: the same
    CG (iterations, solution, true residual) and the same Ritz pairs."""
    mass = 0.1
    u = gen_gauge(L, seed=191)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpWilson(lat, mass=0.02) if kind == "wilson" else DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls)
    src = gen_gaussian(D.f_size, seed=192)
    so, ito, tro, Vo, Mo = ops.inveigcg(kind, src, nev, m, mass=mass, kappa=D.kappa, stop_rsd=1e-11)
    sol = np.ones(D.f_size)
    it, tr, V, M = D.InvEigCg(sol, src, nev=nev, m=m, stop_rsd=1e-11)
    assert abs(it - ito) <= 1 and tr < 1e-11 and rel(sol, so) < 1e-10
    _ritz_match(V, M, Vo, Mo[:2 * nev])
    # low-mode deflation with the Ritz vectors as FP32 U and invH = (U^dag A U)^-1
    U = [np.asarray(v, dtype=np.float32) for v in Vo[:nev]]
    Ud = [x.astype(np.float64) for x in U]
    AU = [ops.wilson_mdagm(x, D.kappa)[0] if kind == "wilson" else ops.dwf_mdagm(x, mass)[0] for x in Ud]
    cplx = lambda x: x[0::2] + 1j * x[1::2]
    Hm = np.array([[np.vdot(cplx(a), cplx(b)) for b in AU] for a in Ud])
    invH = np.linalg.inv(Hm)
    so2, ito2, _, _, _ = ops.inveigcg(kind, src, 0, 0, mass=mass, kappa=D.kappa, stop_rsd=1e-11, U=Ud, invH=invH,
                                      restart=[1e-4])
    sol2 = np.zeros(D.f_size)
    it2, tr2, _, _ = D.InvEigCg(sol2, src, stop_rsd=1e-11, U=U, invH=invH, restart=[1e-4])
    assert abs(it2 - ito2) <= 1 and tr2 < 1e-11 and rel(sol2, so2) < 1e-10


def test_inveigcg_argument_checks(oracle):
    L = (4, 4, 4, 4)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=193))
    D = DiracOpWilson(lat, mass=0.1)
    with pytest.raises(A.CpsGpuError):
        D.InvEigCg(np.zeros(D.f_size), np.ones(D.f_size), nev=4, m=8)  # m must exceed 2 nev


@pytest.mark.parametrize("kind,L,ls", [("wilson", (4, 4, 4, 4), 1), ("dwf", (4, 4, 2, 4), 4)])
def test_ritz_matches_oracle(oracle, kind, L, ls):
    """DiracOp::Ritz (ritz.C:152-532) against the oracle: the two lowest
    eigenpairs in turn, the same iteration counts, eigenvalues and vectors."""
    mass = 0.1
    u = gen_gauge(L, seed=201)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpWilson(lat, mass=0.02) if kind == "wilson" else DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls)
    go, gg = [], []
    for ne in range(2):
        x = gen_gaussian(D.f_size, seed=202 + ne)
        go.append(x.copy())
        gg.append(x.copy())
        ko, lo = ops.ritz(kind, go, mass=mass, kappa=D.kappa, RsdR_r=1e-8, Rsdlam=1e-11)
        k, lam = D.Ritz(gg, RsdR_r=1e-8, Rsdlam=1e-11)
        assert abs(k - ko) <= 1 and abs(lam - lo) < 1e-11 * lo
        assert rel(gg[-1], go[-1]) < 1e-7


@pytest.mark.parametrize("kind,L,ls,nvec,neg", [("dwf", (4, 4, 2, 4), 4, 4, False), ("wilson", (2, 2, 2, 4), 1, 3, True)])
def test_ritz_eig_and_jacobi_match_oracle(oracle, kind, L, ls, nvec, neg):
    """DiracOpWilsonTypes::RitzEig (eigen_wilson.C:89-586: Kalkreuter-Simma
    sweeps and the projection stage) and DiracOp::Jacobi (jacobi.C:48-268)
    against the oracle: the same iteration count, eigenvalues and valid
    flags, the same eigenvectors up to a phase."""
    mass = 0.1
    u = gen_gauge(L, seed=211)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpWilson(lat, mass=0.02) if kind == "wilson" else DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls)
    start = [gen_gaussian(D.f_size, seed=212 + k) for k in range(nvec)]
    po = [x.copy() for x in start]
    ro, lo, vo = ops.ritz_eig(kind, po, mass=mass, kappa=D.kappa, neg=neg)
    pg = [x.copy() for x in start]
    rg, lg, vg = D.RitzEig(pg, neg=neg)
    assert ro > 0 and abs(rg - ro) <= 4 and np.allclose(lg, lo, rtol=1e-9, atol=0)
    assert vg.tolist() == vo.tolist()
    cplx = lambda x: x[0::2] + 1j * x[1::2]
    for a, b in zip(pg, po):
        assert abs(abs(np.vdot(cplx(a), cplx(b))) - 1.0) < 1e-6
    if neg or nvec % 2:
        return
    mixed = mix_pairs(po, 7)
    AM = [ops.dwf_mdagm(x, mass)[0] for x in mixed]
    lam = np.array([np.vdot(cplx(x), cplx(y)).real for x, y in zip(mixed, AM)])
    off = np.array([np.vdot(cplx(mixed[i]), cplx(AM[j])) for j in range(1, 4) for i in range(j)])
    mg, lamg, offg = [x.copy() for x in mixed], lam.copy(), off.copy()
    kg = D.Jacobi(mg, lamg, offg)
    pv = (C.POINTER(C.c_double) * 4)(*[p(x) for x in mixed])
    ko = oracle.orc_jacobi(pv, ops.n, 4, p(lam), p(off.view(np.float64)), 1e-10, 50)
    assert kg == ko and np.allclose(lamg, lam, rtol=1e-12, atol=0)
    for a, b in zip(mg, mixed):
        assert rel(a, b) < 1e-12


@pytest.mark.parametrize("kind", ["dwf", "mobius"])
def test_imp_res_lanczos_matches_oracle(oracle, kind):
    """DiracOp::ImpResLanczos (lanczos.C:193-745, Chebyshev filter of
    d_op_dwf.C:852-960 / d_op_mobius.C:1279) against the oracle from the same
    float start vector: the same restart count, the nt lowest eigenvalues of
    MatPcDagMatPc (also against a dense diagonalisation), the same Ritz
    vectors up to a phase."""
    L, ls, mass = (2, 2, 2, 4), 4, 0.1
    u = gen_gauge(L, seed=41)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=mass, ls=ls) if kind == "dwf" else DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
    ops = OracleOps(oracle, L, u, ls=ls)
    n = ops.n
    mdagm = ops.dwf_mdagm if kind == "dwf" else ops.mobius_mdagm
    A_ = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        A_[:, k] = mdagm(e, mass)[0]
    ev = np.linalg.eigvalsh(A_[0::2, 0::2] + 1j * A_[1::2, 0::2])
    nk, nt, np_, Npol = 8, 4, 8, 6
    params = (np.sqrt(1.1 * ev[-1]), np.sqrt(ev[12]))
    v0 = gen_gaussian(n, seed=5).astype(np.float32)
    Vo = [np.zeros(n, dtype=np.float32) for _ in range(nk + np_)]
    Vo[0][:] = v0
    ao = np.zeros(nk + np_)
    pv = (C.POINTER(C.c_float) * len(Vo))(*[x.ctypes.data_as(C.POINTER(C.c_float)) for x in Vo])
    ito = oracle.orc_lanczos(ops._op(kind, mass, 0.0), None, 0, 0, n, pv, p(ao), nk, nt, np_, 100, 1e-5, 1, Npol,
                             params[0], params[1], 0.0)
    Vg = [np.zeros(n, dtype=np.float32) for _ in range(nk + np_)]
    Vg[0][:] = v0
    itg, ag = D.ImpResLanczos(Vg, nk, nt, np_, Npol, params, stop_residual=1e-5)
    assert 1 <= ito < 100 and abs(itg - ito) <= 1
    assert np.allclose(ag[:nt], ao[:nt], rtol=1e-7, atol=0) and np.allclose(ag[:nt], ev[:nt], rtol=1e-7, atol=0)
    cplx = lambda x: x[0::2].astype(np.float64) + 1j * x[1::2]
    for a, b in zip(Vg[:nt], Vo[:nt]):
        c = abs(np.vdot(cplx(a), cplx(b))) / (np.linalg.norm(a) * np.linalg.norm(b))
        assert abs(c - 1.0) < 1e-5


def test_imp_res_lanczos_argument_checks(oracle):
    L = (2, 2, 2, 4)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=42))
    W = DiracOpWilson(lat, mass=0.1)
    V = [np.zeros(W.f_size, dtype=np.float32) for _ in range(4)]
    with pytest.raises(A.CpsGpuError):  # DiracOp::RitzMat(V*,V*,MP*) is NotImplemented for Wilson
        W.ImpResLanczos(V, 2, 1, 2, 4, (2.0, 0.1))
    D = DiracOpDwf(lat, mass=0.1, ls=4)
    V = [np.ones(D.f_size, dtype=np.float32) for _ in range(4)]
    with pytest.raises(A.CpsGpuError):
        D.ImpResLanczos(V, 2, 1, 2, 1, (2.0, 0.1))  # Npol < 2
    with pytest.raises(A.CpsGpuError):
        D.ImpResLanczos(V, 2, 3, 2, 4, (2.0, 0.1))  # nt > nk


def _f32p(V):
    return (C.POINTER(C.c_float) * len(V))(*[x.ctypes.data_as(C.POINTER(C.c_float)) for x in V])


def test_inv_lowmode_approx_matches_oracle(oracle):
    """DiracOp::InvLowModeApprox (inv_lowmode_approx.C:272-512) from a device
    eigenvector cache against the oracle: 10 sources (two chunks of the
    dot-product kernel), float vectors, MATPCDAG_MATPC and MAT_HERM
    (squared eigenvalues); a missing cache is an error."""
    L, ls = (4, 4, 4, 4), 4
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=301))
    D = DiracOpDwf(lat, mass=0.1, ls=ls)
    rng = np.random.default_rng(302)
    neig, len_ = 12, 10
    V = [rng.normal(size=D.f_size).astype(np.float32) for _ in range(neig)]
    lam = rng.uniform(0.01, 1.0, size=neig)
    D.EigenCacheLoad("evecs", V, lam)
    src = [gen_gaussian(D.f_size, seed=303 + k) for k in range(len_)]
    for oper, sq in ((A.RITZ_MATPCDAG_MATPC, 0), (A.RITZ_MAT_HERM, 1)):
        out = [np.empty(D.f_size) for _ in range(len_)]
        D.InvLowModeApprox(out, src, "evecs", neig, ritz_mat_oper=oper)
        ref = [np.empty(D.f_size) for _ in range(len_)]
        oracle.orc_inv_lowmode_approx((C.POINTER(C.c_double) * len_)(*[p(x) for x in ref]),
                                      (C.POINTER(C.c_double) * len_)(*[p(x) for x in src]), len_, _f32p(V), p(lam),
                                      neig, D.f_size, sq)
        for a, b in zip(out, ref):
            assert rel(a, b) < 1e-12
    with pytest.raises(A.CpsGpuError):
        D.InvLowModeApprox([np.empty(D.f_size)], src[:1], "evecs", neig - 1)  # no cache of that size
    lat.eigencache_clear()
    with pytest.raises(A.CpsGpuError):
        D.InvLowModeApprox([np.empty(D.f_size)], src[:1], "evecs", neig)


def test_matinv_lowmode_inverters(oracle):
    """MatInv with Inverter LOWMODEAPPROX and CG_LOWMODE_DEFL
    (d_op_dwf.C:468-476): with every eigenvector of MatPcDagMatPc cached the
    low-mode approximation is the solve itself (to the FP32 storage of the
    vectors); with the 16 lowest as CG's initial guess the CG needs fewer
    iterations and reaches the plain CG's solution."""
    L, ls, mass = (2, 2, 2, 4), 2, 0.05
    u = gen_gauge(L, seed=311)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls)
    n = ops.n
    Am = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        Am[:, k] = ops.dwf_mdagm(e, mass)[0]
    w, U = np.linalg.eigh(Am[0::2, 0::2] + 1j * Am[1::2, 0::2])
    V = []
    for k in range(n // 2):
        r = np.empty(n, dtype=np.float32)
        r[0::2], r[1::2] = U[:, k].real, U[:, k].imag
        V.append(r)
    src = gen_gaussian(2 * D.f_size, seed=312)
    x_cg = np.zeros(2 * D.f_size)
    r_cg = D.MatInv(x_cg, src, stop_rsd=1e-11)
    D.EigenCacheLoad("all", V, w)
    x_lm = np.zeros(2 * D.f_size)
    r_lm = D.MatInv(x_lm, src, inverter=A.INV_LOWMODEAPPROX, fname_eigen="all", neig=len(V))
    assert r_lm.iterations == 0 and rel(x_lm, x_cg) < 1e-5
    D.EigenCacheLoad("low16", V[:16], w[:16])
    x_d = np.zeros(2 * D.f_size)
    r_d = D.MatInv(x_d, src, stop_rsd=1e-11, inverter=A.INV_CG_LOWMODE_DEFL, fname_eigen="low16", neig=16)
    assert r_d.status == A.CONVERGED and r_d.true_res < 1e-11
    assert r_d.iterations < r_cg.iterations and rel(x_d, x_cg) < 1e-9


def test_eigensolver_edge_cases(oracle):
    """Edge cases of the eigensolvers against the oracle: RitzEig without the
    Kalkreuter-Simma sweeps (successive Ritz calls, then the projection
    stage), Jacobi on one vector (no off-diagonal elements), and
    ImpResLanczos stopping on maxiters and with conv_check > 1."""
    L, ls, mass = (2, 2, 2, 4), 4, 0.1
    u = gen_gauge(L, seed=41)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls)
    n = ops.n
    start = [gen_gaussian(n, seed=400 + k) for k in range(3)]
    po, pg = [x.copy() for x in start], [x.copy() for x in start]
    ro, lo, vo = ops.ritz_eig("dwf", po, mass=mass, Kalk_Sim=0)
    rg, lg, vg = D.RitzEig(pg, Kalk_Sim=0)
    assert ro > 0 and abs(rg - ro) <= 3 and np.allclose(lg, lo, rtol=1e-9, atol=0) and vg.tolist() == vo.tolist()
    # one vector: Jacobi only sorts, zero sweeps of rotations
    one, lam = [start[0].copy()], np.array([0.5])
    assert D.Jacobi(one, lam, np.zeros(0, dtype=np.complex128)) == 0 and np.array_equal(one[0], start[0])
    # Lanczos: maxiters reached (the reference returns maxiters), and checks every other restart
    nk, nt, np_ = 6, 3, 6
    v0 = gen_gaussian(n, seed=401).astype(np.float32)
    for maxiters, conv_check, stop in ((2, 1, 1e-12), (40, 2, 1e-5)):
        Vo = [np.zeros(n, dtype=np.float32) for _ in range(nk + np_)]
        Vo[0][:] = v0
        ao = np.zeros(nk + np_)
        pv = (C.POINTER(C.c_float) * len(Vo))(*[x.ctypes.data_as(C.POINTER(C.c_float)) for x in Vo])
        ito = oracle.orc_lanczos(ops._op("dwf", mass, 0.0), None, 0, 0, n, pv, p(ao), nk, nt, np_, maxiters, stop,
                                 conv_check, 4, 1.4, 0.35, 0.0)
        Vg = [np.zeros(n, dtype=np.float32) for _ in range(nk + np_)]
        Vg[0][:] = v0
        itg, ag = D.ImpResLanczos(Vg, nk, nt, np_, 4, (1.4, 0.35), stop_residual=stop, maxiters=maxiters,
                                  conv_check=conv_check)
        if maxiters == 2:  # not converged: both stop on maxiters
            assert itg == ito == maxiters and np.allclose(ag[:nt], ao[:nt], rtol=1e-5, atol=0)
        else:  # converged, checked every conv_check restarts
            assert ito < maxiters and abs(itg - ito) <= conv_check
            assert np.allclose(ag[:nt], ao[:nt], rtol=1e-7, atol=0)


def test_lowmode_empty_cases(oracle):
    """InvLowModeApprox with no sources is a no-op; with a cache of zero
    vectors every output is zero (the reference zeroes them before its sum)."""
    L = (2, 2, 2, 4)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=410))
    D = DiracOpDwf(lat, mass=0.1, ls=2)
    D.EigenCacheLoad("none", [], np.zeros(0))
    D.InvLowModeApprox([], [], "none", 0)
    out = [np.ones(D.f_size)]
    D.InvLowModeApprox(out, [gen_gaussian(D.f_size, seed=411)], "none", 0)
    assert not out[0].any()
