"""The oracle restatement against the reference's own kernels, compiled from
the reference sources (oracle/Makefile, target ``ref``), on geometries and
parameters beyond the golden set: boundary-condition variants, a minimal
2^4 lattice, odd and even Ls, zero and large masses."""
import ctypes as C

import numpy as np
import pytest

from helpers import OracleOps, rel, vh_of
from oracle.loader import apply_bc_signs, p
from cps_veloc_b200.dirac import gen_gauge, gen_gaussian

TOL = 1e-13


def _ref_setup(R, L, ls, bc, m5=1.8, b=1.5, c=0.5):
    # the reference harness records only the t boundary; x,y,z stay periodic
    assert bc[0] == bc[1] == bc[2] == 1
    R.ref_init(*L, ls, m5, b, c, bc[3])


@pytest.mark.parametrize("L,bc", [((4, 4, 4, 4), (1, 1, 1, -1)), ((2, 2, 2, 2), (1, 1, 1, 1)),
                                  ((4, 2, 6, 4), (1, 1, 1, -1)), ((6, 4, 2, 8), (1, 1, 1, 1))])
def test_wilson_vs_reference(oracle, reference, L, bc):
    _ref_setup(reference, L, 2, bc)
    u = gen_gauge(L, seed=11)
    us = apply_bc_signs(u, L, bc)
    ops = OracleOps(oracle, L, u, ls=1, bc=bc)
    psi = gen_gaussian(24 * vh_of(L), seed=3)
    for cb in (0, 1):
        for dag in (0, 1):
            y = np.zeros_like(psi)
            reference.ref_wilson_dslash(p(y), p(us), p(psi), cb, dag)
            assert rel(ops.wilson_dslash(psi, cb, dag), y) < TOL
    for kappa in (0.12, 0.125):
        y = np.zeros_like(psi)
        d = C.c_double()
        reference.ref_wilson_mdagm(p(y), p(us), p(psi), C.byref(d), kappa)
        yo, do = ops.wilson_mdagm(psi, kappa)
        assert rel(yo, y) < TOL and abs(do / d.value - 1) < TOL


@pytest.mark.parametrize("L,ls,mass", [((4, 4, 4, 4), 4, 0.01), ((2, 4, 2, 4), 8, 0.1),
                                       ((4, 2, 2, 8), 5, 0.0), ((2, 2, 4, 4), 2, 1.0)])
def test_dwf_vs_reference(oracle, reference, L, ls, mass):
    bc = (1, 1, 1, -1)
    _ref_setup(reference, L, ls, bc)
    u = gen_gauge(L, seed=5)
    us = apply_bc_signs(u, L, bc)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc)
    psi = gen_gaussian(24 * ls * vh_of(L), seed=4)
    assert abs(reference.ref_dwf_kappa() - 1 / (2 * (5 - 1.8))) < 1e-15
    for cb in (0, 1):
        for dag in (0, 1):
            y = np.zeros_like(psi)
            reference.ref_dwf_dslash(p(y), p(us), p(psi), mass, cb, dag)
            assert rel(ops.dwf_dslash(psi, mass, cb, dag), y) < TOL
    for dag, fn in ((0, reference.ref_dwf_m), (1, reference.ref_dwf_mdag)):
        y = np.zeros_like(psi)
        fn(p(y), p(us), p(psi), mass)
        assert rel(ops.dwf_m(psi, mass, dag), y) < TOL
    y = np.zeros_like(psi)
    d = C.c_double()
    reference.ref_dwf_mdagm(p(y), p(us), p(psi), C.byref(d), mass)
    yo, do = ops.dwf_mdagm(psi, mass)
    assert rel(yo, y) < TOL and abs(do / d.value - 1) < TOL


@pytest.mark.parametrize("L,ls,mass,b,c", [((4, 4, 4, 4), 4, 0.01, 1.5, 0.5), ((2, 4, 2, 4), 6, 0.1, 1.5, 0.5),
                                           ((4, 2, 2, 4), 5, 0.005, 2.0, 1.0), ((2, 2, 4, 4), 8, 0.3, 1.0, 0.0)])
def test_mobius_vs_reference(oracle, reference, L, ls, mass, b, c):
    bc = (1, 1, 1, -1)
    _ref_setup(reference, L, ls, bc, b=b, c=c)
    u = gen_gauge(L, seed=9)
    us = apply_bc_signs(u, L, bc)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc, b=b, c=c)
    psi = gen_gaussian(24 * ls * vh_of(L), seed=8)
    for dag in (0, 1):
        y = psi.copy()
        reference.ref_zmobius_m5inv(p(y), mass, dag)
        assert rel(ops.mobius_m5inv(psi, mass, dag), y) < TOL
    # M5 = 1 + K D5 (zmobius_kappa_dslash_5_plus_cmplx accumulates into its output)
    y = psi.copy()
    reference.ref_zmobius_kappa_dslash_5_plus(p(y), p(psi), mass, 0)
    assert rel(ops.mobius_m5(psi, mass), y) < TOL
    for cb in (0, 1):
        for dag in (0, 1):
            y = np.zeros_like(psi)
            reference.ref_zmobius_dslash_4(p(y), p(us), p(psi), cb, dag, mass)
            assert rel(ops.mobius_dslash_4(psi, mass, cb, dag), y) < TOL
    for dag, fn in ((0, reference.ref_zmobius_m), (1, reference.ref_zmobius_mdag)):
        y = np.zeros_like(psi)
        fn(p(y), p(us), p(psi), mass)
        assert rel(ops.mobius_m(psi, mass, dag), y) < TOL
    y = np.zeros_like(psi)
    d = C.c_double()
    reference.ref_zmobius_mdagm(p(y), p(us), p(psi), C.byref(d), mass)
    yo, do = ops.mobius_mdagm(psi, mass)
    assert rel(yo, y) < TOL and abs(do / d.value - 1) < TOL


def zmobius_coefficients(ls):
    """complex b_s, c_s (b_s - c_s = 1) of the kind zMobius approximations use"""
    b = np.array([1.5 + 0.25j * np.sin(1.0 + s) for s in range(ls)])
    return b, b - 1.0


@pytest.mark.parametrize("L,ls,mass", [((4, 4, 2, 4), 6, 0.05), ((2, 2, 4, 4), 5, 0.1)])
def test_zmobius_vs_reference(oracle, reference, L, ls, mass):
    """Complex per-slice coefficients (DiracOpZMobius) through the same kernels"""
    bc = (1, 1, 1, -1)
    _ref_setup(reference, L, ls, bc, b=1.5, c=0.5)
    zb, zc = zmobius_coefficients(ls)
    reference.ref_set_zmobius(p(np.ascontiguousarray(zb.view(np.float64))), p(np.ascontiguousarray(zc.view(np.float64))))
    u = gen_gauge(L, seed=19)
    us = apply_bc_signs(u, L, bc)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc)
    ops.set_zmobius(zb, zc)
    psi = gen_gaussian(24 * ls * vh_of(L), seed=18)
    for dag in (0, 1):
        y = psi.copy()
        reference.ref_zmobius_m5inv(p(y), mass, dag)
        assert rel(ops.mobius_m5inv(psi, mass, dag), y) < TOL
        for cb in (0, 1):
            y = np.zeros_like(psi)
            reference.ref_zmobius_dslash_4(p(y), p(us), p(psi), cb, dag, mass)
            assert rel(ops.mobius_dslash_4(psi, mass, cb, dag), y) < TOL
    for dag, fn in ((0, reference.ref_zmobius_m), (1, reference.ref_zmobius_mdag)):
        y = np.zeros_like(psi)
        fn(p(y), p(us), p(psi), mass)
        assert rel(ops.mobius_m(psi, mass, dag), y) < TOL
    y = np.zeros_like(psi)
    d = C.c_double()
    reference.ref_zmobius_mdagm(p(y), p(us), p(psi), C.byref(d), mass)
    yo, do = ops.mobius_mdagm(psi, mass)
    assert rel(yo, y) < TOL and abs(do / d.value - 1) < TOL


@pytest.mark.parametrize("which", range(8))
@pytest.mark.parametrize("nblk,vs,ws", [(1, 0, 0), (3, 0, 0), (4, 24, 48)])
def test_sproj_tr_vs_reference(oracle, reference, which, nblk, vs, ws):
    """sprojTr{X,Y,Z,T}{m,p} (sproj_tr.C): the oracle's (1 -+ gamma_mu) spin
    projection and trace against the reference's eight routines, with blocks
    and strides as FdwfBase::EvolveMomFforce passes them."""
    v = gen_gaussian((24 + vs) * nblk, seed=170 + which)
    w = gen_gaussian((24 + ws) * nblk, seed=180 + which)
    f_ref, f_orc = np.zeros(18), np.zeros(18)
    reference.ref_sproj_tr(which, p(f_ref), p(v), p(w), nblk, vs, ws)
    oracle.orc_sproj_tr(which % 4, -1 if which < 4 else 1, p(f_orc), p(v), p(w), nblk, vs, ws)
    assert rel(f_orc, f_ref) < 1e-14


def test_force_matrix_steps_vs_reference(oracle, reference):
    """The per-link steps of the force loop (F = U T, TrLessAntiHermMatrix
    with F^dag, *= coeff, Matrix::norm) against the reference's Matrix class."""
    for k in range(5):
        U = gen_gaussian(18, seed=190 + k)
        T = gen_gaussian(18, seed=200 + k)
        fr, fo = np.zeros(18), np.zeros(18)
        nr, no = C.c_double(), C.c_double()
        reference.ref_force_matrix(p(fr), C.byref(nr), p(U), p(T), -0.37)
        oracle.orc_force_matrix(p(fo), C.byref(no), p(U), p(T), -0.37)
        assert rel(fo, fr) < 1e-14 and abs(no.value - nr.value) <= 1e-14 * abs(nr.value)
        # traceless and antihermitian
        m = fo[0::2].reshape(3, 3) + 1j * fo[1::2].reshape(3, 3)
        assert np.abs(m + m.conj().T).max() < 1e-15 and abs(np.trace(m)) < 1e-15


def _canonical_signed(u, L, bc):
    from cps_veloc_b200.dirac import StrOrd, gconvert
    us = apply_bc_signs(u, L, bc)
    gconvert(L, us, StrOrd.CANONICAL, StrOrd.WILSON)
    return us


def test_dwf_force_vs_reference_force_loop(oracle, reference):
    """The oracle's force loop (orc_fforce) against the reference's own
    FforceWilsonType::run (fforce_wilson_type.C) on the same DWF force
    vectors: FforceWilsonType takes v1 and v2 in the other roles, the
    signed links and coef = 2 dt."""
    from helpers import s_inner
    L, ls, mass, dt = (4, 4, 4, 4), 4, 0.1, 0.3
    bc = (1, 1, 1, -1)
    _ref_setup(reference, L, ls, bc)
    u = gen_gauge(L, seed=241)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc)
    chi = gen_gaussian(ops.n, seed=242)
    mo, fo = ops.fforce("dwf", chi, dt, mass=mass)
    v1, v2 = ops.force_vecs("dwf", chi, mass=mass)
    mom, out = np.zeros(4 * 256 * 18), np.zeros(3)
    reference.ref_fforce_wilson_type(p(mom), p(_canonical_signed(u, L, bc)), p(s_inner(v2, L, ls, "dwf")),
                                     p(s_inner(v1, L, ls, "dwf")), ls, 2 * dt, p(out))
    assert rel(mo, mom) < 1e-14 and np.allclose(fo, out, rtol=1e-13, atol=0)


@pytest.mark.parametrize("L,ls,mass,b,c", [((4, 4, 4, 4), 4, 0.1, 1.5, 0.5), ((4, 2, 2, 4), 6, 0.02, 2.0, 1.0)])
def test_mobius_force_vs_reference(oracle, reference, L, ls, mass, b, c):
    """Fmobius::EvolveMomFforce (f_mobius.C:847-887) composed from the
    reference's own kernels (mobius_m, mobius_m5inv, mobius_dslash_4, the
    two steps of mobius_Booee) and FforceWilsonType::run, against the
    oracle's restatement (OracleOps.mobius_fforce)."""
    from helpers import s_inner
    bc = (1, 1, 1, -1)
    _ref_setup(reference, L, ls, bc, b=b, c=c)
    u = gen_gauge(L, seed=243)
    us = apply_bc_signs(u, L, bc)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc, b=b, c=c)
    n = ops.n
    x = gen_gaussian(n, seed=244)
    y = np.zeros(n)
    reference.ref_mobius_booee(p(y), p(x), mass)
    assert rel(ops.mobius_booee(x, mass), y) < TOL
    frm, step = gen_gaussian(n, seed=245), 0.37

    def ref(fn, *a):
        out = np.zeros(n)
        fn(p(out), *a)
        return out

    phi1 = ref(reference.ref_mobius_m, p(us), p(frm), mass)
    phi2 = ref(reference.ref_mobius_m5inv, p(frm), mass, 0)
    tmp2 = ref(reference.ref_mobius_m5inv, p(ref(reference.ref_mobius_dslash_4, p(us), p(phi2), 1, 0, mass)), mass, 0)
    v2 = np.concatenate([ref(reference.ref_mobius_booee, p(tmp2), mass), ref(reference.ref_mobius_booee, p(phi2), mass)])
    tmp4 = ref(reference.ref_mobius_dslash_4, p(us), p(phi1), 1, 1, mass)
    v1 = np.concatenate([ref(reference.ref_mobius_m5inv, p(tmp4), mass, 1), phi1])
    mom, out = np.zeros(4 * int(np.prod(L)) * 18), np.zeros(3)
    reference.ref_fforce_wilson_type(p(mom), p(_canonical_signed(u, L, bc)), p(s_inner(v1, L, ls, "mobius")),
                                     p(s_inner(v2, L, ls, "mobius")), ls, -step, p(out))
    mo, fo = ops.mobius_fforce(frm, step, mass)
    assert rel(mo, mom) < 1e-13 and np.allclose(fo, out, rtol=1e-12, atol=0)


@pytest.mark.parametrize("n", [1, 2, 7, 24])
def test_dense_eigensolver_vs_reference(oracle, reference, n):
    """The oracle's Jacobi eigensolver against the reference's eigen_solver
    (eigen_solver.C:40, Householder tridiagonalisation + implicit QL) on a
    random symmetric matrix in the packed lower-triangle layout eigCG passes:
    the same eigenvalues.  The reference's vectors are not eigenvectors: its
    tqli has the eigenvector update commented out (eigen_solver.C:180-185), so
    Evec holds tred2's orthogonal transform; the test records that, and the
    library's eigCG uses true eigenvectors (Evec[k n + i] = component k of
    vector i)."""
    rng = np.random.default_rng(250 + n)
    a = rng.normal(size=(n, n))
    a = a + a.T
    packed = np.array([a[i, j] for i in range(n) for j in range(i + 1)])
    er, vr, eo, vo = np.zeros(n), np.zeros(n * n), np.zeros(n), np.zeros(n * n)
    reference.ref_eigen_solver(p(packed.copy()), p(vr), p(er), n)
    oracle.orc_sym_eigen(p(packed), p(vo), p(eo), n)
    scale = np.abs(er).max()
    assert np.allclose(np.sort(eo), np.sort(er), rtol=0, atol=1e-12 * scale)
    Vo, Vr = vo.reshape(n, n), vr.reshape(n, n)
    assert np.allclose(a @ Vo, Vo * eo, atol=1e-11 * scale)
    assert np.allclose(Vo.T @ Vo, np.eye(n), atol=1e-12)
    assert np.allclose(Vr.T @ Vr, np.eye(n), atol=1e-12)  # orthogonal ...
    if n > 1:
        assert np.abs(a @ Vr - Vr * er).max() > 1e-3 * scale  # ... but not the eigenvectors


@pytest.mark.parametrize("m,nk,np_", [(6, 6, 0), (12, 8, 4), (20, 12, 8)])
def test_lanczos_tridiagonal_helpers_vs_reference(oracle, reference, m, nk, np_):
    """The tridiagonal algebra of ImpResLanczos against the reference's own
    tqri, QRtrf and eigsrt (eigen_solver.C:206-305, 1442-1498), bit for bit:
    the QR eigenvalues of a leading block with the rotations accumulated,
    np exact-shift QR steps over the whole matrix, and both sorts."""
    rng = np.random.default_rng(700 + m)
    d0, e0 = rng.normal(size=m) + 3.0, np.abs(rng.normal(size=m)) + 0.1
    e0[-1] = 0.3
    out = []
    for lib, fn in ((reference, "ref"), (oracle, "orc")):
        d, e, Q = d0.copy(), e0.copy(), np.eye(m)
        it = lib.ref_tqri(p(d), p(e), nk, m, p(Q)) if fn == "ref" else lib.orc_tqri(p(d), p(e), nk, m, p(Q), m)
        dt, s1, Qs = d.copy(), d.copy(), Q.copy()
        if fn == "ref":
            lib.ref_eigsrt(p(s1), None, m)
            lib.ref_eigsrt(p(d), p(Qs), m)
        else:
            lib.orc_eigsrt(p(s1), None, m, m)
            lib.orc_eigsrt(p(d), p(Qs), m, m)
        a, b, Qr = d0.copy(), e0.copy(), np.eye(m)
        for k in range(np_):
            if fn == "ref":
                lib.ref_qrtrf(p(a), p(b), m, m, p(Qr), s1[nk + k] if nk + k < m else s1[-1], 0, m - 1)
            else:
                lib.orc_qrtrf(p(a), p(b), m, p(Qr), m, s1[nk + k] if nk + k < m else s1[-1], 0, m - 1)
        out.append((it, dt, s1, d, Qs, a, b, Qr))
    (ir, *vr), (io, *vo) = out
    assert ir == io
    for x, y in zip(vr, vo):
        assert np.array_equal(x, y)
    # the leading nk x nk block is diagonalised, its rotations in Q
    T = np.diag(d0[:nk]) + np.diag(e0[:nk - 1], 1) + np.diag(e0[:nk - 1], -1)
    dt, Q = vo[0], np.eye(m)
    oracle.orc_tqri(p(d0.copy()), p(e0.copy()), nk, m, p(Q), m)
    assert np.allclose(np.sort(dt[:nk]), np.linalg.eigvalsh(T), rtol=0, atol=1e-12 * np.abs(d0).max())
    Qk = Q[:nk, :nk]
    assert np.allclose(Qk.T @ T @ Qk, np.diag(dt[:nk]), atol=1e-11 * np.abs(d0).max())
