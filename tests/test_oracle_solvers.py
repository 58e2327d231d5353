"""Oracle CG / multishift CG (restatements of inv_cg.C:84-448 and
minvcg.C:47-353): convergence, the reference's iteration bookkeeping, and
agreement of the multishift solutions with single-shift solves."""
import ctypes as C

import numpy as np
import pytest

from helpers import OracleOps, mix_pairs, rel, vh_of
from oracle.loader import p
from cps_veloc_b200.dirac import gen_gauge, gen_gaussian


@pytest.fixture(scope="module")
def wil(oracle):
    L = (4, 4, 4, 4)
    return OracleOps(oracle, L, gen_gauge(L, seed=21), ls=1)


def test_cg_converges_and_true_residual(wil):
    b = gen_gaussian(wil.n, seed=1)
    x, it, tr = wil.invcg("wilson", b, kappa=0.12, stop_rsd=1e-10)
    Ax, _ = wil.wilson_mdagm(x, 0.12)
    assert tr < 2e-10
    assert rel(Ax, b) == pytest.approx(tr, rel=1e-6)
    assert 2 < it < 200


def test_cg_iteration_bookkeeping(wil):
    b = gen_gaussian(wil.n, seed=2)
    # max_num_iter = 1: no iteration is run, InvCg returns itr + 1 = 1
    x, it, tr = wil.invcg("wilson", b, kappa=0.12, stop_rsd=1e-10, max_num_iter=1)
    assert it == 1 and np.all(x == 0) and tr == pytest.approx(1.0)
    # capped run: returns max_num_iter (max_itr = max_num_iter - 1 iterations, +1)
    x, it, tr = wil.invcg("wilson", b, kappa=0.12, stop_rsd=1e-14, max_num_iter=7)
    assert it == 7
    # already converged initial guess
    xs, _, _ = wil.invcg("wilson", b, kappa=0.12, stop_rsd=1e-12)
    x2, it2, tr2 = wil.invcg("wilson", b, sol0=xs, kappa=0.12, stop_rsd=1e-6)
    assert it2 == 1 and np.array_equal(x2, xs)


def test_cg_shift(wil):
    b = gen_gaussian(wil.n, seed=3)
    x, it, tr = wil.invcg("wilson", b, kappa=0.12, stop_rsd=1e-10, shift=0.5)
    Ax, _ = wil.wilson_mdagm(x, 0.12)
    assert rel(Ax + 0.5 * x, b) < 2e-10


@pytest.mark.parametrize("type_", [1, 0])
def test_minvcg_matches_single_shift(wil, type_):
    chi = gen_gaussian(wil.n, seed=4)
    shifts = [0.01, 0.1, 0.5, 2.0]
    alpha = [1.0, -0.5, 0.25, 2.0]
    psi, k, rs = wil.minvcg("wilson", chi, shifts, [1e-10] * 4, kappa=0.12, type=type_, alpha=alpha)
    sols = [wil.invcg("wilson", chi, kappa=0.12, stop_rsd=1e-12, shift=s)[0] for s in shifts]
    if type_ == 1:
        for s in range(4):
            assert rel(psi[s], sols[s]) < 1e-8
            # MInvCG reports |r_s| (absolute), having been given |r_s|/|chi| targets
            assert rs[s] / np.linalg.norm(chi) < 1e-10
    else:
        comb = sum(a * x for a, x in zip(alpha, sols))
        assert rel(psi[0], comb) < 1e-8
    assert k > 2


def test_dwf_cg(oracle):
    L = (4, 4, 2, 4)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=22), ls=4)
    b = gen_gaussian(ops.n, seed=5)
    x, it, tr = ops.invcg("dwf", b, mass=0.1, stop_rsd=1e-10)
    Ax, _ = ops.dwf_mdagm(x, 0.1)
    assert tr < 2e-10 and rel(Ax, b) < 2e-10


def test_mobius_cg(oracle):
    L = (4, 4, 2, 4)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=23), ls=4)
    b = gen_gaussian(ops.n, seed=6)
    x, it, tr = ops.invcg("mobius", b, mass=0.1, stop_rsd=1e-10)
    Ax, _ = ops.mobius_mdagm(x, 0.1)
    assert tr < 2e-10 and rel(Ax, b) < 2e-10


def _full_m(ops, kind, x, kappa, mass=0.0):
    """The unpreconditioned operator on [odd | even] halves: 1 - kappa Dslash"""
    n = ops.n
    xo, xe = x[:n], x[n:]
    if kind == "wilson":
        ho, he = ops.wilson_dslash(xe, 0, 0), ops.wilson_dslash(xo, 1, 0)
    else:
        ho, he = ops.dwf_dslash(xe, mass, 0, 0), ops.dwf_dslash(xo, mass, 1, 0)
    return np.concatenate([xo - kappa * ho, xe - kappa * he])


@pytest.mark.parametrize("kind", ["wilson", "dwf"])
def test_matinv_solves_the_full_operator(oracle, kind):
    """DiracOpWilson/Dwf::MatInv (d_op_wilson.C:257, d_op_dwf.C:316): the
    returned field solves the unpreconditioned system on both checkerboards."""
    L = (4, 4, 4, 4)
    ls = 1 if kind == "wilson" else 4
    ops = OracleOps(oracle, L, gen_gauge(L, seed=31), ls=ls)
    b = gen_gaussian(2 * ops.n, seed=32)
    kappa = 0.12 if kind == "wilson" else 1 / (2 * (5 - 1.8))
    x, it, tr = ops.matinv(kind, b, mass=0.1, kappa=kappa, stop_rsd=1e-12)
    assert tr < 1e-11 and it > 2
    assert rel(_full_m(ops, kind, x, kappa, mass=0.1), b) < 1e-9


def test_mobius_m5_and_m5inv_are_inverse(oracle):
    L = (4, 4, 2, 4)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=33), ls=6, b=1.5, c=0.5)
    x = gen_gaussian(ops.n, seed=34)
    assert rel(ops.mobius_m5inv(ops.mobius_m5(x, 0.05), 0.05, 0), x) < 1e-13


def test_mobius_matinv_converges(oracle):
    L = (4, 4, 2, 4)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=35), ls=6, b=1.5, c=0.5)
    b = gen_gaussian(2 * ops.n, seed=36)
    x, it, tr = ops.matinv("mobius", b, mass=0.05, stop_rsd=1e-12)
    assert tr < 1e-11 and it > 2 and np.all(np.isfinite(x))


@pytest.mark.parametrize("n", [1, 2, 4])
@pytest.mark.parametrize("kind", ["wilson", "dwf", "mobius"])
def test_bicgstab_solves_matpc(oracle, kind, n):
    """DiracOpWilsonTypes::BiCGstab (bicgstab.C:35-229) on MatPc itself: the
    reported |r| is the true residual of the returned psi, below stop_rsd |chi|,
    and k advances in steps of n from 1."""
    L = (4, 4, 2, 4)
    ls = 1 if kind == "wilson" else 4
    ops = OracleOps(oracle, L, gen_gauge(L, seed=41), ls=ls)
    chi = gen_gaussian(ops.n, seed=42 + n)
    stop = 1e-10
    psi, k, tr = ops.bicgstab(kind, chi, n=n, mass=0.1, kappa=0.12, stop_rsd=stop)
    if kind == "wilson":
        r = chi - ops.wilson_m(psi, 0.12, 0)
    elif kind == "dwf":
        r = chi - ops.dwf_m(psi, 0.1, 0)
    else:
        r = chi - ops.mobius_m(psi, 0.1, 0)
    nc = np.linalg.norm(chi)
    assert (k - 1) % n == 0 and k > 1
    assert 0 < tr < stop * nc
    # the recursed residual tracks the true one to rounding
    assert abs(np.linalg.norm(r) - tr) < 1e-3 * tr + 1e-13 * nc


def test_bicgstab_zero_source_and_no_convergence(oracle):
    L = (4, 4, 2, 4)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=43), ls=1)
    psi, k, tr = ops.bicgstab("wilson", np.zeros(ops.n), psi0=np.ones(ops.n), kappa=0.12)
    assert k == 0 and not psi.any() and tr == 0.0
    chi = gen_gaussian(ops.n, seed=44)
    psi, k, tr = ops.bicgstab("wilson", chi, n=2, kappa=0.12, stop_rsd=1e-14, max_num_iter=4)
    assert k == 5 and tr == 0.0  # two sweeps of n = 2, true_res untouched


@pytest.mark.parametrize("kind", ["wilson", "dwf"])
def test_minresext_properties(oracle, kind):
    """DiracOp::MinResExt (minresext.C): the basis comes back orthonormal,
    vm[i] = A v[i], and a basis holding the exact solution gives it back."""
    L = (4, 4, 2, 4)
    ls = 1 if kind == "wilson" else 4
    ops = OracleOps(oracle, L, gen_gauge(L, seed=51), ls=ls)
    phi = gen_gaussian(ops.n, seed=52)
    x, _, _ = ops.invcg(kind, phi, mass=0.1, kappa=0.12, stop_rsd=1e-13)
    basis = [gen_gaussian(ops.n, seed=53), 3.0 * x + 0.1 * gen_gaussian(ops.n, seed=54), x]
    psi, v, vm, err = ops.minresext(kind, phi, basis, mass=0.1, kappa=0.12)
    assert rel(psi, x) < 1e-10 and err < 1e-10
    for i in range(3):
        for j in range(3):
            d = np.dot(v[i], v[j])  # real part of the complex inner product
            assert abs(d - (i == j)) < 1e-12
    y, _ = (ops.wilson_mdagm(v[1], 0.12) if kind == "wilson" else ops.dwf_mdagm(v[1], 0.1))
    assert rel(vm[1], y) < 1e-14
    psi0, _, _, e0 = ops.minresext(kind, phi, [], mass=0.1, kappa=0.12)
    assert not psi0.any()


def _dense_mdagm(ops, kappa):
    """MatPcDagMatPc of a tiny Wilson lattice as a dense real matrix"""
    A = np.zeros((ops.n, ops.n))
    for k in range(ops.n):
        e = np.zeros(ops.n)
        e[k] = 1.0
        A[:, k] = ops.wilson_mdagm(e, kappa)[0]
    return 0.5 * (A + A.T)


def test_inveigcg_cg_unchanged_and_ritz_pairs(oracle):
    """DiracOp::InvEigCg (inv_eig_cg.C): the eigCG bookkeeping leaves the CG
    iterates untouched (same iterations, same solution), the first 2 nev of V
    are orthonormal Ritz vectors with M their Rayleigh quotients, and the
    lowest Ritz value approaches the lowest eigenvalue of MatPcDagMatPc."""
    L, kappa = (2, 2, 2, 4), 0.1245
    ops = OracleOps(oracle, L, gen_gauge(L, seed=61), ls=1)
    A = _dense_mdagm(ops, kappa)
    ev = np.linalg.eigvalsh(A)
    src = gen_gaussian(ops.n, seed=62)
    s0, it0, tr0, _, _ = ops.inveigcg("wilson", src, 0, 0, kappa=kappa, stop_rsd=1e-12)
    s1, it1, tr1, V, M = ops.inveigcg("wilson", src, 4, 20, kappa=kappa, stop_rsd=1e-12)
    assert it0 == it1 and np.array_equal(s0, s1) and tr1 < 1e-12
    xo, _, _ = ops.invcg("wilson", src, kappa=kappa, stop_rsd=1e-12)
    assert rel(s1, xo) < 1e-9
    rank = int(np.count_nonzero(M))
    assert rank >= 4
    W = np.array(V[:rank])
    assert np.allclose(W @ W.T, np.eye(rank), atol=1e-8)  # CG residuals stay orthogonal to rounding
    for j in range(rank):
        assert abs(W[j] @ A @ W[j] - M[j]) < 1e-9 * ev[-1]
    assert abs(np.min(M[:rank]) - ev[0]) < 1e-3 * ev[0]


def test_inveigcg_deflation(oracle):
    """Low-mode deflation: with U the Ritz vectors of a previous eigCG solve
    (FP32, as the reference stores them) and invH = (U^dag A U)^-1, the
    deflated solve starts from U invH U^dag src, restarts deflated at the
    given residual, and converges to the same solution in fewer iterations."""
    L, kappa = (2, 2, 2, 4), 0.1245
    ops = OracleOps(oracle, L, gen_gauge(L, seed=63), ls=1)
    src = gen_gaussian(ops.n, seed=64)
    s0, it0, _, V, M = ops.inveigcg("wilson", src, 4, 20, kappa=kappa, stop_rsd=1e-12)
    U = [np.asarray(v, dtype=np.float32).astype(np.float64) for v in V[:6]]
    Uc = [u[0::2] + 1j * u[1::2] for u in U]
    AU = [ops.wilson_mdagm(u, kappa)[0] for u in U]
    AUc = [a[0::2] + 1j * a[1::2] for a in AU]
    Hm = np.array([[np.vdot(Uc[i], AUc[j]) for j in range(6)] for i in range(6)])
    s1, it1, tr1, _, _ = ops.inveigcg("wilson", src, 0, 0, kappa=kappa, stop_rsd=1e-12, U=U,
                                      invH=np.linalg.inv(Hm), restart=[1e-5])
    assert tr1 < 1e-12 and rel(s1, s0) < 1e-9 and it1 < it0


def test_ritz_finds_the_lowest_eigenpairs(oracle):
    """DiracOp::Ritz (ritz.C:152-532): successive calls, each orthogonal to
    the eigenvectors already found, give the lowest eigenvalues of
    MatPcDagMatPc in order (checked against a dense diagonalisation of the
    complex operator); NEG_MATPCDAG_MATPC gives minus the largest."""
    L, kappa = (2, 2, 2, 4), 0.1245
    ops = OracleOps(oracle, L, gen_gauge(L, seed=61), ls=1)
    A = _dense_mdagm(ops, kappa)
    Ac = A[0::2, 0::2] + 1j * A[1::2, 0::2]
    ev = np.linalg.eigvalsh(Ac)
    psis = []
    for ne in range(3):
        psis.append(gen_gaussian(ops.n, seed=70 + ne))
        k, lam = ops.ritz("wilson", psis, kappa=kappa, RsdR_a=1e-10, RsdR_r=1e-9, Rsdlam=1e-12)
        v = psis[-1][0::2] + 1j * psis[-1][1::2]
        assert k > 0 and abs(lam - ev[ne]) < 1e-12 * ev[-1]
        assert np.linalg.norm(Ac @ v - lam * v) < 2e-9 * lam and abs(np.linalg.norm(v) - 1) < 1e-12
    k, lam = ops.ritz("wilson", [gen_gaussian(ops.n, seed=80)], kappa=kappa, neg=True, RsdR_r=1e-9,
                      Rsdlam=1e-12)
    assert abs(lam + ev[-1]) < 1e-12 * ev[-1]


def test_ritz_eig_kalkreuter_simma_and_jacobi(oracle):
    """DiracOpWilsonTypes::RitzEig (eigen_wilson.C:89-586): the four lowest
    eigenvalues of MatPcDagMatPc and orthonormal eigenvectors, through the
    Kalkreuter-Simma sweeps (in fewer Ritz iterations than four successive
    Ritz calls) and the projection stage; and DiracOp::Jacobi (jacobi.C)
    undoing a unitary mixing of eigenvector pairs."""
    L, kappa = (2, 2, 2, 4), 0.1245
    ops = OracleOps(oracle, L, gen_gauge(L, seed=61), ls=1)
    A = _dense_mdagm(ops, kappa)
    Ac = A[0::2, 0::2] + 1j * A[1::2, 0::2]
    ev = np.linalg.eigvalsh(Ac)
    psi = [gen_gaussian(ops.n, seed=90 + k) for k in range(4)]
    r, lh, valid = ops.ritz_eig("wilson", psi, kappa=kappa)
    assert r > 0 and np.allclose(lh[:4], ev[:4], rtol=1e-8, atol=0) and np.allclose(lh[4:], ev[:4], rtol=1e-8, atol=0)
    assert valid.tolist() == [1, 1, 1, 1]
    W = np.array([x[0::2] + 1j * x[1::2] for x in psi])
    assert np.allclose(W.conj() @ W.T, np.eye(4), atol=1e-12)
    for w, l in zip(W, lh[:4]):
        assert np.linalg.norm(Ac @ w - l * w) < 1e-4 * l
    plain = [gen_gaussian(ops.n, seed=90 + k) for k in range(4)]
    r0, lam0, _ = ops.ritz_eig("wilson", plain, kappa=kappa, Kalk_Sim=0, Rsdlam=1e-12, RsdR_r=1e-10)
    assert np.allclose(lam0[:4], ev[:4], rtol=1e-10, atol=0) and r < r0
    # RitzMatOper NEG_MATPCDAG_MATPC: the three largest, negated, sorted by |lambda|
    top = [gen_gaussian(ops.n, seed=95 + k) for k in range(3)]
    rn, ln, _ = ops.ritz_eig("wilson", top, kappa=kappa, neg=True)
    assert rn > 0 and np.allclose(ln[:3], -ev[-3:], rtol=1e-8, atol=0)
    lam = lh[:4]
    # Jacobi on a mixed basis
    mixed = mix_pairs(psi, 5)
    Mc = [x[0::2] + 1j * x[1::2] for x in mixed]
    lj = np.array([np.vdot(m, Ac @ m).real for m in Mc])
    off = np.array([np.vdot(Mc[i], Ac @ Mc[j]) for j in range(1, 4) for i in range(j)])
    pv = (C.POINTER(C.c_double) * 4)(*[p(x) for x in mixed])
    k = oracle.orc_jacobi(pv, ops.n, 4, p(lj), p(off.view(np.float64)), 1e-10, 50)
    assert k >= 1 and np.allclose(lj, lam, rtol=1e-12, atol=0) and np.abs(off).max() < 1e-10 * lam.max()
    for x, v in zip(mixed, psi):
        xc, vc = x[0::2] + 1j * x[1::2], v[0::2] + 1j * v[1::2]
        assert abs(abs(np.vdot(vc, xc)) - 1.0) < 1e-6


def _f32_ptrs(V):
    return (C.POINTER(C.c_float) * len(V))(*[x.ctypes.data_as(C.POINTER(C.c_float)) for x in V])


@pytest.mark.parametrize("Npol", [2, 6])
def test_lanczos_lowest_eigenpairs(oracle, Npol):
    """DiracOp::ImpResLanczos (lanczos.C:193-745) with the Chebyshev filter of
    DiracOpDwf::RitzMat (d_op_dwf.C:852-960) on DWF MatPcDagMatPc: the nt
    lowest eigenvalues against a dense diagonalisation, the Ritz vectors
    (float) orthonormal and eigenvectors to the stopping residual."""
    L, ls, mass = (2, 2, 2, 4), 4, 0.1
    ops = OracleOps(oracle, L, gen_gauge(L, seed=41), ls=ls)
    n = ops.n
    A = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        A[:, k] = ops.dwf_mdagm(e, mass)[0]
    Ac = A[0::2, 0::2] + 1j * A[1::2, 0::2]
    ev = np.linalg.eigvalsh(Ac)
    nk, nt, np_ = 8, 4, 8
    V = [np.zeros(n, dtype=np.float32) for _ in range(nk + np_)]
    V[0][:] = gen_gaussian(n, seed=5)
    alpha = np.zeros(nk + np_)
    it = oracle.orc_lanczos(ops._op("dwf", mass, 0.0), None, 0, 0, n, _f32_ptrs(V), p(alpha), nk, nt, np_, 100, 1e-5,
                            1, Npol, np.sqrt(ev[-1] * 1.1), np.sqrt(ev[12]), 0.0)
    assert 1 <= it < 100
    assert np.allclose(alpha[:nt], ev[:nt], rtol=1e-7, atol=0)
    W = np.array([x[0::2].astype(np.float64) + 1j * x[1::2] for x in V[:nt]])
    assert np.allclose(W.conj() @ W.T, np.eye(nt), atol=1e-5)
    for w, lam in zip(W, alpha[:nt]):
        assert np.linalg.norm(Ac @ w - lam * w) < 2e-5


@pytest.mark.parametrize("square", [0, 1])
def test_inv_lowmode_approx(oracle, square):
    """DiracOp::InvLowModeApprox (inv_lowmode_approx.C:272-512) against numpy:
    out_i = sum_k <v_k, in_i> / lambda_k v_k (lambda_k^2 for MAT_HERM), and
    with a complete eigenbasis of a hermitian matrix it is its inverse."""
    rng = np.random.default_rng(7)
    n, neig, len_ = 48, 6, 3
    V = [rng.normal(size=n).astype(np.float32) for _ in range(neig)]
    lam = rng.uniform(0.5, 2.0, size=neig)
    src = [rng.normal(size=n) for _ in range(len_)]
    out = [np.empty(n) for _ in range(len_)]
    po = (C.POINTER(C.c_double) * len_)(*[p(x) for x in out])
    pi = (C.POINTER(C.c_double) * len_)(*[p(x) for x in src])
    oracle.orc_inv_lowmode_approx(po, pi, len_, _f32_ptrs(V), p(lam), neig, n, square)
    cplx = lambda x: x[0::2].astype(np.float64) + 1j * x[1::2]
    ev = lam ** 2 if square else lam
    for o, s in zip(out, src):
        ref = sum(np.vdot(cplx(v), cplx(s)) / e * cplx(v) for v, e in zip(V, ev))
        assert np.allclose(cplx(o), ref, rtol=1e-12, atol=1e-12)
    # complete orthonormal eigenbasis: the exact inverse (up to FP32 storage of the vectors)
    m = n // 2
    H = rng.normal(size=(m, m)) + 1j * rng.normal(size=(m, m))
    H = H @ H.conj().T + m * np.eye(m)
    w, U = np.linalg.eigh(H)
    Vb = []
    for k in range(m):
        r = np.empty(n, dtype=np.float32)
        r[0::2], r[1::2] = U[:, k].real, U[:, k].imag
        Vb.append(r)
    b = rng.normal(size=n)
    x = np.empty(n)
    oracle.orc_inv_lowmode_approx((C.POINTER(C.c_double) * 1)(p(x)), (C.POINTER(C.c_double) * 1)(p(b)), 1,
                                  _f32_ptrs(Vb), p(w), m, n, 0)
    assert np.linalg.norm(H @ cplx(x) - cplx(b)) < 1e-5 * np.linalg.norm(cplx(b))
