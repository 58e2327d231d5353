"""The oracle's HMC fermion force (Fwilson / FdwfBase::EvolveMomFforce)
checked as what it is: the negative gradient of the pseudofermion action.
With chi = (MatPc^dag MatPc)^-1 phi and S(U) = phi . chi, a variation
U_l -> exp(eps X_l) U_l (X traceless antihermitian) must change S at the rate
dS/deps = -sum_l <X_l, F_l> for the force F that EvolveMomFforce adds to the
momenta at dt = 1 (the normalisation under which the reference's leapfrog
conserves H = 1/2 <P, P> + S).  Its pieces are pinned to the reference's own
routines in test_oracle_reference.py.  CPU only."""
import numpy as np
import pytest
from scipy.linalg import expm

from helpers import OracleOps
from cps_veloc_b200.dirac import gen_gauge, gen_gaussian


def _gauge_sites(L):
    """WILSON-order gauge site of every lexicographic site"""
    lx, ly, lz, lt = L
    vh = lx * ly * lz * lt // 2
    t, z, y, x = np.meshgrid(*(np.arange(n) for n in (lt, lz, ly, lx)), indexing="ij")
    x, y, z, t = (a.ravel() for a in (x, y, z, t))
    return x // 2 + (lx // 2) * (y + ly * (z + lz * t)) + vh * ((x + y + z + t) & 1)


def _perturb(u, L, X, eps):
    """U_l -> exp(eps X_l) U_l on a WILSON-order field (element (row, col) at 2 (row + 3 col))"""
    u2 = u.copy().reshape(-1, 4, 3, 3, 2)
    gs = _gauge_sites(L)
    m = np.swapaxes(u2[gs, :, :, :, 0] + 1j * u2[gs, :, :, :, 1], -1, -2)  # [lex][mu][row][col]
    e = np.array([[expm(eps * X[a, mu]) for mu in range(4)] for a in range(X.shape[0])])
    mn = np.swapaxes(e @ m, -1, -2)
    u2[gs, :, :, :, 0], u2[gs, :, :, :, 1] = mn.real, mn.imag
    return u2.ravel()


def _random_su3_algebra(rng, n):
    a = rng.normal(size=(n, 4, 3, 3)) + 1j * rng.normal(size=(n, 4, 3, 3))
    a = 0.5 * (a - np.conj(np.swapaxes(a, -1, -2)))
    return a - (np.trace(a, axis1=-2, axis2=-1) / 3)[..., None, None] * np.eye(3)


@pytest.mark.parametrize("kind,ls,bc", [("wilson", 1, (1, 1, 1, -1)), ("wilson", 1, (-1, 1, 1, 1)),
                                        ("dwf", 4, (1, 1, 1, -1))])
def test_force_is_the_action_gradient(oracle, kind, ls, bc):
    L, mass, kappa = (4, 4, 4, 4), 0.1, 0.12
    vol = int(np.prod(L))
    u = gen_gauge(L, seed=211)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc)
    phi = gen_gaussian(ops.n, seed=212)
    chi, _, _ = ops.invcg(kind, phi, mass=mass, kappa=kappa, stop_rsd=1e-13)
    F, (l1, l2, linf) = ops.fforce(kind, chi, 1.0, mass=mass, kappa=kappa)
    Fm = (F[0::2] + 1j * F[1::2]).reshape(vol, 4, 3, 3)
    assert np.abs(Fm + np.conj(np.swapaxes(Fm, -1, -2))).max() < 1e-13  # antihermitian
    assert np.abs(np.trace(Fm, axis1=-2, axis2=-1)).max() < 1e-13      # traceless
    nrm = np.sqrt(2 * np.sum(np.abs(Fm) ** 2, axis=(-1, -2))).ravel()  # Matrix::norm = -2 tr F^2
    assert abs(l1 - nrm.mean()) < 1e-12 * l1 and abs(linf - nrm.max()) < 1e-12 * linf
    assert abs(l2 - np.sqrt(np.mean(nrm ** 2))) < 1e-12 * l2
    rng = np.random.default_rng(213)
    for _ in range(2):
        X = _random_su3_algebra(rng, vol)

        def S(eps):
            o2 = OracleOps(oracle, L, _perturb(u, L, X, eps), ls=ls, bc=bc)
            c2, _, _ = o2.invcg(kind, phi, mass=mass, kappa=kappa, stop_rsd=1e-13)
            return float(np.dot(c2, phi))

        eps = 1e-5
        dS = (S(eps) - S(-eps)) / (2 * eps)
        assert abs(dS + np.sum((np.conj(X) * Fm).real)) < 1e-7 * abs(dS)


def test_force_accumulates_and_scales_with_dt(oracle):
    L = (4, 4, 2, 4)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=214), ls=1)
    chi = gen_gaussian(ops.n, seed=215)
    m0 = gen_gaussian(4 * int(np.prod(L)) * 18, seed=216)
    f1, a1 = ops.fforce("wilson", chi, 1.0, kappa=0.12)
    f2, a2 = ops.fforce("wilson", chi, -0.25, kappa=0.12, mom=m0)
    assert np.allclose(f2 - m0, -0.25 * f1, rtol=0, atol=1e-14 * np.abs(f1).max())
    assert np.allclose(np.array(a2), 0.25 * np.array(a1), rtol=1e-13)
    fz, az = ops.fforce("wilson", np.zeros(ops.n), 1.0, kappa=0.12)
    assert not fz.any() and az == (0.0, 0.0, 0.0)


def test_mobius_force_normalisation(oracle):
    """Fmobius::EvolveMomFforce with SYM2 preconditioning: the force it adds is
    the gradient of S = phi . (MatPc^dag MatPc)^-1 phi up to the factor
    2 kappa_b^2, dS/deps = -2 kappa_b^2 sum <X, F>.  The reference applies
    coef *= 2 kappa_b^2 only for the ORIG and SYM1 preconditionings
    (f_mobius.C:818-823), and the library reproduces its SYM2 force as is."""
    L, ls, mass = (4, 4, 2, 4), 4, 0.1
    b, c, m5 = 1.5, 0.5, 1.8
    u = gen_gauge(L, seed=217)
    ops = OracleOps(oracle, L, u, ls=ls, b=b, c=c)
    phi = gen_gaussian(ops.n, seed=218)
    chi, _, _ = ops.invcg("mobius", phi, mass=mass, stop_rsd=1e-13)
    F, _ = ops.mobius_fforce(chi, 1.0, mass)
    Fm = (F[0::2] + 1j * F[1::2]).reshape(-1, 4, 3, 3)
    X = _random_su3_algebra(np.random.default_rng(219), Fm.shape[0])

    def S(eps):
        o2 = OracleOps(oracle, L, _perturb(u, L, X, eps), ls=ls, b=b, c=c)
        c2, _, _ = o2.invcg("mobius", phi, mass=mass, stop_rsd=1e-13)
        return float(np.dot(c2, phi))

    eps = 1e-5
    dS = (S(eps) - S(-eps)) / (2 * eps)
    kb = 1 / (2 * (b * (4 - m5) + 1))
    assert abs(dS + 2 * kb * kb * np.sum((np.conj(X) * Fm).real)) < 1e-7 * abs(dS)
