"""Oracle CG / multishift CG (restatements of inv_cg.C:84-448 and
minvcg.C:47-353): convergence, the reference's iteration bookkeeping, and
agreement of the multishift solutions with single-shift solves."""
import numpy as np
import pytest

from helpers import OracleOps, rel, vh_of
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
