"""HMC fermion force on the GPU (cpsgpu_calc_hmd_force_vecs,
cpsgpu_evolve_mom_fforce) against the oracle's restatement of
DiracOp*::CalcHmdForceVecs and Fwilson / FdwfBase::EvolveMomFforce."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpMobius, DiracOpWilson, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel

pytestmark = pytest.mark.gpu

CASES = [("wilson", (4, 4, 4, 8), 1, (1, 1, 1, -1)), ("wilson", (8, 4, 6, 4), 1, (-1, 1, -1, -1)),
         ("dwf", (4, 4, 4, 8), 8, (1, 1, 1, -1)), ("dwf", (8, 8, 4, 4), 4, (1, -1, 1, 1))]


def _setup(oracle, kind, L, ls, bc, seed):
    u = gen_gauge(L, seed=seed)
    lat = Lattice(L, bc)
    lat.import_gauge(u)
    mass = 0.1
    D = DiracOpWilson(lat, mass=mass) if kind == "wilson" else DiracOpDwf(lat, mass=mass, ls=ls)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc)
    return D, ops, mass


@pytest.mark.parametrize("kind,L,ls,bc", CASES)
def test_calc_hmd_force_vecs(oracle, kind, L, ls, bc):
    D, ops, mass = _setup(oracle, kind, L, ls, bc, 221)
    chi = gen_gaussian(D.f_size, seed=222)
    f_out, f_in = D.CalcHmdForceVecs(chi)
    v1, v2 = ops.force_vecs(kind, chi, mass=mass, kappa=D.kappa)
    assert rel(f_out, v1) < 1e-14 and rel(f_in, v2) < 1e-13


@pytest.mark.parametrize("kind,L,ls,bc", CASES)
def test_evolve_mom_fforce_matches_oracle(oracle, kind, L, ls, bc):
    D, ops, mass = _setup(oracle, kind, L, ls, bc, 223)
    chi = gen_gaussian(D.f_size, seed=224)
    mom0 = gen_gaussian(4 * int(np.prod(L)) * 18, seed=225)
    dt = 0.0371
    mo, fo = ops.fforce(kind, chi, dt, mass=mass, kappa=D.kappa, mom=mom0)
    mom = mom0.copy()
    fg = D.EvolveMomFforce(mom, chi, dt)
    assert rel(mom - mom0, mo - mom0) < 1e-12
    assert np.allclose(fg, fo, rtol=1e-12, atol=0)
    # a second call accumulates
    D.EvolveMomFforce(mom, chi, dt)
    assert rel(mom - mom0, 2 * (mo - mom0)) < 1e-12


@pytest.mark.parametrize("L,ls,bc", [((4, 4, 4, 8), 8, (1, 1, 1, -1)), ((8, 4, 4, 4), 4, (-1, 1, 1, 1))])
def test_mobius_force_matches_oracle(oracle, L, ls, bc):
    """Fmobius::EvolveMomFforce (SYM2): the force vectors and the force."""
    u = gen_gauge(L, seed=232)
    lat = Lattice(L, bc)
    lat.import_gauge(u)
    mass = 0.05
    D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc, b=1.5, c=0.5)
    frm = gen_gaussian(D.f_size, seed=233)
    f_out, f_in = D.CalcHmdForceVecs(frm)
    v1, v2 = ops.mobius_force_vecs(ops.mobius_m(frm, mass, 0), frm, mass)
    assert rel(f_out, v1) < 1e-13 and rel(f_in, v2) < 1e-13
    mom0 = gen_gaussian(4 * int(np.prod(L)) * 18, seed=234)
    mo, fo = ops.mobius_fforce(frm, 0.21, mass, mom=mom0)
    mom = mom0.copy()
    fg = D.EvolveMomFforce(mom, frm, 0.21)
    assert rel(mom - mom0, mo - mom0) < 1e-12
    assert np.allclose(fg, fo, rtol=1e-12, atol=0)


def test_force_rejects_zmobius_and_bad_sizes(oracle):
    L = (4, 4, 4, 4)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=226))
    D = DiracOpMobius(lat, mass=0.1, ls=4)
    zb = np.array([1.5 + 0.1j] * 4)
    D.set_zmobius(zb, zb - 1.0)
    with pytest.raises(A.CpsGpuError):
        D.EvolveMomFforce(np.zeros(4 * 256 * 18), np.zeros(D.f_size), 0.1)
    W = DiracOpWilson(lat, mass=0.1)
    with pytest.raises(TypeError):
        W.EvolveMomFforce(np.zeros(10), np.zeros(W.f_size), 0.1)


@pytest.mark.parametrize("measure", [False, True])
def test_rhmc_evolve_mom_fforce(oracle, measure):
    """RHMC_EvolveMomFforce (f_wilson.C:689-757): the pole sum, and with
    FORCE_MEASURE_YES the ForceArg of the summed force (Matrix::norm per link)."""
    kind, L, ls, bc = "dwf", (4, 4, 4, 4), 4, (1, 1, 1, -1)
    D, ops, mass = _setup(oracle, kind, L, ls, bc, 227)
    sols = [gen_gaussian(D.f_size, seed=228 + k) for k in range(3)]
    alpha = np.array([0.5, -0.125, 2.0])
    dt = 0.02
    mom0 = gen_gaussian(4 * int(np.prod(L)) * 18, seed=231)
    tot = np.zeros_like(mom0)
    for s_, a in zip(sols, alpha):
        tot, _ = ops.fforce(kind, s_, dt * a, mass=mass, kappa=D.kappa, mom=tot)
    mom = mom0.copy()
    fa = D.RHMC_EvolveMomFforce(mom, sols, alpha, dt, force_measure=measure)
    assert rel(mom - mom0, tot) < 1e-12
    if measure:
        t = (tot[0::2] + 1j * tot[1::2]).reshape(-1, 3, 3)
        n = np.sqrt(np.maximum(-2 * np.einsum("lab,lba->l", t, t).real, 0))
        assert np.allclose(fa, (n.mean(), np.sqrt(np.mean(n ** 2)), n.max()), rtol=1e-12, atol=0)
    else:
        assert fa == (0.0, 0.0, 0.0)
