"""Parity of the sm_100a operators (through the C ABI) with the oracle:
Wilson, Shamir DWF and Mobius, every precision.  FP64 must agree to 1e-13
relative (one dslash application); FP32 to 2e-6; FP16 storage with per-site
norms to 5e-3."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpMobius, DiracOpWilson, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel, vh_of
from oracle.loader import apply_bc_signs

pytestmark = pytest.mark.gpu

TOL = {A.DOUBLE: 1e-13, A.SINGLE: 2e-6, A.HALF: 5e-3}
PRECS = [A.DOUBLE, A.SINGLE, A.HALF]


@pytest.fixture(params=[18, 12, "f32"], ids=["links18", "links12", "f32links"])
def link_reals(request):
    """FP32 / FP16 operators read full links or rebuild the third row; the
    FP16 operator may read FP32 links (12 reals here, 18 for FP32)."""
    return request.param


def _set_links(lat, reals):
    if reals == "f32":
        A.check(A.lib().cpsgpu_set_link_reals(lat._h, A.SINGLE, 18))
        A.check(A.lib().cpsgpu_set_link_reals(lat._h, A.HALF, A.LINKS_F32_12))
        return
    for prec in (A.SINGLE, A.HALF):
        A.check(A.lib().cpsgpu_set_link_reals(lat._h, prec, reals))


def _lat(L, u, bc=(1, 1, 1, -1), signs=False):
    lat = Lattice(L, bc)
    lat.import_gauge(apply_bc_signs(u, L, bc) if signs else u, signs_applied=signs)
    return lat


@pytest.mark.parametrize("L,bc", [((4, 4, 4, 4), (1, 1, 1, -1)), ((8, 8, 8, 8), (1, 1, 1, -1)),
                                  ((4, 6, 2, 8), (-1, 1, -1, -1)), ((2, 2, 2, 2), (1, 1, 1, 1))])
def test_wilson_operators(oracle, link_reals, L, bc):
    u = gen_gauge(L, seed=31)
    ops = OracleOps(oracle, L, u, ls=1, bc=bc)
    lat = _lat(L, u, bc)
    _set_links(lat, link_reals)
    D = DiracOpWilson(lat, mass=1 / (2 * 0.12) - 4)
    assert D.kappa == pytest.approx(0.12, rel=1e-15)
    psi = gen_gaussian(ops.n, seed=32)
    for prec in PRECS:
        for cb in (0, 1):
            for dag in (0, 1):
                assert rel(D.Dslash(psi, cb, dag, prec), ops.wilson_dslash(psi, cb, dag)) < TOL[prec]
        for dag in (0, 1):
            assert rel((D.MatPcDag if dag else D.MatPc)(psi, prec), ops.wilson_m(psi, D.kappa, dag)) < TOL[prec]
        y, d = D.MatPcDagMatPc(psi, prec)
        yo, do = ops.wilson_mdagm(psi, D.kappa)
        assert rel(y, yo) < TOL[prec] and abs(d / do - 1) < TOL[prec]


def test_signs_applied_import_and_recon(oracle):
    L, bc = (4, 4, 4, 8), (1, 1, 1, -1)
    u = gen_gauge(L, seed=33)
    ops = OracleOps(oracle, L, u, ls=1, bc=bc)
    lat = _lat(L, u, bc, signs=True)
    err, recon12 = lat.gauge_info()
    assert err < 1e-14 and recon12
    D = DiracOpWilson(lat, mass=0.1)
    psi = gen_gaussian(ops.n, seed=34)
    assert rel(D.Dslash(psi, 1, 0), ops.wilson_dslash(psi, 1, 0)) < 1e-13


def test_non_su3_links_use_18_reals(oracle):
    """Links that are not SU(3): the FP64 path must fall back to full links."""
    L = (4, 4, 2, 4)
    u = gen_gaussian(int(np.prod(L)) * 72, seed=35)
    ops = OracleOps(oracle, L, u, ls=1)
    lat = _lat(L, u)
    err, recon12 = lat.gauge_info()
    assert err > 1e-3 and not recon12
    D = DiracOpWilson(lat, mass=0.1)
    psi = gen_gaussian(ops.n, seed=36)
    for cb in (0, 1):
        assert rel(D.Dslash(psi, cb, 1), ops.wilson_dslash(psi, cb, 1)) < 1e-13
    with pytest.raises(A.CpsGpuError):
        D.InvCg(np.zeros(ops.n), psi, precision=A.SINGLE, max_num_iter=5)


@pytest.mark.parametrize("L,ls,mass", [((4, 4, 4, 8), 8, 0.01), ((4, 2, 4, 4), 5, 0.1), ((2, 2, 2, 2), 2, 0.5)])
def test_dwf_operators(oracle, link_reals, L, ls, mass):
    u = gen_gauge(L, seed=41)
    ops = OracleOps(oracle, L, u, ls=ls)
    lat = _lat(L, u)
    _set_links(lat, link_reals)
    D = DiracOpDwf(lat, mass=mass, ls=ls, m5=1.8)
    psi = gen_gaussian(ops.n, seed=42)
    for prec in PRECS:
        for cb in (0, 1):
            for dag in (0, 1):
                assert rel(D.Dslash(psi, cb, dag, prec), ops.dwf_dslash(psi, mass, cb, dag)) < TOL[prec]
        for dag in (0, 1):
            assert rel((D.MatPcDag if dag else D.MatPc)(psi, prec), ops.dwf_m(psi, mass, dag)) < TOL[prec]
        y, d = D.MatPcDagMatPc(psi, prec)
        yo, do = ops.dwf_mdagm(psi, mass)
        assert rel(y, yo) < TOL[prec] and abs(d / do - 1) < TOL[prec]


@pytest.mark.parametrize("L,ls,mass,b,c", [((4, 4, 4, 8), 12, 0.005, 1.5, 0.5), ((4, 2, 4, 4), 5, 0.1, 2.0, 1.0),
                                           ((2, 2, 4, 4), 4, 0.3, 1.0, 0.0)])
def test_mobius_operators(oracle, link_reals, L, ls, mass, b, c):
    u = gen_gauge(L, seed=51)
    ops = OracleOps(oracle, L, u, ls=ls, b=b, c=c)
    lat = _lat(L, u)
    _set_links(lat, link_reals)
    D = DiracOpMobius(lat, mass=mass, ls=ls, m5=1.8, b=b, c=c)
    psi = gen_gaussian(ops.n, seed=52)
    for prec in PRECS:
        for dag in (0, 1):
            assert rel(D.M5inv(psi, dag, prec), ops.mobius_m5inv(psi, mass, dag)) < TOL[prec]
            for cb in (0, 1):
                assert rel(D.Dslash4(psi, cb, dag, prec), ops.mobius_dslash_4(psi, mass, cb, dag)) < TOL[prec]
            assert rel((D.MatPcDag if dag else D.MatPc)(psi, prec), ops.mobius_m(psi, mass, dag)) < TOL[prec]
        y, d = D.MatPcDagMatPc(psi, prec)
        yo, do = ops.mobius_mdagm(psi, mass)
        assert rel(y, yo) < TOL[prec] and abs(d / do - 1) < TOL[prec]


def test_reductions_are_deterministic(oracle):
    L = (8, 8, 8, 8)
    u = gen_gauge(L, seed=61)
    lat = _lat(L, u)
    D = DiracOpDwf(lat, mass=0.01, ls=4)
    psi = gen_gaussian(D.f_size, seed=62)
    outs = [D.MatPcDagMatPc(psi) for _ in range(3)]
    for y, d in outs[1:]:
        assert d == outs[0][1] and np.array_equal(y, outs[0][0])


@pytest.mark.parametrize("L,ls,mass", [((4, 4, 4, 8), 8, 0.01), ((4, 2, 4, 4), 5, 0.1)])
def test_zmobius_operators(oracle, L, ls, mass):
    """Complex per-slice b_s, c_s (DiracOpZMobius) in every precision"""
    u = gen_gauge(L, seed=53)
    ops = OracleOps(oracle, L, u, ls=ls)
    b = np.array([1.5 + 0.25j * np.sin(1.0 + s) for s in range(ls)])
    c = b - 1.0
    ops.set_zmobius(b, c)
    lat = _lat(L, u)
    D = DiracOpMobius(lat, mass=mass, ls=ls, m5=1.8, b=1.5, c=0.5)
    D.set_zmobius(b, c)
    psi = gen_gaussian(ops.n, seed=54)
    for prec in PRECS:
        for dag in (0, 1):
            assert rel(D.M5inv(psi, dag, prec), ops.mobius_m5inv(psi, mass, dag)) < TOL[prec]
            for cb in (0, 1):
                assert rel(D.Dslash4(psi, cb, dag, prec), ops.mobius_dslash_4(psi, mass, cb, dag)) < TOL[prec]
            assert rel((D.MatPcDag if dag else D.MatPc)(psi, prec), ops.mobius_m(psi, mass, dag)) < TOL[prec]
        y, d = D.MatPcDagMatPc(psi, prec)
        yo, do = ops.mobius_mdagm(psi, mass)
        assert rel(y, yo) < TOL[prec] and abs(d / do - 1) < TOL[prec]
