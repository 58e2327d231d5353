"""The unpreconditioned operators (Mat, MatDag, MatHerm), the shifted Mobius
MatPcDagMatPc and the fifth-direction spacing a5 through the C ABI against
the oracle, whose compositions of these operators and whose a5 kernels are
pinned to the reference's own code (tests/test_reference_operators.py):
d_op_wilson.C:362-443, d_op_dwf.C:541-660, d_op_mobius.C:235, :735-942,
dwf_dslash_5_plus_omp.C:137-138, dwf_init.C:97-98, d_op_mobius.C:105-108."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpMobius, DiracOpWilson, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _setup(kind, L, ls, a5=1.0, seed=601):
    A.check(A.lib().cpsgpu_set_device(0))
    u = gen_gauge(L, seed=seed)
    lat = Lattice(L)
    lat.import_gauge(u)
    mass = 0.1
    if kind == "wilson":
        D = DiracOpWilson(lat, mass=mass)
    elif kind == "dwf":
        D = DiracOpDwf(lat, mass=mass, ls=ls, a5_inv=a5)
    else:
        D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5, a5_inv=a5)
    return lat, D, mass


@pytest.mark.parametrize("kind,L,ls,a5", [("wilson", (4, 4, 4, 8), 1, 1.0), ("dwf", (4, 4, 4, 4), 6, 1.0),
                                          ("dwf", (4, 4, 2, 4), 5, 0.8), ("mobius", (4, 4, 4, 4), 6, 1.0),
                                          ("mobius", (4, 2, 4, 4), 4, 1.25)])
def test_mat_matdag_matherm(oracle, kind, L, ls, a5):
    lat, D, mass = _setup(kind, L, ls, a5)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=601), ls=ls, b=1.5, c=0.5, a5_inv=a5)
    x = gen_gaussian(2 * D.f_size, seed=602)
    assert rel(D.Mat(x), ops.mat(kind, x, mass, D.kappa, 0)) < TOL
    if kind == "mobius":
        with pytest.raises(A.CpsGpuError):
            D.MatDag(x)
    else:
        assert rel(D.MatDag(x), ops.mat(kind, x, mass, D.kappa, 1)) < TOL
    assert rel(D.MatHerm(x), ops.matherm(kind, x, mass, D.kappa)) < TOL


@pytest.mark.parametrize("a5", [1.0, 1.25])
def test_mobius_matpc_dag_matpc_shift(oracle, a5):
    L, ls = (4, 4, 4, 4), 6
    lat, D, mass = _setup("mobius", L, ls, a5)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=601), ls=ls, b=1.5, c=0.5, a5_inv=a5)
    x = gen_gaussian(D.f_size, seed=603)
    y, dot = D.MatPcDagMatPcShift(x, 0.3)
    yo, do = ops.mobius_mdagm_shift(x, mass, 0.3)
    assert rel(y, yo) < TOL and abs(dot / do - 1) < TOL
    y32, _ = D.MatPcDagMatPcShift(x, 0.3, prec=A.SINGLE)
    assert rel(y32, yo) < 2e-6
    # mu = 0 is MatPcDagMatPc
    y0, d0 = D.MatPcDagMatPcShift(x, 0.0)
    y1, d1 = D.MatPcDagMatPc(x)
    assert rel(y0, y1) < TOL and abs(d0 / d1 - 1) < TOL
    D2 = DiracOpDwf(lat, mass=0.1, ls=ls)
    with pytest.raises(A.CpsGpuError):  # DiracOpMobius only
        A.check(A.lib().cpsgpu_matpc_dag_matpc_shift(D2._h, A.dptr(np.zeros(D2.f_size)), A.dptr(x), 0.3, None,
                                                      A.DOUBLE))


@pytest.mark.parametrize("kind", ["dwf", "mobius"])
def test_a5_inv_operators_and_solve(oracle, kind):
    """dwf_a5_inv != 1: MatPcDagMatPc in every precision and the mixed CG"""
    L, ls, a5 = (4, 4, 4, 8), 8, 0.8
    lat, D, mass = _setup(kind, L, ls, a5)
    ops = OracleOps(oracle, L, gen_gauge(L, seed=601), ls=ls, b=1.5, c=0.5, a5_inv=a5)
    if kind == "dwf":
        assert abs(D.kappa - 1 / (2 * (4 + a5 - 1.8))) < 1e-15
    x = gen_gaussian(D.f_size, seed=604)
    yo, do = ops.dwf_mdagm(x, mass) if kind == "dwf" else ops.mobius_mdagm(x, mass)
    y, d = D.MatPcDagMatPc(x)
    assert rel(y, yo) < TOL and abs(d / do - 1) < TOL
    assert rel(D.MatPcDagMatPc(x, prec=A.SINGLE)[0], yo) < 2e-6
    assert rel(D.MatPcDagMatPc(x, prec=A.HALF)[0], yo) < 5e-3
    sol = np.zeros(D.f_size)
    r = D.InvCg(sol, x, stop_rsd=1e-10, precision=A.SINGLE)
    assert r.status == A.CONVERGED
    Ax, _ = ops.dwf_mdagm(sol, mass) if kind == "dwf" else ops.mobius_mdagm(sol, mass)
    assert rel(Ax, x) <= 1.5e-10
