"""Block traversal orders of the hop launches (cpsgpu_set_hop_shape's
`order`): which (site block, slice group) each thread block takes changes
nothing a thread computes, so every field written is bit-identical between
orders; only the fused reductions add their per-block partials in another
order.  Covered: Wilson and DWF Dslash (both checkerboards, both daggers),
MatPc, MatPcDagMatPc at FP64, FP32 and FP16, one and two slices per thread,
against each other and the oracle; a mixed-precision CG per order; the
refusals."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpWilson, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel

pytestmark = pytest.mark.gpu

TOL = {A.DOUBLE: 1e-13, A.SINGLE: 2e-6, A.HALF: 5e-3}
ORDERS = (DiracOpDwf.ORDER_SLICES, DiracOpDwf.ORDER_SITES)


def _lat(L, seed=51):
    A.check(A.lib().cpsgpu_set_device(0))
    u = gen_gauge(L, seed=seed)
    lat = Lattice(L, (1, 1, 1, -1))
    lat.import_gauge(u)
    return u, lat


def _apply(D, psi, prec):
    res = {}
    for cb in (0, 1):
        for dag in (0, 1):
            res[f"dslash{cb}{dag}"] = D.Dslash(psi, cb, dag, prec)
    res["matpc"] = D.MatPc(psi, prec)
    res["mdagm"], res["dot"] = D.MatPcDagMatPc(psi, prec)
    return res


def _same(out, tol_dot=1e-12):
    base = out[ORDERS[0]]
    for o in ORDERS[1:]:
        for k in base:
            if k == "dot":
                assert out[o][k] == pytest.approx(base[k], rel=tol_dot)
            else:
                np.testing.assert_array_equal(out[o][k], base[k], err_msg=f"order {o}: {k}")


@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE, A.HALF])
@pytest.mark.parametrize("ns", [1, 2])
@pytest.mark.parametrize("L,ls,shape", [((8, 8, 8, 8), 16, (64, 2)), ((4, 4, 4, 8), 8, (32, 1)),
                                        ((8, 4, 4, 6), 8, (32, 2))])
def test_dwf_orders_bitwise(oracle, prec, ns, L, ls, shape):
    if ns == 2 and (prec == A.DOUBLE or ls % (4 * shape[1])):
        pytest.skip("no pair kernel for this case")
    u, lat = _lat(L)
    D = DiracOpDwf(lat, mass=0.05, ls=ls, m5=1.8)
    psi = gen_gaussian(D.f_size, seed=52)
    out = {}
    for o in ORDERS:
        D.set_hop_shape(prec, shape[0], shape[1], ns, o)
        assert D.hop_shape(prec) == (shape[0], shape[1], ns, o)
        out[o] = _apply(D, psi, prec)
    _same(out)
    ops = OracleOps(oracle, L, u, ls=ls, m5=1.8)
    for cb in (0, 1):
        for dag in (0, 1):
            ref = ops.dwf_dslash(psi, 0.05, cb, dag)
            assert rel(out[ORDERS[-1]][f"dslash{cb}{dag}"], ref) < TOL[prec]


@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE, A.HALF])
def test_wilson_orders_bitwise(oracle, prec):
    L = (8, 8, 8, 8)
    u, lat = _lat(L, seed=53)
    D = DiracOpWilson(lat, mass=0.1)
    psi = gen_gaussian(D.f_size, seed=54)
    out = {}
    for o in ORDERS:
        D.set_hop_shape(prec, 64, 1, 1, o)
        out[o] = _apply(D, psi, prec)
    _same(out)
    ops = OracleOps(oracle, L, u)
    for cb in (0, 1):
        for dag in (0, 1):
            assert rel(out[ORDERS[-1]][f"dslash{cb}{dag}"], ops.wilson_dslash(psi, cb, dag)) < TOL[prec]


def test_orders_mixed_cg():
    _, lat = _lat((8, 8, 8, 8), seed=55)
    D = DiracOpDwf(lat, mass=0.05, ls=8, m5=1.8)
    src = gen_gaussian(D.f_size, seed=56)
    sols = {}
    for o in ORDERS:
        D.set_hop_shape(A.SINGLE, 32, 2, 1, o)
        x = np.zeros_like(src)
        r = D.InvCg(x, src, stop_rsd=1e-10, max_num_iter=3000, precision=A.SINGLE)
        assert r.status == A.CONVERGED and r.true_res <= 1e-10
        sols[o] = (x, r.iterations)
    for o in ORDERS[1:]:
        assert abs(sols[o][1] - sols[ORDERS[0]][1]) <= 2
        assert rel(sols[o][0], sols[ORDERS[0]][0]) < 1e-8


def test_order_validation():
    _, lat = _lat((6, 4, 2, 6))
    D = DiracOpDwf(lat, mass=0.05, ls=4, m5=1.8)
    with pytest.raises(A.CpsGpuError):
        D.set_hop_shape(A.SINGLE, 32, 1, 1, 2)
    D.set_hop_shape(A.SINGLE, 32, 1, 1, D.ORDER_SITES)
    assert D.hop_shape(A.SINGLE)[3] == D.ORDER_SITES


def test_finalize_forgets_tuned_shapes():
    """cpsgpu_finalize (the end of a job) waits for the device and drops the
    launch-shape table: the default shape is back, and the library works on"""
    _, lat = _lat((4, 4, 4, 8))
    D = DiracOpDwf(lat, mass=0.05, ls=8, m5=1.8)
    A.check(A.lib().cpsgpu_finalize())  # earlier tests set shapes for this key
    default = D.hop_shape(A.SINGLE)
    D.set_hop_shape(A.SINGLE, 64, 1, 1, D.ORDER_SITES)
    assert D.hop_shape(A.SINGLE) == (64, 1, 1, D.ORDER_SITES)
    psi = gen_gaussian(D.f_size, seed=57)
    before = D.Dslash(psi, 1, 0, A.SINGLE)
    A.check(A.lib().cpsgpu_finalize())
    assert D.hop_shape(A.SINGLE) == default
    np.testing.assert_array_equal(D.Dslash(psi, 1, 0, A.SINGLE), before)
