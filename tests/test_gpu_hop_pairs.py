"""The DWF slice-pair hop kernel (two same-parity slices per thread sharing
their links) against the one-slice kernel and the oracle.

Per slice the pair kernel does the one-slice kernel's arithmetic operation
for operation, so every field it writes is bit-identical; only the order in
which the fused reductions (|M psi|^2, |r|^2) add up per-thread partial sums
changes, which moves them by rounding.  Covered: Dslash both checkerboards
and both daggers, MatPc with its norm, MatPcDagMatPc, a mixed-precision CG
on each, at FP32 and FP16 storage, 12- and 18-real links, several block
shapes, Ls 4, 8, 16, and a lattice whose checkerboard volume is not a
multiple of the block's site count."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel

pytestmark = pytest.mark.gpu

TOL = {A.SINGLE: 2e-6, A.HALF: 5e-3}


def _op(L, ls, reals, seed=41):
    A.check(A.lib().cpsgpu_set_device(0))
    u = gen_gauge(L, seed=seed)
    lat = Lattice(L, (1, 1, 1, -1))
    lat.import_gauge(u)
    for prec in (A.SINGLE, A.HALF):
        lat.set_link_reals(prec, reals)
    return u, lat, DiracOpDwf(lat, mass=0.05, ls=ls, m5=1.8)


@pytest.mark.parametrize("prec", [A.SINGLE, A.HALF])
@pytest.mark.parametrize("reals", [12, 18])
@pytest.mark.parametrize("L,ls,shape", [((4, 4, 4, 8), 8, (32, 2)), ((8, 8, 8, 8), 16, (32, 4)),
                                        ((8, 8, 8, 8), 16, (64, 1)), ((6, 4, 2, 6), 4, (32, 1)),
                                        ((4, 4, 4, 4), 8, (128, 2))])
def test_pairs_bitwise_against_single_slices(oracle, prec, reals, L, ls, shape):
    u, lat, D = _op(L, ls, reals)
    n = D.f_size
    psi = gen_gaussian(n, seed=42)
    bx, bs = shape
    out = {}
    for ns in (1, 2):
        D.set_hop_shape(prec, bx, bs, ns)
        assert D.hop_shape(prec) == (bx, bs, ns, D.ORDER_SLICES)
        res = {}
        for cb in (0, 1):
            for dag in (0, 1):
                res[f"dslash{cb}{dag}"] = D.Dslash(psi, cb, dag, prec)
        res["matpc"] = D.MatPc(psi, prec)
        res["mdagm"], res["dot"] = D.MatPcDagMatPc(psi, prec)
        out[ns] = res
    for k in out[1]:
        if k == "dot":
            assert out[2][k] == pytest.approx(out[1][k], rel=1e-12)
        else:
            np.testing.assert_array_equal(out[2][k], out[1][k], err_msg=k)
    # and the oracle
    ops = OracleOps(oracle, L, u, ls=ls, m5=1.8)
    for cb in (0, 1):
        for dag in (0, 1):
            ref = ops.dwf_dslash(psi, 0.05, cb, dag)
            assert rel(out[2][f"dslash{cb}{dag}"], ref) < TOL[prec]


@pytest.mark.parametrize("prec", [A.SINGLE, A.HALF])
def test_pairs_mixed_cg(prec):
    L, ls = (8, 8, 8, 8), 8
    _, lat, D = _op(L, ls, 12)
    src = gen_gaussian(D.f_size, seed=43)
    sols = {}
    for ns in (1, 2):
        D.set_hop_shape(prec, 32, 2, ns)
        x = np.zeros_like(src)
        r = D.InvCg(x, src, stop_rsd=1e-10, max_num_iter=3000, precision=prec)
        assert r.status == A.CONVERGED and r.true_res <= 1e-10
        sols[ns] = (x, r.iterations)
    # the reductions round differently: the same solve within its tolerance
    assert abs(sols[2][1] - sols[1][1]) <= 2
    assert rel(sols[2][0], sols[1][0]) < 1e-8


def test_pair_shape_validation():
    _, lat, D = _op((4, 4, 4, 4), 6, 12)
    with pytest.raises(A.CpsGpuError):
        D.set_hop_shape(A.SINGLE, 32, 2, 2)  # 6 is not a multiple of 8
    with pytest.raises(A.CpsGpuError):
        D.set_hop_shape(A.DOUBLE, 32, 1, 2)  # FP64 has no pair kernel
    with pytest.raises(A.CpsGpuError):
        D.set_hop_shape(A.SINGLE, 24, 1, 1)  # not a whole number of warps
