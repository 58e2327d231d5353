"""The bulk-copy staged Ls x Ls mixing kernel (mix_bulk.cu, cpsgpu_set_mix_impl
3: FP16 fields, real b, c, Ls 8, 10, 12, 16, sites per checkerboard slice a
multiple of 32) against the register-tiled kernel whose arithmetic it
repeats: the same bits for M5^-1 and its dagger, MatPc, MatPcDag and
MatPcDagMatPc, over lattices with one and with many 32-site tiles per slice
(so every block of the persistent grid walks several tiles through both
stages), a batched FP16-inner solve with its gated right-hand sides, and the
oracle; cases the kernel does not cover (FP32 and FP64 fields, other Ls, a
checkerboard volume not a multiple of 32) fall back to the register-tiled
kernel with the same results."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpMobius, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel

pytestmark = pytest.mark.gpu


def _op(L, ls, seed):
    A.check(A.lib().cpsgpu_set_device(0))
    u = gen_gauge(L, seed=seed)
    lat = Lattice(L)
    lat.import_gauge(u)
    return u, lat, DiracOpMobius(lat, mass=0.05, ls=ls, b=1.5, c=0.5)


@pytest.mark.parametrize("L,ls", [((4, 4, 4, 4), 8), ((4, 4, 4, 8), 12), ((8, 8, 8, 8), 12), ((8, 8, 8, 16), 16),
                                  ((4, 4, 4, 8), 10), ((4, 4, 4, 4), 6), ((6, 2, 2, 2), 12)])
@pytest.mark.parametrize("prec", [A.HALF, A.SINGLE])
def test_mix_bulk_bitwise_and_oracle(oracle, L, ls, prec):
    u, lat, D = _op(L, ls, 911)
    x = gen_gaussian(D.f_size, seed=912)
    out = {}
    for impl in (D.MIX_REG, D.MIX_BULK):
        D.set_mix_impl(impl)
        out[impl] = ([D.M5inv(x, dag, prec=prec) for dag in (0, 1)] + [D.MatPcDagMatPc(x, prec=prec)[0]]
                     + [D.MatPc(x, prec=prec), D.MatPcDag(x, prec=prec)])
    for a, b in zip(out[D.MIX_REG], out[D.MIX_BULK]):
        np.testing.assert_array_equal(a, b)
    ops = OracleOps(oracle, L, u, ls=ls, b=1.5, c=0.5)
    tol = {A.SINGLE: 2e-6, A.HALF: 5e-3}[prec]
    for dag in (0, 1):
        assert rel(out[D.MIX_BULK][dag], ops.mobius_m5inv(x, 0.05, dag)) < tol


def test_mix_bulk_multi_rhs_solve_and_timing():
    L, ls = (8, 8, 8, 8), 12
    _, lat, D = _op(L, ls, 913)
    srcs = [gen_gaussian(D.f_size, seed=914 + k) for k in range(3)]
    res = {}
    for impl in (D.MIX_REG, D.MIX_BULK):
        D.set_mix_impl(impl)
        sols = [np.zeros(D.f_size) for _ in srcs]
        r = D.InvCgMulti(sols, srcs, stop_rsd=1e-10, precision=A.HALF)
        assert all(x.status == A.CONVERGED and x.true_res <= 1e-10 for x in r)
        res[impl] = (sols, [x.iterations for x in r])
    assert res[D.MIX_REG][1] == res[D.MIX_BULK][1]
    for a, b in zip(res[D.MIX_REG][0], res[D.MIX_BULK][0]):
        np.testing.assert_array_equal(a, b)
    # the timing entry reports an error if any bounded wait of the kernel ran out
    import ctypes as C
    ms, by = C.c_double(), C.c_double()
    A.check(A.lib().cpsgpu_time_m5inv(D._h, A.HALF, 3, C.byref(ms), C.byref(by)))
    assert ms.value > 0
