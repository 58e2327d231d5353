"""The register-tiled Ls x Ls mixing kernel (mix_reg.cu, the default for
FP32 and FP16 fields with real b, c at Ls 8, 10, 12, 16, 20, 24) against the
shared-memory kernel it replaced (cpsgpu_set_mix_impl 2) and the oracle.
Both sum the Ls terms of every output in the same order with fused
multiply-adds and store FP16 through the same norm rule, so every field
they write is bit-identical: M5^-1 and its dagger, MatPc, MatPcDag and
MatPcDagMatPc in FP64, FP32 and FP16, several Ls (and one the kernel does
not cover), a checkerboard volume that is not a multiple of the 32-site
block, and a batched FP16-inner solve."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpMobius, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,ls", [((4, 4, 4, 4), 8), ((4, 4, 4, 8), 12), ((6, 2, 2, 2), 16), ((4, 4, 2, 2), 10),
                                  ((2, 2, 2, 4), 20), ((2, 2, 2, 2), 24), ((4, 4, 4, 4), 6)])
@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE, A.HALF])
def test_mix_reg_bitwise_and_oracle(oracle, L, ls, prec):
    A.check(A.lib().cpsgpu_set_device(0))
    mass = 0.05
    u = gen_gauge(L, seed=901)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
    ops = OracleOps(oracle, L, u, ls=ls, b=1.5, c=0.5)
    x = gen_gaussian(D.f_size, seed=902)
    out = {}
    for impl in (D.MIX_REG, D.MIX_SHARED):
        D.set_mix_impl(impl)
        out[impl] = ([D.M5inv(x, dag, prec=prec) for dag in (0, 1)] + [D.MatPcDagMatPc(x, prec=prec)[0]]
                     + [D.MatPc(x, prec=prec), D.MatPcDag(x, prec=prec)])
    for a, b in zip(out[D.MIX_REG], out[D.MIX_SHARED]):
        np.testing.assert_array_equal(a, b)
    tol = {A.DOUBLE: 1e-13, A.SINGLE: 2e-6, A.HALF: 5e-3}[prec]
    for dag in (0, 1):
        assert rel(out[D.MIX_REG][dag], ops.mobius_m5inv(x, mass, dag)) < tol


def test_mix_reg_multi_rhs_and_solve():
    A.check(A.lib().cpsgpu_set_device(0))
    L, ls = (4, 4, 4, 8), 12
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=903))
    D = DiracOpMobius(lat, mass=0.05, ls=ls, b=1.5, c=0.5)
    srcs = [gen_gaussian(D.f_size, seed=904 + k) for k in range(3)]
    res = {}
    for impl in (D.MIX_REG, D.MIX_SHARED):
        D.set_mix_impl(impl)
        sols = [np.zeros(D.f_size) for _ in srcs]
        r = D.InvCgMulti(sols, srcs, stop_rsd=1e-10, precision=A.HALF)
        assert all(x.status == A.CONVERGED and x.true_res <= 1e-10 for x in r)
        res[impl] = (sols, [x.iterations for x in r])
    assert res[D.MIX_REG][1] == res[D.MIX_SHARED][1]
    for a, b in zip(res[D.MIX_REG][0], res[D.MIX_SHARED][0]):
        np.testing.assert_array_equal(a, b)
