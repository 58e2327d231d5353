"""The Ls x Ls mixing of FP16 fields on the tensor cores (mix_tc.cu,
cpsgpu_set_mix_impl): M5^-1 (zmobius_m5inv.C:247-396 as a dense matrix)
against the oracle within the FP16-storage tolerance and against the
CUDA-core kernel, MatPcDagMatPc in FP16, and the FP16-inner solve to a true
residual of 1e-10, for Ls = 5, 8, 12 and 16 (and a checkerboard volume
that is not a multiple of the 16-site block); complex coefficients stay on the CUDA
cores."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpMobius, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,ls", [((4, 4, 4, 8), 12), ((4, 4, 4, 4), 16), ((6, 4, 4, 4), 5), ((6, 2, 2, 2), 8)])
def test_mix_tc(oracle, L, ls):
    A.check(A.lib().cpsgpu_set_device(0))
    mass = 0.05
    u = gen_gauge(L, seed=801)
    lat = Lattice(L)
    lat.import_gauge(u)
    D = DiracOpMobius(lat, mass=mass, ls=ls, b=1.5, c=0.5)
    ops = OracleOps(oracle, L, u, ls=ls, b=1.5, c=0.5)
    x = gen_gaussian(D.f_size, seed=802)
    ref = ops.mobius_m5inv(x, mass, 0)
    cuda_cores = D.M5inv(x, 0, prec=A.HALF)
    D.set_mix_impl(True)
    tc = D.M5inv(x, 0, prec=A.HALF)
    assert rel(tc, ref) < 5e-3
    assert rel(tc, cuda_cores) < 2e-3
    assert rel(D.M5inv(x, 0, prec=A.DOUBLE), ref) < 1e-13  # FP64 keeps the CUDA cores
    yo, _ = ops.mobius_mdagm(x, mass)
    assert rel(D.MatPcDagMatPc(x, prec=A.HALF)[0], yo) < 5e-3
    sol = np.zeros(D.f_size)
    r = D.InvCg(sol, x, stop_rsd=1e-10, precision=A.HALF)
    assert r.status == A.CONVERGED and r.true_res <= 1e-10
    Ax, _ = ops.mobius_mdagm(sol, mass)
    assert rel(Ax, x) <= 1.5e-10
