"""Parity at the benchmarked sizes: the library's FP64 operators against the
reference's own kernels (compiled from its sources, oracle/_ref) on the full
lattices of the measured workloads, and the FP64 CG against the oracle's
CG (pinned to the reference's InvCgShift) for a fixed number of
iterations on the headline system.

* DWF 16^3 x 32, Ls = 16, M5 = 1.8, m_f = 0.01: dwf_dslash
  (dwf_dslash.C:32-51) for (cb, dag) = (1, 0) and (0, 1), <= 1e-13 relative;
  the FP32 and FP16-storage dslash within their storage tolerances;
* Mobius 24^3 x 64, Ls = 12, b = 1.5, c = 0.5, m_f = 0.005: zmobius_dslash_4
  (zmobius_dslash_4.C:34-221) and zmobius_m5inv (zmobius_m5inv.C:807),
  <= 1e-13 relative;
* the DWF headline system: three FP64 CG iterations (max_num_iter = 4,
  inv_cg.C:275) give the oracle's iterate to 1e-12 and its iteration count.
"""
import ctypes as C

import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpMobius, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel
from oracle.loader import apply_bc_signs, p

pytestmark = pytest.mark.gpu
BC = (1, 1, 1, -1)


@pytest.fixture(scope="module")
def dwf_system():
    A.check(A.lib().cpsgpu_set_device(0))
    L, ls = (16, 16, 16, 32), 16
    u = gen_gauge(L, seed=20261203, width=0.3)
    lat = Lattice(L, BC)
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=0.01, ls=ls, m5=1.8)
    yield L, ls, u, D
    D.close()
    lat.close()


def test_dwf_dslash_16x32_ls16_vs_reference(reference, dwf_system):
    L, ls, u, D = dwf_system
    reference.ref_init(*L, ls, 1.8, 1.5, 0.5, BC[3])
    us = apply_bc_signs(u, L, BC)
    x = gen_gaussian(D.f_size, seed=41)
    for cb, dag in ((1, 0), (0, 1)):
        y = np.zeros_like(x)
        reference.ref_dwf_dslash(p(y), p(us), p(x), 0.01, cb, dag)
        assert rel(D.Dslash(x, cb, dag), y) <= 1e-13
        if (cb, dag) == (1, 0):
            assert rel(D.Dslash(x, cb, dag, prec=A.SINGLE), y) <= 2e-6
            assert rel(D.Dslash(x, cb, dag, prec=A.HALF), y) <= 5e-3


def test_mobius_24x64_ls12_vs_reference(reference):
    A.check(A.lib().cpsgpu_set_device(0))
    L, ls, mass = (24, 24, 24, 64), 12, 0.005
    u = gen_gauge(L, seed=20261206, width=0.3)
    lat = Lattice(L, BC)
    lat.import_gauge(u)
    D = DiracOpMobius(lat, mass=mass, ls=ls, m5=1.8, b=1.5, c=0.5)
    reference.ref_init(*L, ls, 1.8, 1.5, 0.5, BC[3])
    us = apply_bc_signs(u, L, BC)
    x = gen_gaussian(D.f_size, seed=42)
    y = np.zeros_like(x)
    reference.ref_zmobius_dslash_4(p(y), p(us), p(x), 0, 0, mass)
    assert rel(D.Dslash4(x, 0, 0), y) <= 1e-13
    y = x.copy()
    reference.ref_zmobius_m5inv(p(y), mass, 0)
    assert rel(D.M5inv(x, 0), y) <= 1e-13
    D.close()
    lat.close()


def test_dwf_headline_fixed_iteration_cg_vs_oracle(oracle, dwf_system):
    L, ls, u, D = dwf_system
    ops = OracleOps(oracle, L, u, ls=ls, bc=BC, m5=1.8)
    b = gen_gaussian(D.f_size, seed=43)
    xo, ito, tro = ops.invcg("dwf", b, mass=0.01, stop_rsd=1e-14, max_num_iter=4)
    x = np.zeros(D.f_size)
    r = D.InvCg(x, b, stop_rsd=1e-14, max_num_iter=4)
    assert r.iterations == ito == 4 and r.status == A.MAX_ITER
    assert rel(x, xo) <= 1e-12
    assert abs(r.true_res - tro) <= 1e-10 * tro
