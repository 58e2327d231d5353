"""The benchmark systems beyond the headline one, at their full sizes, checked
by size-independent properties (the operators themselves are pinned to the
oracle at small sizes in test_gpu_operators.py):

* Mobius 24^3x64, Ls=12, b=1.5, c=0.5, M5=1.8, m_f=0.005: half-precision
  inner solve with FP64 defect correction to a true residual of 1e-10,
  against the plain FP64 CG on the same system (iteration inflation);
* DWF 16^3x32, Ls=16, m_f=0.01 with 12 point sources solved as one batch:
  every right-hand side converges and matches its sequential solve exactly;
* Wilson 32^3x64, kappa=0.125 with 16 shifts log-spaced in [1e-4, 10]:
  FP32 multishift CG then FP64 refinement of every shift to 1e-10;
* eight independent DWF solves with masses log-spaced in [0.001, 0.1] on
  lattices from 8^3x16 to 16^3x32, each to 1e-10.

Every true residual is recomputed here from the returned solution with the
FP64 operator (itself pinned to the oracle), independently of the solver's
own report."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpMobius, DiracOpWilson, Lattice, gen_gauge, gen_gaussian

pytestmark = pytest.mark.gpu


def _true_res(D, x, b, shift=0.0):
    y, _ = D.MatPcDagMatPc(x)
    return float(np.linalg.norm(b - y - shift * x) / np.linalg.norm(b))


# the solvers stop on their own FP64 residual; recomputing it here rounds differently
TOL = 1.01e-10


def test_mobius_24x64_half_inner_fp64_defect_correction():
    L, ls, mass = (24, 24, 24, 64), 12, 0.005
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=301))
    err, recon12 = lat.gauge_info()
    assert recon12 and err < 1e-14  # 12-real links
    D = DiracOpMobius(lat, mass=mass, ls=ls, m5=1.8, b=1.5, c=0.5)
    assert D.kappa == pytest.approx(1 / (2 * (1.5 * 2.2 + 1)), rel=1e-14)
    D.autotune(A.DOUBLE)
    D.autotune(A.HALF)
    b = gen_gaussian(D.f_size, seed=302)
    x64 = np.zeros(D.f_size)
    r64 = D.InvCg(x64, b, stop_rsd=1e-10, max_num_iter=20000)
    xh = np.zeros(D.f_size)
    rh = D.InvCg(xh, b, stop_rsd=1e-10, max_num_iter=20000, precision=A.HALF)
    assert r64.status == A.CONVERGED and rh.status == A.CONVERGED
    assert r64.true_res <= 1e-10 and rh.true_res <= 1e-10
    assert _true_res(D, xh, b) <= TOL and _true_res(D, x64, b) <= TOL
    assert rh.reliable_updates >= 1
    # the half-precision inner solve may take more iterations, not many more
    assert rh.iterations < 2.0 * r64.iterations


def test_dwf_12_point_sources_batched():
    L, ls, mass = (16, 16, 16, 32), 16, 0.01
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=401))
    D = DiracOpDwf(lat, mass=mass, ls=ls)
    D.autotune(A.SINGLE, nrhs=12)
    assert 1 <= D.rhs_tile(A.SINGLE, 12) <= 12
    rng = np.random.default_rng(402)
    site = int(rng.integers(0, D.f_size // 24))
    srcs = []
    for k in range(12):  # the 12 spin-colour unit vectors at one site
        e = np.zeros(D.f_size)
        e[24 * site + 2 * k] = 1.0
        srcs.append(e)
    sols = [np.zeros(D.f_size) for _ in srcs]
    res = D.InvCgMulti(sols, srcs, stop_rsd=1e-10, precision=A.SINGLE)
    for k in (0, 5, 11):
        y = np.zeros(D.f_size)
        r1 = D.InvCg(y, srcs[k], stop_rsd=1e-10, precision=A.SINGLE)
        assert res[k].iterations == r1.iterations
        assert np.array_equal(sols[k], y)
    for k in range(12):
        assert res[k].status == A.CONVERGED and res[k].true_res <= 1e-10
    assert _true_res(D, sols[7], srcs[7]) <= TOL


def test_wilson_32x64_multishift_fp32_then_fp64_refinement():
    L = (32, 32, 32, 64)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=501))
    D = DiracOpWilson(lat, mass=1 / (2 * 0.125) - 4)
    assert D.kappa == pytest.approx(0.125, rel=1e-15)
    shifts = list(np.logspace(-4, 1, 16))
    chi = gen_gaussian(D.f_size, seed=502)
    psi = [np.zeros(D.f_size) for _ in shifts]
    rs = np.full(len(shifts), 1e-10)
    D.MInvCG(psi, chi, float(chi @ chi), shifts, rs, type=A.MS_MULTI, precision=A.SINGLE)
    for s in (0, 5, 10, 15):
        assert _true_res(D, psi[s], chi, shifts[s]) <= TOL


def test_eight_independent_dwf_solves():
    masses = np.logspace(-3, -1, 8)
    lattices = [(8, 8, 8, 16), (8, 8, 8, 16), (8, 8, 8, 32), (8, 8, 16, 16), (8, 16, 16, 16), (16, 16, 16, 16),
                (16, 16, 16, 24), (16, 16, 16, 32)]
    for k, (L, mass) in enumerate(zip(lattices, masses)):
        lat = Lattice(L)
        lat.import_gauge(gen_gauge(L, seed=601 + k))
        D = DiracOpDwf(lat, mass=float(mass), ls=16)
        b = gen_gaussian(D.f_size, seed=611 + k)
        x = np.zeros(D.f_size)
        r = D.InvCg(x, b, stop_rsd=1e-10, max_num_iter=20000, precision=A.SINGLE)
        assert r.status == A.CONVERGED and r.true_res <= 1e-10
        assert _true_res(D, x, b) <= TOL
        D.close()
        lat.close()
