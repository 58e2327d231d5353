"""The Mobius operator under every preconditioning type (cpsgpu_dirac_set_pc_type:
ORIG, SYM1, SYM2, SYM1_MIT, SYM2_MIT, SYM3; zmobius_m.C:40-74,
zmobius_mdag.C:41-69) against the oracle's orc_mobius_m_pc, which is pinned
to the compiled reference (tests/test_reference_mobius_pc.py), and once
directly against the reference's own DiracOpMobius (oracle/_ref):

* MatPc, MatPcDag and MatPcDagMatPc in FP64 (<= 1e-13), FP32 and FP16;
* the CG on MatPcDagMatPc (FP64 and the FP32-inner mixed solve) to a true
  residual of 1e-10 for every type but SYM3 (its MatPc lacks the kappa_b
  factors and the CG does not converge on it, in the reference alike), and a
  capped SYM3 solve that stops at the oracle's iterate;
* MatInv (d_op_mobius.C:407-700) for ORIG, SYM1, SYM2 and SYM3 against the
  oracle's, and the MIT types refused as the reference refuses them;
* the multishift CG under a non-default type."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpMobius, Lattice, gen_gauge, gen_gaussian
from helpers import OracleOps, rel
from oracle import refsolve

pytestmark = pytest.mark.gpu

L, LS, MASS, B, C = (4, 4, 4, 8), 8, 0.1, 1.5, 0.5
PCS = {"ORIG": 0, "SYM1": 1, "SYM2": 2, "SYM1_MIT": 3, "SYM2_MIT": 4, "SYM3": 5}
TOL = {A.DOUBLE: 1e-13, A.SINGLE: 2e-6, A.HALF: 5e-3}


@pytest.fixture(scope="module")
def setup(oracle):
    A.check(A.lib().cpsgpu_set_device(0))
    u = gen_gauge(L, seed=71)
    lat = Lattice(L)
    lat.import_gauge(u)
    ops = OracleOps(oracle, L, u, ls=LS, b=B, c=C)
    return lat, ops


@pytest.mark.parametrize("name", list(PCS))
@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE, A.HALF])
def test_pc_operators(setup, name, prec):
    lat, ops = setup
    D = DiracOpMobius(lat, mass=MASS, ls=LS, b=B, c=C, pc_type=PCS[name])
    assert D.pc_type == PCS[name]
    x = gen_gaussian(D.f_size, seed=72)
    assert rel(D.MatPc(x, prec), ops.mobius_m_pc(x, MASS, 0, PCS[name])) < TOL[prec]
    assert rel(D.MatPcDag(x, prec), ops.mobius_m_pc(x, MASS, 1, PCS[name])) < TOL[prec]
    y, dot = D.MatPcDagMatPc(x, prec)
    yo, doto = ops.mobius_mdagm_pc(x, MASS, PCS[name])
    assert rel(y, yo) < TOL[prec]
    assert dot == pytest.approx(doto, rel=max(TOL[prec], 1e-12))


@pytest.mark.parametrize("name", ["ORIG", "SYM1_MIT"])
def test_pc_operators_against_the_reference(tmp_path, name):
    """the reference's own DiracOpMobius under the type, on its own gauge field"""
    if not refsolve.available():
        pytest.skip("reference solver library not built")
    from oracle import convert as CV
    n = 24 * LS * int(np.prod(L)) // 2
    src = gen_gaussian(n, seed=73)
    np.save(tmp_path / "src.npy", src)
    r = refsolve.run_child({"L": list(L), "ls": LS, "kind": "mobius", "task": "pcops", "gauge": "disord",
                            "src": str(tmp_path / "src.npy"), "mass": MASS, "b": B, "c": C, "pc_type": PCS[name]})
    A.check(A.lib().cpsgpu_set_device(0))
    lat = Lattice(L)
    lat.import_gauge(CV.gcanon_to_wilson(r["gauge"], L))
    D = DiracOpMobius(lat, mass=MASS, ls=LS, b=B, c=C, pc_type=PCS[name])
    assert rel(D.MatPc(src), r["matpc"]) < 1e-13
    assert rel(D.MatPcDag(src), r["matpcdag"]) < 1e-13


@pytest.mark.parametrize("name", ["ORIG", "SYM1", "SYM2", "SYM1_MIT", "SYM2_MIT"])
@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE])
def test_pc_cg(setup, name, prec):
    lat, ops = setup
    D = DiracOpMobius(lat, mass=MASS, ls=LS, b=B, c=C, pc_type=PCS[name])
    src = gen_gaussian(D.f_size, seed=74)
    x = np.zeros_like(src)
    r = D.InvCg(x, src, stop_rsd=1e-10, max_num_iter=20000, precision=prec)
    assert r.status == A.CONVERGED and r.true_res <= 1e-10
    ax, _ = ops.mobius_mdagm_pc(x, MASS, PCS[name])
    assert rel(ax, src) <= 1.5e-10


def test_pc_sym3_capped_cg(setup):
    lat, ops = setup
    D = DiracOpMobius(lat, mass=MASS, ls=LS, b=B, c=C, pc_type=PCS["SYM3"])
    src = gen_gaussian(D.f_size, seed=75)
    x = np.zeros_like(src)
    r = D.InvCg(x, src, stop_rsd=1e-14, max_num_iter=21)
    assert r.iterations == 21
    sol, it, tr = ops.invcg("mobius", src, mass=MASS, stop_rsd=1e-14, max_num_iter=21, pc=PCS["SYM3"])
    assert it == 21 and rel(x, sol) < 1e-10


@pytest.mark.parametrize("name,stop,max_iter", [("ORIG", 1e-10, 5000), ("SYM1", 1e-10, 5000),
                                                ("SYM2", 1e-10, 5000), ("SYM3", 1e-14, 21)])
def test_pc_matinv(setup, name, stop, max_iter):
    lat, ops = setup
    D = DiracOpMobius(lat, mass=MASS, ls=LS, b=B, c=C, pc_type=PCS[name])
    src = gen_gaussian(2 * D.f_size, seed=76)
    out = np.zeros_like(src)
    r = D.MatInv(out, src, stop_rsd=stop, max_num_iter=max_iter)
    ref, it, tr = ops.mobius_matinv_pc(src, MASS, PCS[name], stop_rsd=stop, max_num_iter=max_iter)
    if max_iter > 100:
        assert r.status == A.CONVERGED and abs(r.iterations - it) <= 1 and rel(out, ref) < 1e-8
    else:
        assert r.iterations == it == max_iter and rel(out, ref) < 1e-10


@pytest.mark.parametrize("name", ["SYM1_MIT", "SYM2_MIT"])
def test_pc_matinv_refuses_mit(setup, name):
    lat, _ = setup
    D = DiracOpMobius(lat, mass=MASS, ls=LS, b=B, c=C, pc_type=PCS[name])
    src = gen_gaussian(2 * D.f_size, seed=77)
    with pytest.raises(A.CpsGpuError):
        D.MatInv(np.zeros_like(src), src, stop_rsd=1e-8)


def test_pc_multishift(setup):
    lat, ops = setup
    D = DiracOpMobius(lat, mass=MASS, ls=LS, b=B, c=C, pc_type=PCS["SYM1"])
    chi = gen_gaussian(D.f_size, seed=78)
    shifts = [0.001, 0.05, 0.4]
    psi = [np.zeros_like(chi) for _ in shifts]
    rs = np.full(len(shifts), 1e-10)
    D.MInvCG(psi, chi, float(chi @ chi), shifts, rs)
    for sh, x in zip(shifts, psi):
        ax, _ = ops.mobius_mdagm_pc(x, MASS, PCS["SYM1"])
        assert rel(ax + sh * x, chi) < 1e-9


def test_pc_refusals(setup):
    lat, _ = setup
    D = DiracOpMobius(lat, mass=MASS, ls=LS, b=B, c=C)
    with pytest.raises(A.CpsGpuError):
        D.set_pc_type(6)
    D.set_zmobius(np.full(LS, 1.5 + 0.1j), np.full(LS, 0.5))
    with pytest.raises(A.CpsGpuError):
        D.set_pc_type(PCS["SYM1"])  # per-slice complex b, c: SYM2 only
