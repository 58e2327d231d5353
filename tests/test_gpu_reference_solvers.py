"""The library's solvers against the reference's own, on the golden fixture
tests/golden/ref_solvers.npz (made by tests/golden/make_golden_solvers.py
from the reference's compiled Lattice / DiracOp classes):

* DiracOpWilson::MatInv on the reference's f_wilson_inv test (4^4, m = 0.1,
  its fixed-seed gauge field and source, stop_rsd 1e-12): the reference's
  28 iterations (tests/f_wilson_inv/qcdlinux1.log:69) and its solution;
* DiracOpDwf / DiracOpMobius InvCg (4^4 x Ls 6, stop_rsd 1e-10) and
  DiracOpWilson::MInvCG (four shifts): the reference's iteration counts,
  solutions and, for the multishift CG, the achieved residuals;
* the mixed-precision solves reach the reference's solution.
The fields go through the library's own CANONICAL <-> WILSON conversions.
"""
from pathlib import Path

import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpMobius, DiracOpWilson, Lattice, StrOrd, fconvert, gconvert
from helpers import rel

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_solvers.npz"
L = (4, 4, 4, 4)


@pytest.fixture(scope="module")
def G():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def lat(G):
    A.check(A.lib().cpsgpu_set_device(0))
    u = G["gauge"].copy()
    gconvert(L, u, StrOrd.WILSON, StrOrd.CANONICAL)
    lt = Lattice(L, (1, 1, 1, -1))
    lt.import_gauge(u)
    return lt


@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE, A.HALF])
def test_f_wilson_inv_matinv(G, lat, prec):
    D = DiracOpWilson(lat, mass=0.1)
    src = G["fwi_src"].copy()
    fconvert(L, 1, src, StrOrd.WILSON, StrOrd.CANONICAL)
    x = np.zeros_like(src)
    r = D.MatInv(x, src, stop_rsd=1e-12, max_num_iter=500, precision=prec)
    assert r.status == A.CONVERGED and r.true_res <= 1e-12
    fconvert(L, 1, x, StrOrd.CANONICAL, StrOrd.WILSON)
    assert rel(x, G["fwi_sol"]) < 1e-10
    if prec == A.DOUBLE:
        assert r.iterations == int(G["fwi_iters"]) == 28


@pytest.mark.parametrize("kind", ["dwf", "mobius"])
@pytest.mark.parametrize("prec", [A.DOUBLE, A.SINGLE])
def test_5d_invcg(G, lat, kind, prec):
    tag = "dwf" if kind == "dwf" else "mob"
    if kind == "dwf":
        D = DiracOpDwf(lat, mass=0.1, ls=6, m5=1.8)
    else:
        D = DiracOpMobius(lat, mass=0.1, ls=6, m5=1.8, b=1.5, c=0.5)
    x = np.zeros(D.f_size)
    r = D.InvCg(x, G[tag + "_src"], stop_rsd=1e-10, max_num_iter=2000, precision=prec)
    assert r.status == A.CONVERGED and r.true_res <= 1e-10
    assert rel(x, G[tag + "_sol"]) < 1e-9
    if prec == A.DOUBLE:
        assert r.iterations == int(G[tag + "_iters"])
        assert abs(r.true_res - float(G[tag + "_true_res"])) <= 1e-2 * float(G[tag + "_true_res"]) + 5e-12


def test_minvcg(G, lat):
    D = DiracOpWilson(lat, mass=0.1)
    chi, shifts = G["ms_chi"], list(G["ms_shifts"])
    psi = [np.zeros_like(chi) for _ in shifts]
    rs = np.full(len(shifts), 1e-10)
    k = D.MInvCG(psi, chi, float(chi @ chi), shifts, rs, type=A.MS_MULTI)
    assert k == int(G["ms_iters"])
    for s in range(len(shifts)):
        assert rel(psi[s], G["ms_psi"][s]) < 1e-9
    assert np.allclose(rs, G["ms_rsd"], rtol=1e-2, atol=0)
