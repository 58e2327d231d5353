"""The oracle's solvers against the golden fixture the reference's own
solvers produced (tests/golden/ref_solvers.npz): the CPU check that travels
to machines without the reference tree.  Same iteration counts and
solutions as the reference (tests/test_reference_solvers.py runs the
reference itself where it is built)."""
from pathlib import Path

import numpy as np
import pytest

from oracle import convert as CV
from tests.helpers import OracleOps, rel

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_solvers.npz"
L = (4, 4, 4, 4)
KAPPA = 1.0 / (2.0 * (0.1 + 4.0))


@pytest.fixture(scope="module")
def G():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def test_f_wilson_inv(oracle, G):
    ops = OracleOps(oracle, L, CV.gcanon_to_wilson(G["gauge"], L), ls=1)
    sol, it, tr = ops.matinv("wilson", CV.fcanon_to_wilson_4d(G["fwi_src"], L), kappa=KAPPA, stop_rsd=1e-12,
                             max_num_iter=500)
    assert it == int(G["fwi_iters"]) == 28
    assert rel(sol, CV.fcanon_to_wilson_4d(G["fwi_sol"], L)) < 1e-10


@pytest.mark.parametrize("kind,tag", [("dwf", "dwf"), ("mobius", "mob")])
def test_5d_invcg(oracle, G, kind, tag):
    ops = OracleOps(oracle, L, CV.gcanon_to_wilson(G["gauge"], L), ls=6, m5=1.8, b=1.5, c=0.5)
    sol, it, tr = ops.invcg(kind, G[tag + "_src"], mass=0.1, stop_rsd=1e-10, max_num_iter=2000)
    assert it == int(G[tag + "_iters"])
    assert rel(sol, G[tag + "_sol"]) < 1e-9


def test_minvcg(oracle, G):
    ops = OracleOps(oracle, L, CV.gcanon_to_wilson(G["gauge"], L), ls=1)
    psi, k, rs = ops.minvcg("wilson", G["ms_chi"], list(G["ms_shifts"]), [1e-10] * 4, kappa=KAPPA, type=1,
                            max_num_iter=2000)
    assert k == int(G["ms_iters"])
    for s in range(4):
        assert rel(psi[s], G["ms_psi"][s]) < 1e-9
