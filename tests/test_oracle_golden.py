"""The oracle restatement against golden vectors made by the reference's own
kernels (tests/golden/make_golden.py).  Bit-level agreement is not expected
(summation order differs); FP64 agreement to 1e-13 relative is required."""
from pathlib import Path

import numpy as np
import pytest

from helpers import OracleOps, rel

GOLD = Path(__file__).resolve().parent / "golden" / "ref_kernels.npz"
TOL = 1e-13


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("name", ["w44", "w2468"])
def test_wilson_golden(oracle, gold, name):
    L = tuple(int(x) for x in gold[f"{name}_L"])
    ops = OracleOps(oracle, L, gold[f"{name}_u"], ls=1)
    psi = gold[f"{name}_psi"]
    for cb in (0, 1):
        for dag in (0, 1):
            assert rel(ops.wilson_dslash(psi, cb, dag), gold[f"{name}_dslash_{cb}{dag}"]) < TOL
    y, d = ops.wilson_mdagm(psi, 0.12)
    assert rel(y, gold[f"{name}_mdagm"]) < TOL
    assert abs(d / float(gold[f"{name}_mdagm_dot"]) - 1) < TOL
    for dag in (0, 1):
        assert rel(ops.wilson_m(psi, 0.12, dag), gold[f"{name}_m_{dag}"]) < TOL


@pytest.mark.parametrize("name", ["d4", "d2"])
def test_dwf_mobius_golden(oracle, gold, name):
    L = tuple(int(x) for x in gold[f"{name}_L"])
    ls = int(gold[f"{name}_ls"])
    mass = float(gold["mass"])
    ops = OracleOps(oracle, L, gold[f"{name}_u"], ls=ls)
    psi = gold[f"{name}_psi"]
    for cb in (0, 1):
        for dag in (0, 1):
            assert rel(ops.dwf_dslash(psi, mass, cb, dag), gold[f"{name}_dwf_dslash_{cb}{dag}"]) < TOL
            assert rel(ops.mobius_dslash_4(psi, mass, cb, dag), gold[f"{name}_mob_dslash4_{cb}{dag}"]) < TOL
    y, d = ops.dwf_mdagm(psi, mass)
    assert rel(y, gold[f"{name}_dwf_mdagm"]) < TOL
    assert abs(d / float(gold[f"{name}_dwf_mdagm_dot"]) - 1) < TOL
    for dag in (0, 1):
        assert rel(ops.mobius_m5inv(psi, mass, dag), gold[f"{name}_mob_m5inv_{dag}"]) < TOL
        assert rel(ops.mobius_m(psi, mass, dag), gold[f"{name}_mob_m_{dag}"]) < TOL
    y, d = ops.mobius_mdagm(psi, mass)
    assert rel(y, gold[f"{name}_mob_mdagm"]) < TOL
    assert abs(d / float(gold[f"{name}_mob_mdagm_dot"]) - 1) < TOL
