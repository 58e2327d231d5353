"""The unpreconditioned operators, the shifted Mobius MatPcDagMatPc and the
fifth-direction spacing a5 of the oracle, pinned to the reference's own
code (compiled from its sources, oracle/_ref):

* DiracOpWilson / DiracOpDwf / DiracOpMobius Mat, MatDag and MatHerm
  (d_op_wilson.C:362-443, d_op_dwf.C:541-660, d_op_mobius.C:735-942; the
  reference's Mobius MatDag stops with an error and is not compared) and
  DiracOpMobius::MatPcDagMatPcShift (d_op_mobius.C:235, zmobius_mdagm.C
  :79-135), through the reference's Lattice / DiracOp classes;
* dwf_dslash, dwf_mdagm, zmobius_m5inv and zmobius_mdagm with
  DoArg.dwf_a5_inv != 1 (dwf_dslash_5_plus_omp.C:137-138, dwf_init.C:97-98,
  d_op_mobius.C:105-108), through the reference's kernels.
The reference's Lattice classes stop with a segmentation fault on odd Ls
(GwilsonFdwf, in this build), so the DiracOp comparisons use even Ls; the
kernel comparisons cover odd Ls.
"""
import ctypes as C
import tempfile
from pathlib import Path

import numpy as np
import pytest

from oracle import convert as CV
from oracle import refsolve
from oracle.loader import apply_bc_signs, p
from tests.helpers import OracleOps, rel, vh_of

TOL = 1e-13


def kappa_of(mass):
    return 1.0 / (2.0 * (mass + 4.0))


@pytest.mark.skipif(not refsolve.available(), reason="reference solver library not built")
@pytest.mark.parametrize("kind,L,ls,a5", [("wilson", (4, 4, 4, 4), 0, 1.0), ("dwf", (4, 4, 4, 4), 6, 1.0),
                                          ("dwf", (4, 4, 2, 4), 4, 0.8), ("mobius", (4, 4, 4, 4), 6, 1.0),
                                          ("mobius", (4, 2, 4, 4), 4, 1.25)])
def test_full_operators_vs_reference(oracle, kind, L, ls, a5):
    mass, extra = 0.1, {"m5": 1.8, "b": 1.5, "c": 0.5, "a5_inv": a5}
    n = 2 * 24 * max(ls, 1) * vh_of(L)
    x = np.random.default_rng(3).normal(size=n)
    with tempfile.TemporaryDirectory() as d:
        np.save(Path(d) / "x.npy", x)
        r = refsolve.run_child({"L": list(L), "ls": ls, "kind": kind, "task": "ops", "gauge": "disord",
                                "src": str(Path(d) / "x.npy"), "mass": mass, "mu": 0.3} | extra)
    ops = OracleOps(oracle, L, CV.gcanon_to_wilson(r["gauge"], L), ls=max(ls, 1), m5=1.8, b=1.5, c=0.5, a5_inv=a5)
    k = kappa_of(mass)
    assert rel(ops.mat(kind, x, mass, k, 0), r["mat"]) < TOL
    if kind != "mobius":
        assert rel(ops.mat(kind, x, mass, k, 1), r["matdag"]) < TOL
    assert rel(ops.matherm(kind, x, mass, k), r["matherm"]) < TOL
    if kind == "mobius":
        y, dot = ops.mobius_mdagm_shift(x[:n // 2], mass, 0.3)
        assert rel(y, r["shift"]) < TOL
        assert abs(dot / float(r["shift_dot"]) - 1) < TOL


@pytest.mark.parametrize("L,ls,a5", [((4, 4, 4, 4), 4, 0.8), ((2, 4, 2, 4), 5, 1.5)])
def test_dwf_and_mobius_a5_vs_reference_kernels(oracle, reference, L, ls, a5):
    from cps_veloc_b200.dirac import gen_gauge, gen_gaussian

    bc, mass = (1, 1, 1, -1), 0.05
    reference.ref_init_a5(*L, ls, 1.8, 1.5, 0.5, bc[3], a5)
    u = gen_gauge(L, seed=21)
    us = apply_bc_signs(u, L, bc)
    ops = OracleOps(oracle, L, u, ls=ls, bc=bc, m5=1.8, b=1.5, c=0.5, a5_inv=a5)
    psi = gen_gaussian(24 * ls * vh_of(L), seed=22)
    assert abs(reference.ref_dwf_kappa() - 1 / (2 * (4 + a5 - 1.8))) < 1e-15
    for cb, dag in ((0, 0), (1, 1)):
        y = np.zeros_like(psi)
        reference.ref_dwf_dslash(p(y), p(us), p(psi), mass, cb, dag)
        assert rel(ops.dwf_dslash(psi, mass, cb, dag), y) < TOL
    y = np.zeros_like(psi)
    d = C.c_double()
    reference.ref_dwf_mdagm(p(y), p(us), p(psi), C.byref(d), mass)
    yo, do = ops.dwf_mdagm(psi, mass)
    assert rel(yo, y) < TOL and abs(do / d.value - 1) < TOL
    y = psi.copy()
    reference.ref_zmobius_m5inv(p(y), mass, 0)
    assert rel(ops.mobius_m5inv(psi, mass, 0), y) < TOL
    y = np.zeros_like(psi)
    reference.ref_zmobius_mdagm(p(y), p(us), p(psi), C.byref(d), mass)
    yo, do = ops.mobius_mdagm(psi, mass)
    assert rel(yo, y) < TOL and abs(do / d.value - 1) < TOL
