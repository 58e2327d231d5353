"""The oracle's Krylov solvers pinned to the reference's own.

The reference's Lattice / DiracOp classes and their solvers are compiled
unchanged from its sources (oracle/Makefile, target refsolve) and run in a
child process per geometry (oracle/refsolve.py).  These CPU tests check:

* the compiled reference reproduces its published f_wilson_inv test:
  28 CG iterations (tests/f_wilson_inv/qcdlinux1.log:69) to a true residual
  below the 1e-12 stopping residual;
* the oracle's MatInv / InvCg (orc_wilson_matinv, orc_invcg: inv_cg.C:84-448)
  take the reference's iteration count and reach its solution on Wilson,
  DWF and Mobius systems (the reference's own disordered gauge start);
* the oracle's multishift CG (orc_minvcg: minvcg.C:47-353) takes the
  reference's iteration count and returns its solutions and residuals.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import convert as CV
from oracle import refsolve
from tests.helpers import OracleOps, rel

pytestmark = pytest.mark.skipif(not refsolve.available(),
                                reason="reference solver library not built (make -C oracle refsolve)")

# tests/f_wilson_inv/main.C: 4^4, m = 0.1, stop_rsd = 1e-12, max_num_iter = 500
F_WILSON_INV_ITERS = 28  # tests/f_wilson_inv/qcdlinux1.log:69


def kappa_of(mass):
    return 1.0 / (2.0 * (mass + 4.0))  # d_op_wilson.C:134-136


def test_reference_reproduces_f_wilson_inv(oracle):
    L = (4, 4, 4, 4)
    r = refsolve.run_child({"L": list(L), "kind": "wilson", "task": "fwilsoninv", "mass": 0.1,
                            "stop_rsd": 1e-12, "max_iter": 500})
    assert int(r["iters"]) == F_WILSON_INV_ITERS
    assert r["true_res"] < 1e-12
    assert len(r["res_hist"]) == F_WILSON_INV_ITERS
    # the oracle's MatInv on the same gauge field and source
    u = CV.gcanon_to_wilson(r["gauge"], L)
    src = CV.fcanon_to_wilson_4d(r["src"], L)
    ops = OracleOps(oracle, L, u, ls=1)
    sol, it, tr = ops.matinv("wilson", src, kappa=kappa_of(0.1), stop_rsd=1e-12, max_num_iter=500)
    assert it == F_WILSON_INV_ITERS
    assert rel(sol, CV.fcanon_to_wilson_4d(r["sol"], L)) < 1e-10


CASES = [
    ("wilson", (4, 4, 4, 4), 0, 0.1, {}),
    ("wilson", (4, 4, 4, 8), 0, 0.05, {}),
    ("dwf", (4, 4, 4, 4), 6, 0.1, {"m5": 1.8}),
    ("dwf", (4, 4, 4, 8), 8, 0.04, {"m5": 1.7}),
    ("mobius", (4, 4, 4, 4), 6, 0.1, {"m5": 1.8, "b": 1.5, "c": 0.5}),
]


def _invcg_ref(tmp_path, kind, L, ls, mass, extra, stop_rsd, max_iter=2000, shift=0.0, seed=11):
    n = 24 * max(ls, 1) * int(np.prod(L)) // 2
    src = np.random.default_rng(seed).normal(size=n)
    np.save(tmp_path / "src.npy", src)
    spec = {"L": list(L), "ls": ls, "kind": kind, "task": "invcg", "gauge": "disord", "src": str(tmp_path / "src.npy"),
            "mass": mass, "stop_rsd": stop_rsd, "max_iter": max_iter, "shift": shift} | extra
    return src, refsolve.run_child(spec)


def _ops(oracle, kind, L, ls, gauge, extra):
    u = CV.gcanon_to_wilson(gauge, L)
    return OracleOps(oracle, L, u, ls=max(ls, 1), m5=extra.get("m5", 1.8), b=extra.get("b", 1.5),
                     c=extra.get("c", 0.5))


@pytest.mark.parametrize("kind,L,ls,mass,extra", CASES)
def test_oracle_invcg_matches_reference(oracle, tmp_path, kind, L, ls, mass, extra):
    src, r = _invcg_ref(tmp_path, kind, L, ls, mass, extra, 1e-10)
    ops = _ops(oracle, kind, L, ls, r["gauge"], extra)
    sol, it, tr = ops.invcg(kind, src, mass=mass, kappa=kappa_of(mass), stop_rsd=1e-10, max_num_iter=2000)
    assert it == int(r["iters"]), (it, int(r["iters"]))
    # the true residual of a 1e-10 solve carries rounding noise of ~1e-13 in either code
    assert abs(tr - float(r["true_res"])) <= 1e-2 * float(r["true_res"]) + 5e-12
    assert rel(sol, r["sol"]) < 1e-9


@pytest.mark.parametrize("kind,L,ls,mass,extra", [CASES[0], CASES[2]])
def test_oracle_invcg_fixed_iterations_and_shift(oracle, tmp_path, kind, L, ls, mass, extra):
    """max_num_iter caps the loop at max_num_iter - 1 iterations and returns
    itr + 1 (inv_cg.C:275, :446); the shifted system (H + shift) as
    InvCgShift applies it"""
    src, r = _invcg_ref(tmp_path, kind, L, ls, mass, extra, 1e-14, max_iter=12, shift=0.25)
    ops = _ops(oracle, kind, L, ls, r["gauge"], extra)
    sol, it, tr = ops.invcg(kind, src, mass=mass, kappa=kappa_of(mass), stop_rsd=1e-14, max_num_iter=12,
                            shift=0.25)
    assert it == int(r["iters"])
    assert rel(sol, r["sol"]) < 1e-11
    assert abs(tr - float(r["true_res"])) <= 1e-8 * float(r["true_res"])


@pytest.mark.parametrize("kind,L,ls,mass,extra", [CASES[0], CASES[2], CASES[4]])
def test_oracle_minvcg_matches_reference(oracle, tmp_path, kind, L, ls, mass, extra):
    n = 24 * max(ls, 1) * int(np.prod(L)) // 2
    chi = np.random.default_rng(5).normal(size=n)
    np.save(tmp_path / "chi.npy", chi)
    shifts = [0.0005, 0.01, 0.2, 1.5]
    rsd = [1e-9] * len(shifts)
    spec = {"L": list(L), "ls": ls, "kind": kind, "task": "minvcg", "gauge": "disord", "src": str(tmp_path / "chi.npy"),
            "mass": mass, "shifts": shifts, "rsd": rsd, "type": 1, "max_iter": 2000} | extra
    r = refsolve.run_child(spec)
    ops = _ops(oracle, kind, L, ls, r["gauge"], extra)
    psi, k, rs = ops.minvcg(kind, chi, shifts, rsd, mass=mass, kappa=kappa_of(mass), type=1, max_num_iter=2000)
    assert k == int(r["iters"]), (k, int(r["iters"]))
    for s in range(len(shifts)):
        assert rel(psi[s], r["psi"][s]) < 1e-9
    # the achieved residuals come out of the shifted recurrences: rounding-level agreement
    assert np.allclose(rs, r["rsd_out"], rtol=1e-2, atol=0)
