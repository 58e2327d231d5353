"""The reference's own solver drivers running on the GPU through the CPS-side
shim (cps_veloc_b200/shim/dirac_op_gpu.C).

oracle/_ref/libcpsref_gpu.so is the reference's Lattice / DiracOp code
compiled unchanged with DiracOp::InvCgShift (inv_cg.C:84-448) replaced by
the shim, which solves through the C ABI (cpsgpu_invcg).  The same reference
entry points then run once on the CPU (libcpsref_solve.so) and once with the
GPU CG:

* the f_wilson_inv test (tests/f_wilson_inv/main.C: DiracOpWilson::MatInv,
  4^4, m = 0.1, stop_rsd 1e-12): 28 iterations
  (tests/f_wilson_inv/qcdlinux1.log:69) and the CPU reference's solution;
* DiracOp::InvCgShift for DWF and Mobius, with and without a shift, and a
  capped iteration count: the CPU reference's iteration counts and solutions;
* a mixed-precision inner solve (CPSGPU_INNER=single) reaching the CPU
  reference's solution.
"""
import numpy as np
import pytest

from oracle import refsolve
from helpers import rel

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (refsolve.available("gpu") and refsolve.available("cpu")),
                                 reason="reference + shim not built (make -C oracle refsolve refgpu)")]

F_WILSON_INV_ITERS = 28  # tests/f_wilson_inv/qcdlinux1.log:69


def test_f_wilson_inv_through_the_shim():
    spec = {"L": [4, 4, 4, 4], "kind": "wilson", "task": "fwilsoninv", "mass": 0.1, "stop_rsd": 1e-12,
            "max_iter": 500}
    cpu = refsolve.run_child(spec)
    gpu = refsolve.run_child(spec | {"backend": "gpu"})
    assert int(cpu["iters"]) == int(gpu["iters"]) == F_WILSON_INV_ITERS
    assert gpu["true_res"] < 1e-12
    np.testing.assert_array_equal(cpu["src"], gpu["src"])
    assert rel(gpu["sol"], cpu["sol"]) < 1e-10


CASES = [
    ("dwf", [4, 4, 4, 8], 8, 0.04, {"m5": 1.7}),
    ("mobius", [4, 4, 4, 4], 6, 0.1, {"m5": 1.8, "b": 1.5, "c": 0.5}),
]


@pytest.mark.parametrize("kind,L,ls,mass,extra", CASES)
@pytest.mark.parametrize("shift,max_iter,stop", [(0.0, 2000, 1e-10), (0.25, 2000, 1e-10), (0.0, 12, 1e-14)])
def test_invcg_through_the_shim(tmp_path, kind, L, ls, mass, extra, shift, max_iter, stop):
    n = 24 * ls * int(np.prod(L)) // 2
    np.save(tmp_path / "src.npy", np.random.default_rng(3).normal(size=n))
    spec = {"L": L, "ls": ls, "kind": kind, "task": "invcg", "gauge": "disord", "src": str(tmp_path / "src.npy"),
            "mass": mass, "stop_rsd": stop, "max_iter": max_iter, "shift": shift} | extra
    cpu = refsolve.run_child(spec)
    gpu = refsolve.run_child(spec | {"backend": "gpu"})
    if kind == "mobius" and max_iter > 100:
        # the GPU applies the Mobius M5^-1 chain as one dense Ls x Ls matrix, the
        # reference as its recursion (zmobius_m5inv.C): the late |r|^2 of a
        # 170-iteration solve differ by a few percent, and a stop test that
        # falls between them moves by one iteration
        assert abs(int(gpu["iters"]) - int(cpu["iters"])) <= 1
    else:
        assert int(gpu["iters"]) == int(cpu["iters"])
    # a capped solve stops at the same iterate; a converged one within its tolerance
    assert rel(gpu["sol"], cpu["sol"]) < (1e-11 if max_iter < 100 else 1e-9)
    if int(gpu["iters"]) == int(cpu["iters"]):
        assert abs(gpu["true_res"] - cpu["true_res"]) <= 1e-2 * cpu["true_res"] + 5e-12
    else:
        assert gpu["true_res"] <= 1.5 * stop


def test_mixed_inner_through_the_shim(tmp_path):
    kind, L, ls, mass, extra = CASES[0]
    n = 24 * ls * int(np.prod(L)) // 2
    np.save(tmp_path / "src.npy", np.random.default_rng(4).normal(size=n))
    spec = {"L": L, "ls": ls, "kind": kind, "task": "invcg", "gauge": "disord", "src": str(tmp_path / "src.npy"),
            "mass": mass, "stop_rsd": 1e-10, "max_iter": 2000} | extra
    cpu = refsolve.run_child(spec)
    gpu = refsolve.run_child(spec | {"backend": "gpu"}, env={"CPSGPU_INNER": "single"})
    assert gpu["true_res"] <= 1e-10
    assert rel(gpu["sol"], cpu["sol"]) < 1e-8
    # reliable updates add a few iterations at most
    assert int(cpu["iters"]) <= int(gpu["iters"]) <= int(cpu["iters"]) * 1.15 + 5


@pytest.mark.parametrize("kind,L,ls,mass,extra", CASES)
@pytest.mark.parametrize("inner", [None, "single"])
def test_minvcg_through_the_shim(tmp_path, kind, L, ls, mass, extra, inner):
    """DiracOp::MInvCG (minvcg.C:47-353) of the reference's own DiracOp with
    the shim's multishift (cpsgpu_minvcg) against the CPU reference, type
    MULTI: in FP64 the same iteration count and solutions; with the FP32
    recurrences and the FP64 refinement of every shift (CPSGPU_INNER=single)
    the same solutions within the refinement's residual."""
    n = 24 * ls * int(np.prod(L)) // 2
    np.save(tmp_path / "src.npy", np.random.default_rng(5).normal(size=n))
    shifts = [0.01, 0.1, 0.5]
    spec = {"L": L, "ls": ls, "kind": kind, "task": "minvcg", "gauge": "disord", "src": str(tmp_path / "src.npy"),
            "mass": mass, "max_iter": 5000, "shifts": shifts, "rsd": [1e-10] * 3, "type": 1} | extra
    cpu = refsolve.run_child(spec)
    gpu = refsolve.run_child(spec | {"backend": "gpu"}, env={"CPSGPU_INNER": inner} if inner else None)
    for k in range(len(shifts)):
        assert rel(gpu["psi"][k], cpu["psi"][k]) < (1e-9 if inner is None else 1e-8)
    if inner is None:
        # the Mobius M5^-1 as one dense matrix against the reference's recursion
        assert abs(int(gpu["iters"]) - int(cpu["iters"])) <= (1 if kind == "mobius" else 0)
