"""Generate the solver golden fixtures from the reference's own solvers.

Runs the reference's Lattice / DiracOp classes and Krylov solvers (compiled
unchanged from the reference sources by ``make -C oracle refsolve``) in
child processes (oracle/refsolve.py) and stores inputs and outputs in
``tests/golden/ref_solvers.npz``, so that GPU tests can compare the
library's solvers with the reference on machines without the reference
tree.  The gauge field ("gauge") is the reference's own fixed-seed
disordered start of the 4^4 lattice, shared by every case, in CANONICAL
order without boundary signs.  Re-run only when the fixture set
changes:

    python tests/golden/make_golden_solvers.py

Cases:
  fwi_*  tests/f_wilson_inv/main.C: 4^4 Wilson, m = 0.1, its RandGaussVector
         source, DiracOpWilson::MatInv to stop_rsd 1e-12 (CANONICAL fields);
  dwf_*  DiracOpDwf InvCg, 4^4 x Ls 6, M5 1.8, m_f 0.1, stop_rsd 1e-10;
  mob_*  DiracOpMobius InvCg, 4^4 x Ls 6, b 1.5, c 0.5, M5 1.8, m_f 0.1;
  ms_*   DiracOpWilson::MInvCG, 4^4, m = 0.1, four shifts, MULTI.
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refsolve  # noqa: E402

OUT = Path(__file__).resolve().parent / "ref_solvers.npz"


def main():
    data = {}
    r = refsolve.run_child({"L": [4, 4, 4, 4], "kind": "wilson", "task": "fwilsoninv", "mass": 0.1,
                            "stop_rsd": 1e-12, "max_iter": 500})
    gauge = r["gauge"]
    data["gauge"] = gauge  # the same fixed-seed start in every case (checked below)
    for k in ("src", "sol", "iters", "true_res", "res_hist"):
        data["fwi_" + k] = r[k]
    with tempfile.TemporaryDirectory() as d:
        for tag, kind, extra in (("dwf", "dwf", {"m5": 1.8}), ("mob", "mobius", {"m5": 1.8, "b": 1.5, "c": 0.5})):
            n = 24 * 6 * 4 ** 4 // 2
            src = np.random.default_rng(31 if kind == "dwf" else 32).normal(size=n)
            np.save(Path(d) / "src.npy", src)
            r = refsolve.run_child({"L": [4, 4, 4, 4], "ls": 6, "kind": kind, "task": "invcg", "gauge": "disord",
                                    "src": str(Path(d) / "src.npy"), "mass": 0.1, "stop_rsd": 1e-10,
                                    "max_iter": 2000} | extra)
            data[tag + "_src"] = src
            assert np.array_equal(r["gauge"], gauge)
            for k in ("sol", "iters", "true_res", "res_hist"):
                data[tag + "_" + k] = r[k]
        chi = np.random.default_rng(33).normal(size=24 * 4 ** 4 // 2)
        np.save(Path(d) / "chi.npy", chi)
        shifts = [0.0005, 0.01, 0.2, 1.5]
        r = refsolve.run_child({"L": [4, 4, 4, 4], "kind": "wilson", "task": "minvcg", "gauge": "disord",
                                "src": str(Path(d) / "chi.npy"), "mass": 0.1, "shifts": shifts,
                                "rsd": [1e-10] * 4, "type": 1, "max_iter": 2000})
        assert np.array_equal(r["gauge"], gauge)
        data.update(ms_chi=chi, ms_shifts=np.array(shifts), ms_psi=r["psi"],
                    ms_iters=r["iters"], ms_rsd=r["rsd_out"])
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT}: " + ", ".join(f"{k}{list(np.shape(v))}" for k, v in data.items()))


if __name__ == "__main__":
    main()
