"""Test infrastructure only: runs the reference's own Lattice / DiracOp
solvers (oracle/_ref/libcpsref_solve.so, built by ``make -C oracle refsolve``)
in a child process, one geometry per process (the reference keeps a single
static gauge field, lattice_base.C:56, 320-325).

    python -m oracle.refsolve SPEC.json OUT.npz

SPEC keys: L (4 ints), ls, kind ("wilson" | "dwf" | "mobius"), m5, a5_inv,
b, c, bc_t, backend, pc_type (the Mobius preconditioning, dwf.h:42-48;
default SYM2), task, and per task:

* ``fwilsoninv``: the steps of the reference's tests/f_wilson_inv/main.C on
  its own disordered start and RandGaussVector source (mass, stop_rsd,
  max_iter): DiracOpWilson::MatInv on both checkerboards;
* ``invcg``: DiracOp::InvCgShift on one checkerboard (gauge: a CANONICAL
  gauge .npy, or "disord" for the reference's own disordered start; src: a
  .npy; mass, stop_rsd, max_iter, shift);
* ``minvcg``: DiracOp::MInvCG (gauge, src, shifts, rsd, type, mass,
  max_iter);
* ``ops``: Mat, MatDag (not Mobius: the reference's stops with an error),
  MatHerm on the full vector src, and for Mobius MatPcDagMatPcShift
  (eigen_shift mu) on its first half (gauge, src, mass, mu);
* ``pcops``: MatPc and MatPcDag of the checkerboard vector src (gauge, src,
  mass);
* ``matinv``: DiracOp*::MatInv on the full vector src (both checkerboards,
  the DiracOp's order), zero initial guess (gauge, src, mass, stop_rsd,
  max_iter);
* ``cgtime``: wall time of DiracOp::InvCgShift capped at each max_iter of
  ``caps`` (zero initial guess each time, after ``warmup`` untimed capped
  runs), on the source MatPcDag(src) (gauge, src, mass, stop_rsd).

``backend`` "gpu" loads oracle/_ref/libcpsref_gpu.so (``make -C oracle
refgpu``) instead: the same reference code with DiracOp::InvCgShift replaced
by the library's CPS-side shim (cps_veloc_b200/shim/dirac_op_gpu.C), so every
solve above runs the reference's own drivers (MatInv, InvCg) around the GPU
CG.  CPSGPU_INNER in the environment selects its precision.

OUT holds the iteration count, true residual, solution(s), the inputs and
``res_hist``, the |r|^2 of every iteration as the reference prints it
(inv_cg.C:352-353), read back from its standard output.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import re
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SOLVE_SO = HERE / "_ref" / "libcpsref_solve.so"
GPU_SO = HERE / "_ref" / "libcpsref_gpu.so"
KINDS = {"wilson": 0, "dwf": 1, "mobius": 2}
_dp = C.POINTER(C.c_double)


def available(backend: str = "cpu") -> bool:
    return (GPU_SO if backend == "gpu" else SOLVE_SO).exists()


def _p(a):
    return a.ctypes.data_as(_dp)


def _lib(backend: str = "cpu"):
    L = C.CDLL(str(GPU_SO if backend == "gpu" else SOLVE_SO))
    L.rs_init.argtypes = [C.c_int] * 6 + [C.c_double] * 4 + [C.c_int] * 3
    L.rs_vol.restype = C.c_long
    L.rs_rand_gauss.argtypes = [_dp, C.c_double]
    L.rs_fconvert.argtypes = [_dp, C.c_int, C.c_int]
    L.rs_get_gauge.argtypes = [_dp]
    L.rs_set_gauge.argtypes = [_dp]
    L.rs_invcg.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_int, C.c_double, _dp]
    L.rs_matinv.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_int, _dp]
    L.rs_matpc_dag_matpc.argtypes = [_dp, _dp, C.c_double, _dp]
    L.rs_matpc_dag.argtypes = [_dp, _dp, C.c_double]
    L.rs_matpc.argtypes = [_dp, _dp, C.c_double]
    L.rs_set_pc_type.argtypes = [C.c_int]
    L.rs_mat.argtypes = [_dp, _dp, C.c_double, C.c_int]
    L.rs_matherm.argtypes = [_dp, _dp, C.c_double]
    L.rs_mdagm_shift.argtypes = [_dp, _dp, C.c_double, C.c_double, _dp]
    L.rs_minvcg.argtypes = [C.POINTER(_dp), _dp, C.c_double, _dp, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_double,
                            C.c_int]
    return L


class _Stdout:
    """capture the C library's standard output (fd 1) into a string"""

    def __enter__(self):
        sys.stdout.flush()
        self.tmp = tempfile.TemporaryFile(mode="w+b")
        self.saved = os.dup(1)
        os.dup2(self.tmp.fileno(), 1)
        return self

    def __exit__(self, *a):
        libc = C.CDLL(None)
        libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        self.tmp.seek(0)
        self.text = self.tmp.read().decode(errors="replace")
        self.tmp.close()


def _hist(text: str) -> np.ndarray:
    return np.array([float(m.group(2)) for m in re.finditer(r"\|res\[(\d+)\]\|\^2 = ([-+0-9.eE]+)", text)])


def run(spec: dict) -> dict:
    L = _lib(spec.get("backend", "cpu"))
    lx, ly, lz, lt = spec["L"]
    kind = KINDS[spec.get("kind", "wilson")]
    ls = int(spec.get("ls", 0))
    start_disord = 1 if (spec["task"] == "fwilsoninv" or spec.get("gauge") == "disord") else 0
    if L.rs_init(lx, ly, lz, lt, ls, kind, spec.get("m5", 1.8), spec.get("a5_inv", 1.0), spec.get("b", 1.0),
                 spec.get("c", 0.0), spec.get("bc_t", -1), start_disord, 1) != 0:
        raise RuntimeError("rs_init failed")
    vol = L.rs_vol()
    fsite = 24 * (ls if kind else 1)
    out = {}
    if not start_disord:
        u = np.ascontiguousarray(np.load(spec["gauge"]), dtype=np.float64)
        L.rs_set_gauge(_p(u))
    else:
        u = np.zeros(vol * 72)
        L.rs_get_gauge(_p(u))
    out["gauge"] = u
    if "pc_type" in spec:
        L.rs_set_pc_type(int(spec["pc_type"]))
    tr = C.c_double()
    with _Stdout() as cap:
        if spec["task"] == "fwilsoninv":
            x_in = np.zeros(vol * fsite)
            L.rs_rand_gauss(_p(x_in), 1.0)
            src_canonical = x_in.copy()
            sol = np.zeros(vol * fsite)
            L.rs_fconvert(_p(sol), 2, 0)
            L.rs_fconvert(_p(x_in), 2, 0)
            it = L.rs_matinv(_p(sol), _p(x_in), spec["mass"], spec["stop_rsd"], spec["max_iter"], C.byref(tr))
            L.rs_fconvert(_p(sol), 0, 2)
            out.update(src=src_canonical, sol=sol)
        elif spec["task"] == "invcg":
            src = np.ascontiguousarray(np.load(spec["src"]), dtype=np.float64)
            sol = np.zeros_like(src)
            it = L.rs_invcg(_p(sol), _p(src), spec["mass"], spec["stop_rsd"], spec["max_iter"],
                            spec.get("shift", 0.0), C.byref(tr))
            out.update(sol=sol)
        elif spec["task"] == "pcops":
            src = np.ascontiguousarray(np.load(spec["src"]), dtype=np.float64)
            mp, md = np.zeros_like(src), np.zeros_like(src)
            L.rs_matpc(_p(mp), _p(src.copy()), spec["mass"])
            L.rs_matpc_dag(_p(md), _p(src.copy()), spec["mass"])
            out.update(matpc=mp, matpcdag=md)
            it = 0
        elif spec["task"] == "matinv":
            src = np.ascontiguousarray(np.load(spec["src"]), dtype=np.float64)
            sol = np.zeros_like(src)
            it = L.rs_matinv(_p(sol), _p(src.copy()), spec["mass"], spec["stop_rsd"], spec["max_iter"], C.byref(tr))
            out.update(sol=sol)
        elif spec["task"] == "minvcg":
            src = np.ascontiguousarray(np.load(spec["src"]), dtype=np.float64)
            sh = np.ascontiguousarray(spec["shifts"], dtype=np.float64)
            n = len(sh)
            typ = int(spec.get("type", 1))
            npsi = 1 if typ == 0 else n
            psi = [np.zeros_like(src) for _ in range(npsi)]
            arr = (_dp * npsi)(*[_p(x) for x in psi])
            rsd = np.ascontiguousarray(spec["rsd"], dtype=np.float64).copy()
            alpha = np.ascontiguousarray(spec.get("alpha", [1.0] * n), dtype=np.float64)
            it = L.rs_minvcg(arr, _p(src), float(src @ src), _p(sh), n, int(spec.get("isz", 0)), _p(rsd), typ,
                             _p(alpha), spec["mass"], spec["max_iter"])
            out.update(psi=np.array(psi), rsd_out=rsd)
        elif spec["task"] == "cgtime":
            import time
            w = np.ascontiguousarray(np.load(spec["src"]), dtype=np.float64)
            src = np.zeros_like(w)
            L.rs_matpc_dag(_p(src), _p(w), spec["mass"])
            times, iters = [], []
            caps = [int(c) for c in spec["caps"]]
            for k in range(int(spec.get("warmup", 0)) + len(caps)):
                limit = caps[0] if k < int(spec.get("warmup", 0)) else caps[k - int(spec.get("warmup", 0))]
                sol = np.zeros_like(src)
                t0 = time.perf_counter()
                it = L.rs_invcg(_p(sol), _p(src), spec["mass"], spec["stop_rsd"], limit, 0.0, C.byref(tr))
                dt = time.perf_counter() - t0
                if k >= int(spec.get("warmup", 0)):
                    times.append(dt)
                    iters.append(it)
            out.update(times=np.array(times), caps_iters=np.array(iters))
        elif spec["task"] == "ops":
            full = np.ascontiguousarray(np.load(spec["src"]), dtype=np.float64)
            res = {}
            for dag in ((0,) if kind == 2 else (0, 1)):
                o = np.zeros_like(full)
                L.rs_mat(_p(o), _p(full.copy()), spec["mass"], dag)
                res["matdag" if dag else "mat"] = o
            o = np.zeros_like(full)
            L.rs_matherm(_p(o), _p(full.copy()), spec["mass"])
            res["matherm"] = o
            if kind == 2:
                half = np.ascontiguousarray(full[:full.size // 2])
                o = np.zeros_like(half)
                d = C.c_double()
                L.rs_mdagm_shift(_p(o), _p(half.copy()), spec["mass"], spec.get("mu", 0.3), C.byref(d))
                res.update(shift=o, shift_dot=d.value)
            out.update(res)
            it = 0
        else:
            raise ValueError(spec["task"])
    out.update(iters=it, true_res=tr.value, res_hist=_hist(cap.text))
    return out


def run_child(spec: dict, timeout: float = 600, env: dict | None = None) -> dict:
    """run() in a fresh process (one reference geometry per process); env:
    extra environment variables of the child"""
    with tempfile.TemporaryDirectory() as d:
        sp, op = Path(d) / "spec.json", Path(d) / "out.npz"
        sp.write_text(json.dumps(spec))
        # the reference writes its error logs (phys.error.*) into the working directory
        env = dict(os.environ) | (env or {})
        env["PYTHONPATH"] = str(HERE.parent) + os.pathsep + env.get("PYTHONPATH", "")
        r = subprocess.run([sys.executable, "-m", "oracle.refsolve", str(sp), str(op)], cwd=d, env=env,
                           capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference solver run failed:\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        with np.load(op) as z:
            return {k: z[k] for k in z.files}


if __name__ == "__main__":
    spec = json.loads(Path(sys.argv[1]).read_text())
    res = run(spec)
    np.savez(sys.argv[2], **res)
