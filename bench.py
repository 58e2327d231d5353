#!/usr/bin/env python3
"""Benchmark of the fermion-solve hot path on B200.

Workload (one step = one full solve from a zero initial guess):
  Shamir domain-wall fermions, 16^3 x 32 lattice, Ls = 16, M5 = 1.8,
  m_f = 0.01, periodic in space and antiperiodic in time; seeded SU(3) links
  U = exp(i 0.3 H); source = MatPcDag of a wall source built from a seeded
  Gaussian 4D field (upper chirality on s = 0, lower on s = Ls-1, the
  Ffour2five placement); CG on MatPcDagMatPc to a true residual of 1e-10.

Metric: time to a true residual of 1e-10 (seconds, lower is better) of the
mixed-precision CG (FP64 reliable updates and solution, FP32 inner iteration;
the FP16-storage inner solve is reported beside it), next to the plain FP64
CG of this library on the same
system, the dslash HBM bandwidth against the measured peak, the end-to-end
time through the host-pointer C ABI, and the reference's CPU code timed on a
bounded sample on this host: its DWF dslash on the GPU dslash's own input
(with the GPU result's relative error against it).

``--impl reference`` runs the reference's own DiracOpDwf::InvCg (compiled
unchanged, oracle/_ref) on the same system built by the numpy restatement of
the seeded generator (no library under test is loaded), capped at 1 and
1 + K iterations; seconds per iteration times the FP64 iteration count
gives its time to 1e-10.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 (under torchrun) every rank solves its own system (the same
lattice and operator, its own wall source) on its own GPU: N independent
solves, weak scaling (one solve does not shard without a halo exchange);
the reported time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "time to true residual 1e-10, mixed/batched vs FP64 CG on B200; dslash HBM GB/s"
L4 = (16, 16, 16, 32)
LS = 16
M5 = 1.8
MF = 0.01
SEED = 20261203
STOP = 1e-10
# Iterations of the plain FP64 CG to a true residual of 1e-10 on this
# workload, as measured by this library's FP64 CG on a B200 (196; it runs the
# reference's InvCgShift recurrence step for step, and on the reference's own
# systems it takes the reference's iteration count, tests/test_gpu_reference_
# solvers.py).  The CPU baselines use it to turn the reference's measured
# seconds per CG iteration into a time to solution without running the
# multi-hour CPU solve; the main arm reports the count it measures beside it.
FP64_CG_ITERS = 196
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# the dslash timed below on this workload, from single-launch ncu captures
# (hop_kernel store epilogue, cold L2; profiles/hop_dwf_*_16x32_ls16.md),
# keyed by (precision, stored link form, launch-shape class: several slices
# per block, one slice per block, or slice pairs per thread, as the autotuner
# may pick any of them; the re-read of links across blocks differs).  The
# algorithmic bytes are 226.5 MB (FP32, 12-real links), 239.0 MB (FP32, 18),
# 127.9 MB (FP16, 18).
DSLASH_TRAFFIC = {(1, 12, "multi"): 132.42e6 + 71.94e6, (1, 12, "one_slice"): 155.93e6 + 80.53e6,
                  (1, 12, "pair"): 132.99e6 + 74.12e6, (1, 18, "multi"): 145.61e6 + 78.76e6,
                  (2, 18, "multi"): 76.92e6 + 28.34e6}


def shape_class(shape) -> str:
    """the DSLASH_TRAFFIC class of a launch shape (sites, slices, slices per thread, order)"""
    if shape[2] == 2:
        return "pair"
    return "one_slice" if shape[1] == 1 else "multi"


WORKLOAD = "DWF 16^3x32 Ls=16 M5=1.8 mf=0.01 CG on MatPcDagMatPc to true residual 1e-10"


def workload_config() -> dict:
    """The config both arms report (the driver compares them key for key)."""
    return {"workload": WORKLOAD, "lattice": list(L4), "ls": LS, "m5": M5, "mf": MF,
            "bc": "periodic xyz, antiperiodic t", "gauge": f"U=exp(i 0.3 H), seed {SEED}",
            "source": "MatPcDag of a Gaussian wall source",
            "l2": "inputs larger than L2 (FP64 vectors 192 MiB; each solve streams GBs)"}


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self

        def rd():
            for line in self.proc.stdout:
                self.samples.append([x.strip() for x in line.split(",")])

        self.thread = threading.Thread(target=rd, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                mx = float(s[1])
                for k, n in enumerate(names):
                    if s[3 + k].lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def wall_source(L, ls, eta4d):
    """Ffour2five placement on the odd preconditioned checkerboard: slice 0
    holds the upper chirality of eta on the odd sites, slice Ls-1 the lower
    chirality on the 4D parity (Ls-1+1)%2 sites (f_dwf_base.C:961)."""
    vol = int(np.prod(L))
    vh = vol // 2
    src = np.zeros((ls, vh, 24))
    # eta4d: [parity][vh][24] in checkerboard order
    par0 = 1  # slice 0 on parity (0 + 1) % 2
    parl = (ls - 1 + 1) % 2
    src[0, :, :12] = eta4d[par0, :, :12]
    src[ls - 1, :, 12:] = eta4d[parl, :, 12:]
    return src.reshape(-1)


def setup_system(device: int, rank: int = 0):
    """the benchmarked system; under torchrun rank r solves its own wall
    source (stream 1 + r): N independent solves, one per GPU"""
    from cps_veloc_b200 import _abi as A
    from cps_veloc_b200.dirac import DiracOpDwf, Lattice, gen_gauge, gen_gaussian

    A.check(A.lib().cpsgpu_set_device(device))
    u = gen_gauge(L4, seed=SEED, width=0.3)
    lat = Lattice(L4, (1, 1, 1, -1))
    lat.import_gauge(u)
    D = DiracOpDwf(lat, mass=MF, ls=LS, m5=M5)
    vol = int(np.prod(L4))
    eta = gen_gaussian(vol * 24, seed=SEED, stream=1 + rank).reshape(2, vol // 2, 24)
    b = D.MatPcDag(wall_source(L4, LS, eta))
    return A, lat, D, u, b


def field(A, D, prec, host=None):
    h = C.c_void_p()
    A.check(A.lib().cpsgpu_field_create(D._h, prec, 1, C.byref(h)))
    if host is not None:
        A.check(A.lib().cpsgpu_field_upload(h, A.dptr(np.ascontiguousarray(host))))
    return h


def solve_dev(A, D, x, bf, zero, prec, delta=0.0):
    a = A.CgArg()
    A.lib().cpsgpu_cg_arg_default(C.byref(a))
    a.stop_rsd = STOP
    a.max_num_iter = 100000
    a.precision = prec
    a.delta = delta
    a.chunk = 16
    r = A.CgResult()
    A.check(A.lib().cpsgpu_field_upload(x, A.dptr(zero)))
    A.check(A.lib().cpsgpu_invcg_field(D._h, x, bf, C.byref(a), C.byref(r)))
    if r.status != A.CONVERGED:
        raise RuntimeError(f"solve did not converge: status {r.status}, true_res {r.true_res}")
    return r


def cpu_reference_dslash(u, x, y_gpu) -> dict:
    """The reference's own DWF dslash (oracle/_ref, compiled from the
    reference sources) on this host, fed the input of the GPU's FP64 dslash:
    its time, and the GPU result's relative error against it."""
    from oracle.loader import REF_SO, apply_bc_signs, load_reference, p

    if not REF_SO.exists():
        return {"error": "the reference kernels are not built here (oracle/_ref/libcpsref.so)"}
    nthreads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(nthreads)
    R = load_reference()
    R.ref_init(*L4, LS, M5, 1.5, 0.5, -1)
    us = apply_bc_signs(u, L4, (1, 1, 1, -1))
    y = np.zeros_like(x)
    t0 = time.perf_counter()
    R.ref_dwf_dslash(p(y), p(us), p(x), MF, 1, 0)
    t = time.perf_counter() - t0
    per_iter = 4 * t
    return {"value": per_iter * FP64_CG_ITERS, "unit": "s", "cores": nthreads, "kind": "reference",
            "sample": f"1 x dwf_dslash (reference noarch, 16^3x32x16) = {t:.3f} s on the GPU dslash's input; "
                      f"x4 per CG iteration x {FP64_CG_ITERS} iterations (wilson_dslash itself is single-threaded; "
                      "bench.py --impl reference times the reference's whole capped CG)",
            "s_per_iteration": per_iter,
            "rel_err_fp64_dslash_vs_reference": float(np.linalg.norm(y_gpu - y) / np.linalg.norm(y))}


def reference_wall_source_inputs():
    """The benchmarked gauge field (CANONICAL order) and wall source, built
    with the numpy restatement of the seeded generator (oracle/inputs.py): the
    reference arm does not load the library under test."""
    from oracle import inputs as I

    u_c = I.gen_gauge(L4, seed=SEED, width=0.3, order="canonical")
    vol = int(np.prod(L4))
    eta = I.gen_gaussian(vol * 24, seed=SEED, stream=1).reshape(2, vol // 2, 24)
    return u_c, wall_source(L4, LS, eta)


def reference_capped_cg(steps: int, warmup: int) -> dict:
    """The reference's own DiracOpDwf::InvCg (InvCgShift, inv_cg.C:84-448,
    compiled unchanged with its Lattice / DiracOp classes into
    oracle/_ref/libcpsref_solve.so) on the benchmarked system, capped at 1 and
    at 1 + steps iterations: the difference of the two wall times gives the
    seconds per CG iteration with the solver's fixed costs (initial residual,
    true residual) cancelled.  Time to 1e-10 = fixed costs + FP64_CG_ITERS
    iterations."""
    import tempfile

    from oracle import refsolve

    if not refsolve.available():
        raise FileNotFoundError("oracle/_ref/libcpsref_solve.so is not built (make -C oracle refsolve)")
    nthreads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(nthreads)
    u_c, w = reference_wall_source_inputs()
    with tempfile.TemporaryDirectory() as d:
        np.save(Path(d) / "u.npy", u_c)
        np.save(Path(d) / "w.npy", w)
        r = refsolve.run_child({"L": list(L4), "ls": LS, "kind": "dwf", "task": "cgtime", "m5": M5, "a5_inv": 1.0,
                                "gauge": str(Path(d) / "u.npy"), "src": str(Path(d) / "w.npy"), "mass": MF,
                                "stop_rsd": STOP, "caps": [2, 2 + steps], "warmup": min(warmup, 1)},
                               timeout=3600)
    t1, tk = (float(x) for x in r["times"])
    s_iter = (tk - t1) / steps
    fixed = t1 - s_iter
    hist = r["res_hist"]
    return {"value": fixed + (FP64_CG_ITERS - 1) * s_iter, "unit": "s", "cores": nthreads, "kind": "reference",
            "sample": f"reference DiracOpDwf::InvCg capped at 1 and {1 + steps} iterations on 16^3x32x16 Ls=16: "
                      f"{s_iter:.3f} s per iteration, {fixed:.3f} s fixed; x {FP64_CG_ITERS} iterations "
                      "(the FP64 CG iteration count of this system: the same InvCgShift recurrence)",
            "s_per_iteration": s_iter, "fixed_s": fixed, "iterations_timed": steps,
            "iterations_extrapolated_to": FP64_CG_ITERS,
            "res_sq_first_last": [float(hist[0]), float(hist[-1])] if len(hist) else None}


def _dev_time(A, fn, D, prec, reps):
    ms, by = C.c_double(), C.c_double()
    A.check(fn(D._h, prec, reps, C.byref(ms), C.byref(by)))
    return ms.value, by.value


def extra_batched(A, D, sloppy) -> dict:
    """12 point sources (the spin-colour unit vectors at one seeded site) on
    the headline system: one batched mixed-precision solve against 12
    sequential mixed solves and 12 sequential FP64 solves."""
    D.autotune(sloppy, nrhs=12)
    site = int(np.random.default_rng(SEED + 4).integers(0, D.f_size // 24))
    srcs = []
    for k in range(12):
        e = np.zeros(D.f_size)
        e[24 * site + 2 * k] = 1.0
        srcs.append(e)
    sols = [np.zeros(D.f_size) for _ in srcs]
    D.InvCgMulti(sols, srcs, stop_rsd=STOP, precision=sloppy)  # warm-up (graph capture)
    sols = [np.zeros(D.f_size) for _ in srcs]
    res = D.InvCgMulti(sols, srcs, stop_rsd=STOP, precision=sloppy)
    t_batch = res[0].seconds
    seq_mixed, seq_fp64, it64 = 0.0, 0.0, []
    for e in srcs:
        y = np.zeros(D.f_size)
        seq_mixed += D.InvCg(y, e, stop_rsd=STOP, precision=sloppy).seconds
        y = np.zeros(D.f_size)
        r = D.InvCg(y, e, stop_rsd=STOP)
        seq_fp64 += r.seconds
        it64.append(r.iterations)
    ok = all(r.status == A.CONVERGED and r.true_res <= STOP for r in res)
    # the batched solve at each right-hand-side tile (links shared by `tile`
    # solves' blocks), the autotuner's choice restored afterwards
    tuned, by_tile = D.rhs_tile(sloppy, 12), {}
    for tile in (1, 2, 4, 12):
        D.set_rhs_tile(sloppy, tile)
        sols = [np.zeros(D.f_size) for _ in srcs]
        D.InvCgMulti(sols, srcs, stop_rsd=STOP, precision=sloppy)
        sols = [np.zeros(D.f_size) for _ in srcs]
        by_tile[str(tile)] = D.InvCgMulti(sols, srcs, stop_rsd=STOP, precision=sloppy)[0].seconds
    D.set_rhs_tile(sloppy, tuned)
    # the same batch with the FP16-storage inner iteration
    D.autotune(A.HALF, nrhs=12)
    sols = [np.zeros(D.f_size) for _ in srcs]
    D.InvCgMulti(sols, srcs, stop_rsd=STOP, precision=A.HALF)
    sols = [np.zeros(D.f_size) for _ in srcs]
    rh = D.InvCgMulti(sols, srcs, stop_rsd=STOP, precision=A.HALF)
    ok_h = all(r.status == A.CONVERGED and r.true_res <= STOP for r in rh)
    return {"rhs": 12, "rhs_tile": tuned, "all_converged_1e-10": ok, "batched_mixed_s_by_rhs_tile": by_tile,
            "batched_mixed_s": t_batch, "per_rhs_batched_mixed_s": t_batch / 12,
            "sequential_mixed_s": seq_mixed, "sequential_fp64_s": seq_fp64,
            "iterations_mixed": [r.iterations for r in res], "iterations_fp64": it64,
            "speedup_batched_mixed_vs_fp64_single_rhs": seq_fp64 / t_batch,
            "speedup_batched_vs_sequential_mixed": seq_mixed / t_batch,
            "batched_half_inner_s": rh[0].seconds, "batched_half_inner_all_converged_1e-10": ok_h,
            "iterations_half_inner": [r.iterations for r in rh],
            "speedup_batched_half_inner_vs_fp64_single_rhs": seq_fp64 / rh[0].seconds}


def extra_mobius(A) -> dict:
    """Mobius 24^3x64, Ls=12, b=1.5, c=0.5, M5=1.8, m_f=0.005, 12-real links:
    FP64 CG against the FP16-storage inner solve with FP64 defect correction."""
    from cps_veloc_b200.dirac import DiracOpMobius, Lattice, gen_gauge, gen_gaussian

    L, ls = (24, 24, 24, 64), 12
    lat = Lattice(L, (1, 1, 1, -1))
    lat.import_gauge(gen_gauge(L, seed=SEED + 3, width=0.3))
    D = DiracOpMobius(lat, mass=0.005, ls=ls, m5=M5, b=1.5, c=0.5)
    for prec in (A.DOUBLE, A.HALF):
        D.autotune(prec)
    b = gen_gaussian(D.f_size, seed=SEED, stream=3)
    x = np.zeros(D.f_size)
    r64 = D.InvCg(x, b, stop_rsd=STOP, max_num_iter=50000)
    x = np.zeros(D.f_size)
    rh = D.InvCg(x, b, stop_rsd=STOP, max_num_iter=50000, precision=A.HALF)
    pk = peaks()["hbm_gbs"]
    out = {"lattice": list(L), "ls": ls, "b": 1.5, "c": 0.5, "mf": 0.005,
           "fp64_cg": {"time_s": r64.seconds, "iterations": r64.iterations, "true_res": r64.true_res},
           "half_inner_cg": {"time_s": rh.seconds, "iterations": rh.iterations, "true_res": rh.true_res,
                             "reliable_updates": rh.reliable_updates},
           "iteration_inflation": rh.iterations / r64.iterations,
           "speedup_vs_fp64_cg": r64.seconds / rh.seconds}
    for name, prec in (("fp64", A.DOUBLE), ("half", A.HALF)):
        ms, by = _dev_time(A, A.lib().cpsgpu_time_m5inv, D, prec, 20)
        flops = 48 * ls * D.f_size // 24  # dense Ls x Ls, both chiralities
        unit = ("CUDA cores, register-tiled (matrix as a kernel parameter), input tiles staged in shared "
                "memory by bulk asynchronous copies" if prec == A.HALF else "CUDA cores, shared-memory staging")
        out[f"m5inv_{name}"] = {"ms": ms, "GB_s": by / ms / 1e6, "frac_of_measured_hbm": by / ms / 1e6 / pk,
                                "flop_per_byte": flops / by, "unit": unit}
        # the other CUDA-core kernels: shared-memory staging, register-tiled without bulk staging
        for key, impl in (("shared_memory_kernel", D.MIX_SHARED), ("register_tiled_kernel", D.MIX_REG)):
            D.set_mix_impl(impl)
            ms2, by2 = _dev_time(A, A.lib().cpsgpu_time_m5inv, D, prec, 20)
            out[f"m5inv_{name}_{key}"] = {"ms": ms2, "GB_s": by2 / ms2 / 1e6,
                                          "frac_of_measured_hbm": by2 / ms2 / 1e6 / pk}
        D.set_mix_impl(D.MIX_DEFAULT)
        m2, b2 = C.c_double(), C.c_double()
        A.check(A.lib().cpsgpu_time_dslash(D._h, prec, 1, 0, 20, C.byref(m2), C.byref(b2)))
        out[f"hop_{name}"] = {"ms": m2.value, "GB_s": b2.value / m2.value / 1e6}
    # the same M5^-1 of the FP16 field on the tensor cores (mma.sync m16n8k16),
    # and the FP16-inner solve with every standalone mixing there
    D.set_mix_impl(D.MIX_TENSOR_CORES)
    ms, by = _dev_time(A, A.lib().cpsgpu_time_m5inv, D, A.HALF, 20)
    out["m5inv_half_tensor_cores"] = {"ms": ms, "GB_s": by / ms / 1e6, "frac_of_measured_hbm": by / ms / 1e6 / pk,
                                      "unit": "tensor cores (mma.sync m16n8k16, FP16 operands, FP32 accumulation)",
                                      "speedup_vs_cuda_cores": out["m5inv_half"]["ms"] / ms}
    x = np.zeros(D.f_size)
    D.InvCg(x, b, stop_rsd=STOP, max_num_iter=50000, precision=A.HALF)
    x = np.zeros(D.f_size)
    rt = D.InvCg(x, b, stop_rsd=STOP, max_num_iter=50000, precision=A.HALF)
    out["half_inner_cg_tensor_core_mixing"] = {"time_s": rt.seconds, "iterations": rt.iterations,
                                               "true_res": rt.true_res, "reliable_updates": rt.reliable_updates}
    # and with the shared-memory mixing kernel, the form before the register-tiled one
    D.set_mix_impl(D.MIX_SHARED)
    x = np.zeros(D.f_size)
    D.InvCg(x, b, stop_rsd=STOP, max_num_iter=50000, precision=A.HALF)
    x = np.zeros(D.f_size)
    rs = D.InvCg(x, b, stop_rsd=STOP, max_num_iter=50000, precision=A.HALF)
    out["half_inner_cg_shared_memory_mixing"] = {"time_s": rs.seconds, "iterations": rs.iterations}
    D.set_mix_impl(D.MIX_DEFAULT)
    D.close()
    lat.close()
    return out


def extra_multishift(A) -> dict:
    """Wilson 32^3x64, kappa=0.125, 16 shifts log-spaced in [1e-4, 10]: FP64
    multishift CG against FP32 multishift + FP64 refinement of every shift
    (wall time of the host-vector call, transfers of 16 solutions included;
    after one untimed call, into solution arrays already resident in host
    memory as a caller's would be)."""
    from cps_veloc_b200.dirac import DiracOpWilson, Lattice, gen_gauge, gen_gaussian

    L = (32, 32, 32, 64)
    lat = Lattice(L, (1, 1, 1, -1))
    lat.import_gauge(gen_gauge(L, seed=SEED + 5, width=0.3))
    D = DiracOpWilson(lat, mass=1 / (2 * 0.125) - 4)
    for prec in (A.DOUBLE, A.SINGLE):
        D.autotune(prec)
    shifts = list(np.logspace(-4, 1, 16))
    chi = gen_gaussian(D.f_size, seed=SEED, stream=5)
    out = {"lattice": list(L), "kappa": 0.125, "shifts": len(shifts)}
    psi = [np.full(D.f_size, 0.0) for _ in shifts]  # touched: resident host memory
    for name, prec in (("fp64", A.DOUBLE), ("fp32_then_fp64_refine", A.SINGLE)):
        for rep in range(2):  # the first call allocates the device workspace
            for x in psi:
                x.fill(0.0)
            rs = np.full(len(shifts), STOP)
            t0 = time.perf_counter()
            k = D.MInvCG(psi, chi, float(chi @ chi), shifts, rs, precision=prec)
            t = time.perf_counter() - t0
        phases = D.minvcg_stats()
        y, _ = D.MatPcDagMatPc(psi[0])
        worst = float(np.linalg.norm(chi - y - shifts[0] * psi[0]) / np.linalg.norm(chi))
        out[name] = {"wall_s": t, "iterations": k, "true_res_smallest_shift": worst, "phases": phases}
    D.close()
    lat.close()
    return out


BATCH_MIXED = [(8, 8, 8, 16), (8, 8, 8, 32), (12, 12, 12, 16), (12, 12, 12, 24), (16, 16, 16, 16),
               (16, 16, 16, 24), (16, 16, 16, 32), (16, 16, 16, 32)]
BATCH_SMALL = [(8, 8, 8, 8)] * 4 + [(8, 8, 8, 16)] * 4


def extra_solve_batch(A, lattices=BATCH_MIXED, ls=LS) -> dict:
    """Eight independent DWF solves, M5 = 1.8, m_f log-spaced in [0.001,
    0.1], on the given lattices (default 8^3x16 ... 16^3x32, Ls 16), mixed
    precision (FP32 inner) to a true residual of 1e-10: one cpsgpu_solve_batch
    call (every solve's loop a branch of one graph launch) against the same
    eight solves one after another (cpsgpu_invcg_field); wall time of the
    device-field calls after one untimed round each."""
    from cps_veloc_b200.dirac import DiracOpDwf, Lattice, gen_gauge, gen_gaussian

    masses = list(np.logspace(-3, -1, 8))
    lats, ops, sols, srcs, zeros = [], [], [], [], []
    for k, (L, m) in enumerate(zip(lattices, masses)):
        lat = Lattice(L, (1, 1, 1, -1))
        lat.import_gauge(gen_gauge(L, seed=SEED + 20 + k, width=0.3))
        D = DiracOpDwf(lat, mass=m, ls=ls, m5=M5)
        D.autotune(A.SINGLE)
        lats.append(lat)
        ops.append(D)
        z = np.zeros(D.f_size)
        zeros.append(z)
        sols.append(field(A, D, A.DOUBLE, z))
        srcs.append(field(A, D, A.DOUBLE, gen_gaussian(D.f_size, seed=SEED, stream=30 + k)))
    arg = A.CgArg()
    A.lib().cpsgpu_cg_arg_default(C.byref(arg))
    arg.stop_rsd, arg.max_num_iter, arg.precision, arg.chunk = STOP, 100000, A.SINGLE, 16
    n = len(ops)
    VP = C.c_void_p * n

    def reset():
        for f, z in zip(sols, zeros):
            A.check(A.lib().cpsgpu_field_upload(f, A.dptr(z)))

    def batch():
        res = (A.CgResult * n)()
        reset()
        t0 = time.perf_counter()
        A.check(A.lib().cpsgpu_solve_batch(n, VP(*[D._h.value for D in ops]), VP(*[f.value for f in sols]),
                                           VP(*[f.value for f in srcs]), (A.CgArg * n)(*([arg] * n)), res))
        return time.perf_counter() - t0, list(res)

    def sequential():
        reset()
        tot, out = 0.0, []
        for D, fx, fb in zip(ops, sols, srcs):
            r = A.CgResult()
            t0 = time.perf_counter()
            A.check(A.lib().cpsgpu_invcg_field(D._h, fx, fb, C.byref(arg), C.byref(r)))
            tot += time.perf_counter() - t0
            out.append(r)
        return tot, out

    batch()
    sequential()
    tb, rb = batch()
    ts, rs = sequential()
    for f in sols + srcs:
        A.lib().cpsgpu_field_destroy(f)
    for D, lat in zip(ops, lats):
        D.close()
        lat.close()
    return {"lattices": [list(L) for L in lattices], "ls": ls, "mf": masses, "inner": "fp32",
            "batch_one_launch_s": tb, "sequential_s": ts, "speedup_batch_vs_sequential": ts / tb,
            "iterations": [r.iterations for r in rb], "iterations_sequential": [r.iterations for r in rs],
            "all_converged_1e-10": all(r.status == A.CONVERGED and r.true_res <= STOP for r in rb)}


def extra_force(A, D, pk) -> dict:
    """HMC fermion force on the headline DWF system (FdwfBase::EvolveMomFforce):
    CalcHmdForceVecs (MatPc + two Dslash in FP64) plus the fused force kernel,
    device-resident, event-timed; the kernel's algorithmic bytes are v1, v2
    (both parities, all slices) read once, the FP64 links read once and the
    momentum field read and written."""
    tot, ker, by = C.c_double(), C.c_double(), C.c_double()
    A.check(A.lib().cpsgpu_time_fforce(D._h, 20, C.byref(tot), C.byref(ker), C.byref(by)))
    gbs = by.value / (ker.value * 1e-3) / 1e9
    return {"ms_per_call": tot.value, "force_kernel_ms": ker.value, "force_kernel_GB_s": gbs,
            "force_kernel_frac_of_measured_hbm": gbs / pk["hbm_gbs"], "force_kernel_bytes": by.value}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return dist


def max_over_ranks(dist, v: float) -> float:
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    info = reference_capped_cg(max(1, args.steps), args.warmup)
    v = info["value"]
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": info["s_per_iteration"] * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {k: info[k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "s"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cg": info,
    }
    print(json.dumps(out), flush=True)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sloppy", default="single", choices=["half", "single"],
                    help="inner precision of the timed mixed solve (the workload specifies FP32)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other systems (12 point sources, Mobius 24^3x64, multishift 32^3x64)")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return run_reference_arm(args)

    from cps_veloc_b200.dirac import gen_gaussian

    ws, rank, local = dist_env()
    dist = init_dist(ws)
    A, lat, D, u, b = setup_system(local, rank)
    sloppy = A.HALF if args.sloppy == "half" else A.SINGLE
    n = D.f_size
    zero = np.zeros(n)
    bf = field(A, D, A.DOUBLE, b)
    x = field(A, D, A.DOUBLE, zero)
    for prec in (A.DOUBLE, A.SINGLE, A.HALF):
        D.autotune(prec)

    # plain FP64 CG (the comparison point of the metric)
    solve_dev(A, D, x, bf, zero, A.DOUBLE)  # warm-up
    fp64 = [solve_dev(A, D, x, bf, zero, A.DOUBLE) for _ in range(max(1, args.fp64_steps))]
    x64 = np.empty(n)
    A.check(A.lib().cpsgpu_field_download(x, A.dptr(x64)))

    # mixed precision: W warm-up solves, K timed solves
    for _ in range(args.warmup):
        solve_dev(A, D, x, bf, zero, sloppy)
    if dist:
        dist.barrier()
    lat.synchronize()
    with ClockSampler(local) as clk:
        res = [solve_dev(A, D, x, bf, zero, sloppy) for _ in range(args.steps)]
        lat.synchronize()
    if dist:
        dist.barrier()
    xm = np.empty(n)
    A.check(A.lib().cpsgpu_field_download(x, A.dptr(xm)))
    # the other inner precision, outside the timed region
    other = A.HALF if sloppy == A.SINGLE else A.SINGLE
    solve_dev(A, D, x, bf, zero, other)
    ro = [solve_dev(A, D, x, bf, zero, other) for _ in range(max(1, args.steps))]
    t_other = max_over_ranks(dist, statistics.median(r.seconds for r in ro))
    t_mixed = max_over_ranks(dist, statistics.median(r.seconds for r in res))
    t_fp64 = max_over_ranks(dist, statistics.median(r.seconds for r in fp64))

    # dominant kernel: the inner solver's dslash, timed alone from HBM
    pk = peaks()
    ms = C.c_double()
    by = C.c_double()
    A.check(A.lib().cpsgpu_time_dslash(D._h, sloppy, 1, 0, 50, C.byref(ms), C.byref(by)))
    dsl = {}
    for name, prec in (("fp64", A.DOUBLE), ("fp32", A.SINGLE), ("half", A.HALF)):
        m2, b2 = C.c_double(), C.c_double()
        A.check(A.lib().cpsgpu_time_dslash(D._h, prec, 1, 0, 30, C.byref(m2), C.byref(b2)))
        gbs = b2.value / (m2.value * 1e-3) / 1e9
        dsl[name] = {"ms": m2.value, "GB_s": gbs, "frac_of_measured_hbm": gbs / pk["hbm_gbs"],
                     "GFLOP_s": (1320 + 48) * L4[0] * L4[1] * L4[2] * L4[3] // 2 * LS / (m2.value * 1e-3) / 1e9}
    achieved = by.value / (ms.value * 1e-3) / 1e9
    form = lat.link_reals(sloppy)
    hop_shape = D.hop_shape(sloppy)
    traffic_key = (sloppy, form, shape_class(hop_shape))
    traffic = DSLASH_TRAFFIC.get(traffic_key)

    # end to end through the host-pointer C ABI: H2D source + guess, D2H solution
    pin_b = C.c_void_p()
    pin_x = C.c_void_p()
    A.check(A.lib().cpsgpu_host_alloc(n * 8, C.byref(pin_b)))
    A.check(A.lib().cpsgpu_host_alloc(n * 8, C.byref(pin_x)))
    hb = np.ctypeslib.as_array(C.cast(pin_b, C.POINTER(C.c_double)), shape=(n,))
    hx = np.ctypeslib.as_array(C.cast(pin_x, C.POINTER(C.c_double)), shape=(n,))
    hb[:] = b
    e2e_t = []
    arg = A.CgArg()
    A.lib().cpsgpu_cg_arg_default(C.byref(arg))
    arg.stop_rsd, arg.max_num_iter, arg.precision, arg.chunk = STOP, 100000, sloppy, 16
    for k in range(max(1, args.steps)):
        hx[:] = 0.0
        r = A.CgResult()
        t0 = time.perf_counter()
        A.check(A.lib().cpsgpu_invcg(D._h, A.dptr(hx), A.dptr(hb), C.byref(arg), C.byref(r)))
        e2e_t.append(time.perf_counter() - t0)
        if r.status != A.CONVERGED or r.true_res > STOP:
            raise RuntimeError("end-to-end solve failed")
    e2e = max_over_ranks(dist, statistics.median(e2e_t))

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            xs = gen_gaussian(n, seed=SEED, stream=9)
            cpu = cpu_reference_dslash(u, xs, D.Dslash(xs, 1, 0))
        except Exception as e:  # noqa: BLE001
            cpu = {"error": str(e)}

    extras = None
    if rank == 0 and not args.no_extras:
        extras = {"batched_12_point_sources": extra_batched(A, D, sloppy),
                  "mobius_24x64_ls12": extra_mobius(A),
                  "multishift_wilson_32x64": extra_multishift(A),
                  "batch_8_dwf_solves": extra_solve_batch(A),
                  "batch_8_small_dwf_solves": extra_solve_batch(A, BATCH_SMALL, 8),
                  "hmc_force_dwf_16x32_ls16": extra_force(A, D, pk)}

    rel_err = float(np.linalg.norm(xm - x64) / np.linalg.norm(x64))
    if rank == 0:
        out = {
            "metric": METRIC, "value": t_mixed, "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mixed * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f16" if sloppy == A.HALF else "f64+f32", "data": "synthetic",
            "config": workload_config(),
            "inner": "fp16 storage + per-site norm, fp32 arithmetic" if sloppy == A.HALF else "fp32",
            "parallelism": f"{ws} independent solves, one per GPU" if ws > 1 else "1 GPU",
            "fp64_cg": {"time_s": t_fp64, "iterations": fp64[0].iterations, "true_res": fp64[0].true_res},
            "mixed_cg": {"time_s": t_mixed, "iterations": res[0].iterations,
                         "reliable_updates": res[0].reliable_updates, "true_res": res[0].true_res,
                         "rel_err_vs_fp64": rel_err},
            "speedup_vs_fp64_cg": t_fp64 / t_mixed,
            ("mixed_cg_fp16_inner" if other == A.HALF else "mixed_cg_fp32_inner"): {
                "time_s": t_other, "iterations": ro[0].iterations, "reliable_updates": ro[0].reliable_updates,
                "true_res": ro[0].true_res, "speedup_vs_fp64_cg": t_fp64 / t_other},
            "dslash": dsl,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "traffic": traffic,
                         "traffic_shape_class": traffic_key[2],
                         "algorithmic_bytes": by.value, "traffic_unit": "bytes per launch (ncu, single launch)",
                         "kernel": "hop_kernel DWF dslash, " + ("fp16" if sloppy == A.HALF else "fp32")
                         + f", {form}-real links",
                         # the shape of the timed dslash (the extras below retune the operator)
                         "launch_shape_sites_slices_per_block_slices_per_thread_order": list(hop_shape),
                         "peak_source": pk["source"]},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": 2 * n * 8, "d2h_bytes_per_step": n * 8},
            "clocks": clk.summary(),
            "other_systems": extras,
            "gpu_launches": int(sum(r.kernels for r in res)),
        }
        print(json.dumps(out), flush=True)
    A.lib().cpsgpu_host_free(pin_b)
    A.lib().cpsgpu_host_free(pin_x)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
