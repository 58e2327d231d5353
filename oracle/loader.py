"""Test infrastructure only: ctypes loaders for the oracle libraries.

liboracle.so  the C restatement (oracle.c), built here or on any box by
              ``make -C oracle oracle`` (gcc only);
libcpsref.so  the reference's own noarch kernels compiled from the
              reference source tree (``make -C oracle ref``).  Available only
              where the reference tree exists or the .so was built before.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
ORACLE_SO = OUT / "liboracle.so"
REF_SO = OUT / "libcpsref.so"
# the reference's cps_pp source directory, from the environment only
REF_SRC = Path(os.environ["CPS_REF"]) if os.environ.get("CPS_REF") else None
REF_GPU_SO = OUT / "libcpsref_gpu.so"
REF_SOLVE_SO = OUT / "libcpsref_solve.so"

_dp = C.POINTER(C.c_double)


class OracleGeom(C.Structure):
    _fields_ = [("L", C.c_int * 4), ("ls", C.c_int), ("bc", C.c_double * 4), ("a5_inv", C.c_double)]

    @classmethod
    def make(cls, L, ls=1, bc=(1, 1, 1, -1), a5_inv=1.0):
        g = cls()
        for k in range(4):
            g.L[k] = L[k]
            g.bc[k] = bc[k]
        g.ls = ls
        g.a5_inv = a5_inv
        return g


class OracleMobius(C.Structure):
    _fields_ = [("b", C.c_double * 128), ("c", C.c_double * 128), ("kappa_b", C.c_double * 128),
                ("K", C.c_double * 128)]


MDAGM_FN = C.CFUNCTYPE(None, C.c_void_p, _dp, _dp, _dp)
MATPC_FN = C.CFUNCTYPE(None, C.c_void_p, _dp, _dp)


def _make(target: str) -> None:
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    cmd = ["make", "-s", "-j8", "-C", str(HERE), target] + ([f"REF={REF_SRC}"] if REF_SRC else [])
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"building oracle target {target} failed:\n{r.stdout}\n{r.stderr}")


def build_oracle(force: bool = False) -> Path:
    src = HERE / "oracle.c"
    if force or not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < max(src.stat().st_mtime,
                                                                           (HERE / "oracle.h").stat().st_mtime):
        _make("oracle")
    return ORACLE_SO


def _ref_tree() -> bool:
    return REF_SRC is not None and REF_SRC.exists()


def build_reference() -> Path:
    """the reference's kernels (libcpsref.so); needs CPS_REF unless prebuilt"""
    if not REF_SO.exists():
        if not _ref_tree():
            raise FileNotFoundError("reference kernels not prebuilt and CPS_REF does not name the reference's cps_pp")
        _make("ref")
    return REF_SO


def build_reference_solvers() -> Path:
    """the reference's Lattice / DiracOp solvers (libcpsref_solve.so)"""
    if not REF_SOLVE_SO.exists():
        if not _ref_tree():
            raise FileNotFoundError("reference solvers not prebuilt and CPS_REF does not name the reference's cps_pp")
        _make("refsolve")
    return REF_SOLVE_SO


def build_reference_gpu() -> Path:
    """the reference's solvers with the library's CPS-side shim in place of
    DiracOp::InvCgShift (libcpsref_gpu.so; needs libcpsgpu.so built)"""
    if _ref_tree():
        _make("refgpu")  # relinks when libcpsgpu.so or the shim changed
    elif not REF_GPU_SO.exists():
        raise FileNotFoundError("reference + shim not prebuilt and CPS_REF does not name the reference's cps_pp")
    return REF_GPU_SO


def reference_available() -> bool:
    return REF_SO.exists() or _ref_tree()


_oracle = None
_ref = None


def load_oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        L = C.CDLL(str(build_oracle()))
        g = C.POINTER(OracleGeom)
        m = C.POINTER(OracleMobius)
        i, d = C.c_int, C.c_double
        sig = {
            "orc_wilson_dslash": [g, _dp, _dp, _dp, i, i],
            "orc_wilson_m": [g, _dp, _dp, _dp, d, i],
            "orc_wilson_mdagm": [g, _dp, _dp, _dp, d, _dp],
            "orc_dwf_dslash": [g, _dp, _dp, _dp, d, i, i],
            "orc_dwf_m": [g, _dp, _dp, _dp, d, d, i],
            "orc_dwf_mdagm": [g, _dp, _dp, _dp, d, d, _dp],
            "orc_mobius_dslash_4": [g, m, _dp, _dp, _dp, i, i, d],
            "orc_mobius_m5inv": [g, m, _dp, d, i],
            "orc_mobius_m": [g, m, _dp, _dp, _dp, d, i],
            "orc_mobius_mdagm": [g, m, _dp, _dp, _dp, d, _dp],
            "orc_mobius_m5": [g, m, _dp, d],
            "orc_mobius_m_pc": [g, m, _dp, _dp, _dp, d, i, i],
            "orc_mobius_mdagm_pc": [g, m, _dp, _dp, _dp, d, _dp, i],
            "orc_sproj_tr": [i, i, _dp, _dp, _dp, i, i, i],
            "orc_force_matrix": [_dp, _dp, _dp, _dp, d],
            "orc_fforce": [g, _dp, _dp, _dp, _dp, d, _dp],
            "orc_mobius_booee": [g, m, _dp, _dp, d],
            "orc_fforce_wilson_type": [g, _dp, _dp, _dp, _dp, d, _dp],
        }
        for k, a in sig.items():
            getattr(L, k).argtypes = a
            getattr(L, k).restype = None
        L.orc_mobius_params.argtypes = [m, i, d, d, d]
        L.orc_mobius_params.restype = None
        L.orc_mobius_params_a5.argtypes = [m, i, d, d, d, d]
        L.orc_mobius_params_a5.restype = None
        L.orc_invcg.argtypes = [MDAGM_FN, C.c_void_p, C.c_long, _dp, _dp, d, d, i, _dp, _dp]
        L.orc_invcg.restype = i
        L.orc_wilson_matinv.argtypes = [g, _dp, _dp, _dp, d, d, i, _dp]
        L.orc_dwf_matinv.argtypes = [g, _dp, _dp, _dp, d, d, d, i, _dp]
        L.orc_mobius_matinv.argtypes = [g, m, _dp, _dp, _dp, d, d, i, _dp]
        L.orc_mobius_matinv_pc.argtypes = [g, m, _dp, _dp, _dp, d, d, i, _dp, i]
        L.orc_mobius_matinv_pc.restype = i
        L.orc_bicgstab.argtypes = [MATPC_FN, C.c_void_p, C.c_long, _dp, _dp, d, i, d, i, _dp]
        L.orc_bicgstab.restype = i
        L.orc_minresext.argtypes = [MDAGM_FN, C.c_void_p, C.c_long, _dp, _dp, C.POINTER(_dp), C.POINTER(_dp), i,
                                    _dp]
        L.orc_minresext.restype = None
        L.orc_sym_eigen.argtypes = [_dp, _dp, _dp, i]
        L.orc_sym_eigen.restype = None
        L.orc_inveigcg.argtypes = [MDAGM_FN, C.c_void_p, C.c_long, _dp, _dp, d, i, i, i, C.POINTER(_dp), _dp, i,
                                   C.POINTER(_dp), _dp, _dp, i, _dp]
        L.orc_inveigcg.restype = i
        L.orc_ritz.argtypes = [MDAGM_FN, C.c_void_p, i, C.c_long, C.POINTER(_dp), i, d, d, d, d, i, i, i, i, d, i,
                               i, _dp]
        L.orc_ritz.restype = i
        L.orc_jacobi.argtypes = [C.POINTER(_dp), C.c_long, i, _dp, _dp, d, i]
        L.orc_jacobi.restype = i
        L.orc_ritz_eig.argtypes = [MDAGM_FN, C.c_void_p, i, C.c_long, C.POINTER(_dp), i, d, d, d, d, i, i, i, i, i,
                                   i, i, _dp, C.POINTER(i)]
        L.orc_ritz_eig.restype = i
        L.orc_qrtrf.argtypes = [_dp, _dp, i, _dp, i, d, i, i]
        L.orc_qrtrf.restype = None
        L.orc_tqri.argtypes = [_dp, _dp, i, i, _dp, i]
        L.orc_tqri.restype = i
        L.orc_eigsrt.argtypes = [_dp, _dp, i, i]
        L.orc_eigsrt.restype = None
        L.orc_lanczos.argtypes = [MDAGM_FN, C.c_void_p, i, i, C.c_long, C.POINTER(C.POINTER(C.c_float)), _dp, i, i, i,
                                  i, d, i, i, d, d, d]
        L.orc_lanczos.restype = i
        L.orc_inv_lowmode_approx.argtypes = [C.POINTER(_dp), C.POINTER(_dp), i, C.POINTER(C.POINTER(C.c_float)), _dp,
                                             i, C.c_long, i]
        L.orc_inv_lowmode_approx.restype = None
        for k in ("orc_wilson_matinv", "orc_dwf_matinv", "orc_mobius_matinv"):
            getattr(L, k).restype = i
        L.orc_minvcg.argtypes = [MDAGM_FN, C.c_void_p, C.c_long, C.POINTER(_dp), _dp, d, _dp, i, _dp, i, _dp, i]
        L.orc_minvcg.restype = i
        _oracle = L
    return _oracle


def load_reference() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(str(build_reference()))
        i, d = C.c_int, C.c_double
        L.ref_init.argtypes = [i, i, i, i, i, d, d, d, i]
        L.ref_init.restype = i
        L.ref_init_a5.argtypes = [i, i, i, i, i, d, d, d, i, d]
        L.ref_init_a5.restype = i
        for k in ("ref_dwf_kappa", "ref_mobius_kappa_b", "ref_mobius_kappa_c"):
            getattr(L, k).restype = d
        sig = {
            "ref_wilson_dslash": [_dp, _dp, _dp, i, i],
            "ref_wilson_m": [_dp, _dp, _dp, d],
            "ref_wilson_mdag": [_dp, _dp, _dp, d],
            "ref_wilson_mdagm": [_dp, _dp, _dp, _dp, d],
            "ref_dwf_dslash": [_dp, _dp, _dp, d, i, i],
            "ref_dwf_dslash_4": [_dp, _dp, _dp, i, i],
            "ref_dwf_dslash_5_plus": [_dp, _dp, d, i],
            "ref_dwf_m": [_dp, _dp, _dp, d],
            "ref_dwf_mdag": [_dp, _dp, _dp, d],
            "ref_dwf_mdagm": [_dp, _dp, _dp, _dp, d],
            "ref_zmobius_dslash_4": [_dp, _dp, _dp, i, i, d],
            "ref_zmobius_m5inv": [_dp, d, i],
            "ref_zmobius_kappa_dslash_5_plus": [_dp, _dp, d, i],
            "ref_set_zmobius": [_dp, _dp],
            "ref_zmobius_m": [_dp, _dp, _dp, d],
            "ref_zmobius_mdag": [_dp, _dp, _dp, d],
            "ref_zmobius_mdagm": [_dp, _dp, _dp, _dp, d],
            "ref_sproj_tr": [i, _dp, _dp, _dp, i, i, i],
            "ref_mobius_dslash_4": [_dp, _dp, _dp, i, i, d],
            "ref_mobius_m5inv": [_dp, _dp, d, i],
            "ref_mobius_booee": [_dp, _dp, d],
            "ref_mobius_kappa_dslash_5_plus": [_dp, _dp, d, i, d],
            "ref_mobius_m": [_dp, _dp, _dp, d],
            "ref_fforce_wilson_type": [_dp, _dp, _dp, _dp, i, d, _dp],
            "ref_force_matrix": [_dp, _dp, _dp, _dp, d],
        }
        for k, a in sig.items():
            getattr(L, k).argtypes = a
            getattr(L, k).restype = None
        L.ref_eigen_solver.argtypes = [_dp, _dp, _dp, i]
        L.ref_eigen_solver.restype = i
        L.ref_tqri.argtypes = [_dp, _dp, i, i, _dp]
        L.ref_tqri.restype = i
        L.ref_qrtrf.argtypes = [_dp, _dp, i, i, _dp, d, i, i]
        L.ref_qrtrf.restype = None
        L.ref_eigsrt.argtypes = [_dp, _dp, i]
        L.ref_eigsrt.restype = None
        L.ref_fp_checksum.argtypes = [C.c_char_p, i, i]
        L.ref_fp_checksum.restype = C.c_uint
        _ref = L
    return _ref


def p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def apply_bc_signs(u: np.ndarray, L, bc) -> np.ndarray:
    """The reference's BondCond on a WILSON-order field: links of direction mu
    at x_mu = L_mu - 1 times bc[mu] (lattice_base.C:5336)."""
    u = u.copy().reshape(2, -1, 4, 18)
    vh = u.shape[1]
    hx = L[0] // 2
    for par in range(2):
        i = np.arange(vh)
        r = i // hx
        y = r % L[1]
        r = r // L[1]
        z = r % L[2]
        t = r // L[2]
        x = 2 * (i % hx) + ((y + z + t + par) & 1)
        c = [x, y, z, t]
        for mu in range(4):
            if bc[mu] < 0:
                sel = c[mu] == L[mu] - 1
                u[par, sel, mu, :] *= -1.0
    return u.reshape(-1)
