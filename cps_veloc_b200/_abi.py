"""ctypes binding of the C ABI in include/cpsgpu.h.

The library is the in-tree ``libcpsgpu.so`` built by ``cps_veloc_b200.build``;
loading fails loudly if it is missing (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libcpsgpu.so"

DOUBLE, SINGLE, HALF = 0, 1, 2
LINKS_F32_12, LINKS_F32_18 = 112, 118  # link forms of the FP16 operator that read FP32 links
WILSON, DWF, MOBIUS = 0, 1, 2


class StrOrd:
    """StrOrdType values (enum_int.h:87-97) the host conversions take"""
    CANONICAL = 0
    WILSON = 2

MS_SINGLE, MS_MULTI, MS_GENERAL = 0, 1, 2
CONVERGED, MAX_ITER, BREAKDOWN, NONFINITE = 1, 2, 3, 4

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class DiracArg(C.Structure):
    _fields_ = [("kind", C.c_int), ("ls", C.c_int), ("mass", C.c_double), ("m5", C.c_double),
                ("mobius_b", C.c_double), ("mobius_c", C.c_double), ("a5_inv", C.c_double)]


class ForceArg(C.Structure):
    """cpsgpu_force_arg: the reference's ForceArg (L1, L2, Linf)"""
    _fields_ = [("L1", C.c_double), ("L2", C.c_double), ("Linf", C.c_double)]


class NerscHeader(C.Structure):
    """cpsgpu_nersc_header"""
    _fields_ = [("dims", C.c_int * 4), ("recon_row_3", C.c_int), ("fp_format", C.c_int), ("plaquette", C.c_double),
                ("link_trace", C.c_double), ("checksum", C.c_uint), ("sequence_number", C.c_int),
                ("ensemble_id", C.c_char * 128), ("ensemble_label", C.c_char * 128), ("creator", C.c_char * 128)]


FP_FORMATS = {"IEEE32": 3, "IEEE32BIG": 4, "IEEE32LITTLE": 5, "IEEE64": 6, "IEEE64BIG": 7, "IEEE64LITTLE": 8}


class RitzArg(C.Structure):
    """cpsgpu_ritz_arg (DiracOp::Ritz parameters)"""
    _fields_ = [("RsdR_a", C.c_double), ("RsdR_r", C.c_double), ("Rsdlam", C.c_double), ("Cutl_zero", C.c_double),
                ("Cv_fact", C.c_double), ("n_renorm", C.c_int), ("Kalk_Sim", C.c_int), ("N_min", C.c_int),
                ("N_max", C.c_int), ("MaxCG", C.c_int), ("ProjApsiP", C.c_int), ("neg", C.c_int)]


RITZ_MAT_HERM, RITZ_MATPC_HERM, RITZ_MATPCDAG_MATPC, RITZ_NEG_MATPCDAG_MATPC = 1, 2, 3, 4
INV_CG, INV_LOWMODEAPPROX, INV_CG_LOWMODE_DEFL = 0, 3, 4  # InverterType (enum_int.h:707-716)


class LanczosArg(C.Structure):
    """cpsgpu_lanczos_arg (LanczosArg with its MatrixPolynomialArg)"""
    _fields_ = [("RitzMat_lanczos", C.c_int), ("RitzMat_convcheck", C.c_int), ("nk_lanczos_vectors", C.c_int),
                ("nt_lanczos_vectors", C.c_int), ("np_lanczos_vectors", C.c_int), ("eigen_shift", C.c_double),
                ("stop_residual", C.c_double), ("maxiters", C.c_int), ("conv_check", C.c_int), ("Npol", C.c_int),
                ("params", C.c_double * 2)]


class CgArg(C.Structure):
    _fields_ = [("stop_rsd", C.c_double), ("max_num_iter", C.c_int), ("src_norm_sq", C.c_double),
                ("shift", C.c_double), ("precision", C.c_int), ("delta", C.c_double), ("chunk", C.c_int),
                ("use_graph", C.c_int)]


class MInvCgStats(C.Structure):
    _fields_ = [("upload_s", C.c_double), ("recurrence_s", C.c_double), ("refine_s", C.c_double),
                ("download_s", C.c_double), ("refine_iterations_max", C.c_int), ("refine_iterations_sum", C.c_int)]


class CgResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("true_res", C.c_double),
                ("reliable_updates", C.c_int), ("seconds", C.c_double), ("kernels", C.c_longlong)]


class CpsGpuError(RuntimeError):
    pass


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise CpsGpuError(f"{LIB_PATH} is missing: run `python -m cps_veloc_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        sigs = {
            "cpsgpu_version": (C.c_char_p, []),
            "cpsgpu_last_error": (C.c_char_p, []),
            "cpsgpu_device_count": (C.c_int, [C.POINTER(C.c_int)]),
            "cpsgpu_set_device": (C.c_int, [C.c_int]),
            "cpsgpu_lattice_create": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(vp)]),
            "cpsgpu_lattice_destroy": (C.c_int, [vp]),
            "cpsgpu_import_gauge": (C.c_int, [vp, _dp, C.c_int]),
            "cpsgpu_gauge_info": (C.c_int, [vp, _dp, C.POINTER(C.c_int)]),
            "cpsgpu_synchronize": (C.c_int, [vp]),
            "cpsgpu_set_link_reals": (C.c_int, [vp, C.c_int, C.c_int]),
            "cpsgpu_get_link_reals": (C.c_int, [vp, C.c_int, _ip]),
            "cpsgpu_get_rhs_tile": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_int)]),
            "cpsgpu_set_rhs_tile": (C.c_int, [vp, C.c_int, C.c_int]),
            "cpsgpu_dirac_create": (C.c_int, [vp, C.POINTER(DiracArg), C.POINTER(vp)]),
            "cpsgpu_dirac_destroy": (C.c_int, [vp]),
            "cpsgpu_dirac_set_zmobius": (C.c_int, [vp, _dp, _dp]),
            "cpsgpu_dirac_info": (C.c_int, [vp, _dp, _dp]),
            "cpsgpu_dslash": (C.c_int, [vp, _dp, _dp, C.c_int, C.c_int, C.c_int]),
            "cpsgpu_matpc": (C.c_int, [vp, _dp, _dp, C.c_int, C.c_int]),
            "cpsgpu_matpc_dag_matpc": (C.c_int, [vp, _dp, _dp, _dp, C.c_int]),
            "cpsgpu_matpc_dag_matpc_noalloc": (C.c_int, [vp, vp, vp, _dp]),
            "cpsgpu_mat": (C.c_int, [vp, _dp, _dp, C.c_int]),
            "cpsgpu_set_mix_impl": (C.c_int, [vp, C.c_int]),
            "cpsgpu_mat_herm": (C.c_int, [vp, _dp, _dp]),
            "cpsgpu_matpc_dag_matpc_shift": (C.c_int, [vp, _dp, _dp, C.c_double, _dp, C.c_int]),
            "cpsgpu_mobius_dslash_4": (C.c_int, [vp, _dp, _dp, C.c_int, C.c_int, C.c_int]),
            "cpsgpu_mobius_m5inv": (C.c_int, [vp, _dp, _dp, C.c_int, C.c_int]),
            "cpsgpu_cg_arg_default": (None, [C.POINTER(CgArg)]),
            "cpsgpu_invcg": (C.c_int, [vp, _dp, _dp, C.POINTER(CgArg), C.POINTER(CgResult)]),
            "cpsgpu_matinv": (C.c_int, [vp, _dp, _dp, C.POINTER(CgArg), C.POINTER(CgResult)]),
            "cpsgpu_matinv_lowmode": (C.c_int, [vp, _dp, _dp, C.POINTER(CgArg), C.c_int, C.c_char_p, C.c_int,
                                                C.POINTER(CgResult)]),
            "cpsgpu_eigencache_load": (C.c_int, [vp, C.c_char_p, C.c_int, C.POINTER(C.POINTER(C.c_float)), _dp]),
            "cpsgpu_eigencache_clear": (C.c_int, [vp]),
            "cpsgpu_inv_lowmode_approx": (C.c_int, [vp, C.POINTER(_dp), C.POINTER(_dp), C.c_int, C.c_char_p, C.c_int,
                                                    C.c_int]),
            "cpsgpu_gauge_plaquette": (C.c_int, [vp, _dp, _dp]),
            "cpsgpu_nersc_read": (C.c_int, [C.c_char_p, _ip, _dp, C.POINTER(NerscHeader)]),
            "cpsgpu_nersc_write": (C.c_int, [C.c_char_p, _ip, _dp, C.c_int, C.c_int, C.POINTER(NerscHeader),
                                             C.POINTER(NerscHeader)]),
            "cpsgpu_lattice_load_nersc": (C.c_int, [vp, C.c_char_p, C.c_double, C.POINTER(NerscHeader), _dp]),
            "cpsgpu_calc_hmd_force_vecs": (C.c_int, [vp, _dp, _dp, _dp]),
            "cpsgpu_evolve_mom_fforce": (C.c_int, [vp, _dp, _dp, C.c_double, C.POINTER(ForceArg)]),
            "cpsgpu_time_fforce": (C.c_int, [vp, C.c_int, _dp, _dp, _dp]),
            "cpsgpu_rhmc_evolve_mom_fforce": (C.c_int, [vp, _dp, C.POINTER(_dp), C.c_int, _dp, C.c_double, C.c_int,
                                                        C.POINTER(ForceArg)]),
            "cpsgpu_ritz": (C.c_int, [vp, C.POINTER(_dp), C.c_int, C.POINTER(RitzArg), _dp, _ip]),
            "cpsgpu_jacobi": (C.c_int, [vp, C.POINTER(_dp), C.c_int, _dp, _dp, C.c_double, C.c_int, _ip]),
            "cpsgpu_ritz_eig": (C.c_int, [vp, C.POINTER(_dp), C.c_int, C.POINTER(RitzArg), C.c_int, _dp, _ip, _ip]),
            "cpsgpu_imp_res_lanczos": (C.c_int, [vp, C.POINTER(C.POINTER(C.c_float)), _dp, C.POINTER(LanczosArg), _ip]),
            "cpsgpu_inveigcg": (C.c_int, [vp, _dp, _dp, C.POINTER(CgArg), C.c_int, C.c_int, C.POINTER(_dp), _dp,
                                          C.POINTER(C.POINTER(C.c_float)), _dp, C.c_int, _dp, C.c_int, _ip, _dp]),
            "cpsgpu_minresext": (C.c_int, [vp, _dp, _dp, C.POINTER(_dp), C.POINTER(_dp), C.c_int, _dp]),
            "cpsgpu_bicgstab": (C.c_int, [vp, _dp, _dp, C.c_double, C.c_int, C.POINTER(CgArg), C.POINTER(C.c_int),
                                          _dp]),
            "cpsgpu_fconvert": (C.c_int, [_ip, C.c_int, _dp, C.c_int, C.c_int]),
            "cpsgpu_gconvert": (C.c_int, [_ip, _dp, C.c_int, C.c_int]),
            "cpsgpu_four2five": (C.c_int, [_ip, C.c_int, _dp, _dp, C.c_int, C.c_int, C.c_int]),
            "cpsgpu_five2four": (C.c_int, [_ip, C.c_int, _dp, _dp, C.c_int, C.c_int, C.c_int]),
            "cpsgpu_fconvert_device": (C.c_int, [vp, C.c_int, vp, vp, C.c_int, C.c_int]),
            "cpsgpu_gconvert_device": (C.c_int, [vp, vp, vp, C.c_int, C.c_int]),
            "cpsgpu_four2five_device": (C.c_int, [vp, C.c_int, vp, vp, C.c_int, C.c_int, C.c_int]),
            "cpsgpu_five2four_device": (C.c_int, [vp, C.c_int, vp, vp, C.c_int, C.c_int, C.c_int]),
            "cpsgpu_invcg_multi": (C.c_int, [vp, C.POINTER(_dp), C.POINTER(_dp), C.c_int, C.POINTER(CgArg),
                                             C.POINTER(CgResult)]),
            "cpsgpu_minvcg": (C.c_int, [vp, C.POINTER(_dp), _dp, C.c_double, _dp, C.c_int, _dp, C.c_int, _dp,
                                        C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
            "cpsgpu_get_minvcg_stats": (C.c_int, [vp, C.POINTER(MInvCgStats)]),
            "cpsgpu_field_create": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(vp)]),
            "cpsgpu_field_destroy": (C.c_int, [vp]),
            "cpsgpu_field_upload": (C.c_int, [vp, _dp]),
            "cpsgpu_field_download": (C.c_int, [vp, _dp]),
            "cpsgpu_field_gaussian": (C.c_int, [vp, C.c_ulonglong]),
            "cpsgpu_dslash_field": (C.c_int, [vp, vp, vp, C.c_int, C.c_int]),
            "cpsgpu_lattice_set_t_partition": (C.c_int, [vp, C.c_int, C.c_int]),
            "cpsgpu_dd_face_bytes": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_size_t)]),
            "cpsgpu_dslash_dd_pack": (C.c_int, [vp, vp, C.c_int, C.c_int, vp, vp]),
            "cpsgpu_dslash_dd": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, vp, vp]),
            "cpsgpu_dslash_dd_interior": (C.c_int, [vp, vp, vp, C.c_int, C.c_int]),
            "cpsgpu_lattice_set_stream": (C.c_int, [vp, vp]),
            "cpsgpu_finalize": (C.c_int, []),
            "cpsgpu_field_dot_device": (C.c_int, [vp, vp, vp]),
            "cpsgpu_field_axpby_device": (C.c_int, [vp, vp, C.c_double, vp, vp]),
            "cpsgpu_dslash_dd_boundary": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, vp, vp]),
            "cpsgpu_field_axpby": (C.c_int, [vp, C.c_double, vp, vp]),
            "cpsgpu_field_dot": (C.c_int, [vp, vp, _dp, _dp]),
            "cpsgpu_mdagm_field": (C.c_int, [vp, vp, vp]),
            "cpsgpu_invcg_field": (C.c_int, [vp, vp, vp, C.POINTER(CgArg), C.POINTER(CgResult)]),
            "cpsgpu_solve_batch": (C.c_int, [C.c_int, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(CgArg),
                                             C.POINTER(CgResult)]),
            "cpsgpu_autotune": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.c_int)]),
            "cpsgpu_dirac_set_pc_type": (C.c_int, [vp, C.c_int]),
            "cpsgpu_dirac_get_pc_type": (C.c_int, [vp, C.POINTER(C.c_int)]),
            "cpsgpu_get_hop_shape": (C.c_int, [vp, C.c_int] + [C.POINTER(C.c_int)] * 4),
            "cpsgpu_set_hop_shape": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "cpsgpu_time_dslash": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp]),
            "cpsgpu_time_mdagm": (C.c_int, [vp, C.c_int, C.c_int, _dp, _dp]),
            "cpsgpu_time_m5inv": (C.c_int, [vp, C.c_int, C.c_int, _dp, _dp]),
            "cpsgpu_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(vp)]),
            "cpsgpu_host_free": (C.c_int, [vp]),
            "cpsgpu_gen_gauge": (C.c_int, [C.POINTER(C.c_int), C.c_ulonglong, C.c_double, _dp]),
            "cpsgpu_gen_gaussian": (C.c_int, [_dp, C.c_long, C.c_ulonglong, C.c_uint]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> int:
    if rc != 0:
        msg = lib().cpsgpu_last_error().decode(errors="replace")
        raise CpsGpuError(f"cpsgpu error {rc}: {msg}")
    return rc


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def ints(v) -> C.Array:
    return (C.c_int * len(v))(*v)


def declared_symbols(header: Path) -> list[str]:
    """Function names declared in a C header (``cpsgpu_*(``)."""
    import re

    text = header.read_text()
    return sorted(set(re.findall(r"\b(cpsgpu_[a-z0-9_]+)\s*\(", text)))
