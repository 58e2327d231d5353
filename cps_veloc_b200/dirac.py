"""Python mirror of the reference's operator and solver interface for the
fermion-solve hot path, on top of the C ABI.

Names and argument meanings follow the reference's C++ classes so callers
(and the parity tests) read like CPS code:

  Lattice            geometry + resident gauge field (GJP geometry, the
                     Lattice gauge field, BondCond as a per-direction sign)
  DiracOpWilson      d_op_wilson.C: Dslash, MatPc, MatPcDag, MatPcDagMatPc,
                     InvCg, MInvCG
  DiracOpDwf         d_op_dwf.C: same set on the 5D-preconditioned field
  DiracOpMobius      d_op_mobius.C: same set (SYM2), plus Dslash4 / M5inv

Vectors are numpy float64 arrays in CPS storage order (include/cpsgpu.h).
Errors raise CpsGpuError instead of exiting the process as ERR.General does.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi as A
from ._abi import check, dptr, lib


def gen_gauge(node_sites, seed: int = 20261203, width: float = 0.3) -> np.ndarray:
    """Seeded SU(3) field U = exp(i width H), WILSON order, no boundary signs."""
    vol = int(np.prod(node_sites))
    u = np.empty(vol * 4 * 18)
    check(lib().cpsgpu_gen_gauge(A.ints(node_sites), seed, width, dptr(u)))
    return u


def gen_gaussian(n: int, seed: int = 20261203, stream: int = 0) -> np.ndarray:
    out = np.empty(n)
    check(lib().cpsgpu_gen_gaussian(dptr(out), n, seed, stream))
    return out


StrOrd = A.StrOrd


def fconvert(node_sites, ls: int, f: np.ndarray, to: int, frm: int) -> None:
    """FwilsonTypes / FdwfBase::Fconvert (CANONICAL <-> WILSON) in place"""
    _inplace(f, 24 * ls * int(np.prod(node_sites)))
    check(lib().cpsgpu_fconvert(A.ints(node_sites), ls, dptr(f), to, frm))


def gconvert(node_sites, u: np.ndarray, to: int, frm: int) -> None:
    """Lattice::Convert of the gauge field (CANONICAL <-> WILSON) in place"""
    _inplace(u, 72 * int(np.prod(node_sites)))
    check(lib().cpsgpu_gconvert(A.ints(node_sites), dptr(u), to, frm))


def four2five(node_sites, ls: int, four: np.ndarray, s_u: int, s_l: int, ncb: int = 2) -> np.ndarray:
    """FdwfBase::Ffour2five: the 5D field with the 4D one on the walls"""
    v4 = int(np.prod(node_sites)) * ncb // 2
    four = np.ascontiguousarray(four, dtype=np.float64)
    if four.size != 24 * v4:
        raise ValueError("4D field size")
    five = np.empty(24 * ls * v4)
    check(lib().cpsgpu_four2five(A.ints(node_sites), ls, dptr(five), dptr(four), s_u, s_l, ncb))
    return five


def five2four(node_sites, ls: int, five: np.ndarray, s_u: int, s_l: int, ncb: int = 2) -> np.ndarray:
    """FdwfBase::Ffive2four: the 4D field read off the walls"""
    v4 = int(np.prod(node_sites)) * ncb // 2
    five = np.ascontiguousarray(five, dtype=np.float64)
    if five.size != 24 * ls * v4:
        raise ValueError("5D field size")
    four = np.empty(24 * v4)
    check(lib().cpsgpu_five2four(A.ints(node_sites), ls, dptr(four), dptr(five), s_u, s_l, ncb))
    return four


def _header(h) -> dict:
    name = {v: k for k, v in A.FP_FORMATS.items()}
    return {"dims": tuple(h.dims), "recon_row_3": bool(h.recon_row_3), "floating_point": name.get(h.fp_format),
            "plaquette": h.plaquette, "link_trace": h.link_trace, "checksum": h.checksum,
            "sequence_number": h.sequence_number, "ensemble_id": h.ensemble_id.decode(),
            "ensemble_label": h.ensemble_label.decode(), "creator": h.creator.decode()}


def nersc_read(path, node_sites):
    """ReadLatticeParallel::read of a NERSC archive: (CANONICAL links, header)"""
    u = np.empty(72 * int(np.prod(node_sites)))
    h = A.NerscHeader()
    check(lib().cpsgpu_nersc_read(str(path).encode(), A.ints(node_sites), dptr(u), C.byref(h)))
    return u, _header(h)


def nersc_write(path, node_sites, u, recon_row_3=True, floating_point="IEEE64BIG", ensemble_id="",
                ensemble_label="", sequence_number=0, creator=""):
    """WriteLatticeParallel::write of a CANONICAL field; returns the header written"""
    u = np.ascontiguousarray(u, dtype=np.float64)
    if u.size != 72 * int(np.prod(node_sites)):
        raise ValueError("gauge field size")
    meta = A.NerscHeader()
    meta.ensemble_id, meta.ensemble_label, meta.creator = (s.encode()[:127] for s in
                                                           (ensemble_id, ensemble_label, creator))
    meta.sequence_number = sequence_number
    out = A.NerscHeader()
    check(lib().cpsgpu_nersc_write(str(path).encode(), A.ints(node_sites), dptr(u), 1 if recon_row_3 else 0,
                                   A.FP_FORMATS[floating_point], C.byref(meta), C.byref(out)))
    return _header(out)


def _inplace(a, n):
    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and a.size == n):
        raise TypeError(f"expected a C-contiguous float64 array of {n} reals (converted in place)")


class Lattice:
    def __init__(self, node_sites, bc=(1, 1, 1, -1)):
        self.node_sites = tuple(int(x) for x in node_sites)
        self.bc = tuple(int(b) for b in bc)
        self.vol = int(np.prod(self.node_sites))
        h = C.c_void_p()
        check(lib().cpsgpu_lattice_create(A.ints(self.node_sites), A.ints(self.bc), C.byref(h)))
        self._h = h

    def import_gauge(self, u: np.ndarray, signs_applied: bool = False) -> None:
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.size != self.vol * 72:
            raise ValueError("gauge field must hold vol*4*18 reals")
        check(lib().cpsgpu_import_gauge(self._h, dptr(u), 1 if signs_applied else 0))

    def gauge_info(self):
        e = C.c_double()
        r = C.c_int()
        check(lib().cpsgpu_gauge_info(self._h, C.byref(e), C.byref(r)))
        return e.value, bool(r.value)

    def set_link_reals(self, prec: int, reals: int) -> None:
        """stored link form of the FP32/FP16 operators: 12 or 18 reals, or
        LINKS_F32_12 / LINKS_F32_18 (FP32 links for the FP16 operator)"""
        check(lib().cpsgpu_set_link_reals(self._h, prec, reals))

    def link_reals(self, prec: int) -> int:
        r = C.c_int()
        check(lib().cpsgpu_get_link_reals(self._h, prec, C.byref(r)))
        return r.value

    def eigencache_clear(self):
        """drop every eigenvector cache of this lattice (EigenCacheListCleanup)"""
        check(lib().cpsgpu_eigencache_clear(self._h))

    def plaquette(self):
        """(SumReTrPlaq / (18 V), sum Re tr U / (12 V)) of the resident links"""
        p, t = C.c_double(), C.c_double()
        check(lib().cpsgpu_gauge_plaquette(self._h, C.byref(p), C.byref(t)))
        return p.value, t.value

    def load_nersc(self, path, check_precision=0.01):
        """ReadLatticeParallel::read into this lattice; returns (plaquette, header)"""
        h, p = A.NerscHeader(), C.c_double()
        check(lib().cpsgpu_lattice_load_nersc(self._h, str(path).encode(), check_precision, C.byref(h), C.byref(p)))
        return p.value, _header(h)

    def synchronize(self):
        check(lib().cpsgpu_synchronize(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().cpsgpu_lattice_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class CgResult:
    iterations: int
    status: int
    true_res: float
    reliable_updates: int
    seconds: float
    kernels: int = 0


class _DiracOp:
    kind = A.WILSON

    def __init__(self, lat: Lattice, mass: float, ls: int = 1, m5: float = 1.8, b: float = 1.0, c: float = 0.0,
                 a5_inv: float = 1.0):
        self.lat = lat
        arg = A.DiracArg(self.kind, ls, mass, m5, b, c, a5_inv)
        h = C.c_void_p()
        check(lib().cpsgpu_dirac_create(lat._h, C.byref(arg), C.byref(h)))
        self._h = h
        self.ls = ls if self.kind != A.WILSON else 1
        self.mass = mass
        k, kc = C.c_double(), C.c_double()
        check(lib().cpsgpu_dirac_info(h, C.byref(k), C.byref(kc)))
        self.kappa, self.kappa_c = k.value, kc.value

    @property
    def f_size(self) -> int:
        """reals in one preconditioned vector (InvCgShift's f_size_cb)"""
        return 24 * self.ls * self.lat.vol // 2

    def _vec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != self.f_size:
            raise ValueError(f"vector must hold {self.f_size} reals")
        return x

    def _full(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != 2 * self.f_size:
            raise ValueError(f"full vector must hold {2 * self.f_size} reals")
        return x

    def Mat(self, inp) -> np.ndarray:
        """DiracOp*::Mat on a full vector (both checkerboards, the reference's order)"""
        inp = self._full(inp)
        out = np.empty_like(inp)
        check(lib().cpsgpu_mat(self._h, dptr(out), dptr(inp), 0))
        return out

    def MatDag(self, inp) -> np.ndarray:
        inp = self._full(inp)
        out = np.empty_like(inp)
        check(lib().cpsgpu_mat(self._h, dptr(out), dptr(inp), 1))
        return out

    def MatHerm(self, inp) -> np.ndarray:
        inp = self._full(inp)
        out = np.empty_like(inp)
        check(lib().cpsgpu_mat_herm(self._h, dptr(out), dptr(inp)))
        return out

    def Dslash(self, inp, cb: int, dag: int = 0, prec: int = A.DOUBLE) -> np.ndarray:
        inp = self._vec(inp)
        out = np.empty_like(inp)
        check(lib().cpsgpu_dslash(self._h, dptr(out), dptr(inp), cb, dag, prec))
        return out

    def MatPc(self, inp, prec: int = A.DOUBLE) -> np.ndarray:
        inp = self._vec(inp)
        out = np.empty_like(inp)
        check(lib().cpsgpu_matpc(self._h, dptr(out), dptr(inp), 0, prec))
        return out

    def MatPcDag(self, inp, prec: int = A.DOUBLE) -> np.ndarray:
        inp = self._vec(inp)
        out = np.empty_like(inp)
        check(lib().cpsgpu_matpc(self._h, dptr(out), dptr(inp), 1, prec))
        return out

    def MatPcDagMatPc(self, inp, prec: int = A.DOUBLE):
        """returns (M^+ M in, |M in|^2) as DiracOp::MatPcDagMatPc(out, in, &dot)"""
        inp = self._vec(inp)
        out = np.empty_like(inp)
        dot = C.c_double()
        check(lib().cpsgpu_matpc_dag_matpc(self._h, dptr(out), dptr(inp), C.byref(dot), prec))
        return out, dot.value

    def _cg_arg(self, stop_rsd, max_num_iter, src_norm_sq, shift, precision, delta, chunk, use_graph):
        a = A.CgArg()
        lib().cpsgpu_cg_arg_default(C.byref(a))
        a.stop_rsd = stop_rsd
        a.max_num_iter = max_num_iter
        a.src_norm_sq = src_norm_sq
        a.shift = shift
        a.precision = precision
        a.delta = delta
        a.chunk = chunk
        a.use_graph = 1 if use_graph else 0
        return a

    def InvCg(self, sol, src, stop_rsd=1e-8, max_num_iter=10000, src_norm_sq=0.0, shift=0.0,
              precision=A.DOUBLE, delta=0.0, chunk=8, use_graph=True) -> CgResult:
        """DiracOp::InvCg(out, in, src_norm_sq, true_res): sol is the initial guess, updated in place."""
        src = self._vec(src)
        if not (isinstance(sol, np.ndarray) and sol.dtype == np.float64 and sol.flags.c_contiguous):
            raise TypeError("sol must be a C-contiguous float64 array (updated in place)")
        self._vec(sol)
        a = self._cg_arg(stop_rsd, max_num_iter, src_norm_sq, shift, precision, delta, chunk, use_graph)
        r = A.CgResult()
        check(lib().cpsgpu_invcg(self._h, dptr(sol), dptr(src), C.byref(a), C.byref(r)))
        return CgResult(r.iterations, r.status, r.true_res, r.reliable_updates, r.seconds, r.kernels)

    def MatInv(self, out, src, stop_rsd=1e-8, max_num_iter=10000, precision=A.DOUBLE, delta=0.0, chunk=8,
               use_graph=True, inverter=A.INV_CG, fname_eigen=None, neig=0) -> CgResult:
        """DiracOp*::MatInv(out, in, true_res): both checkerboards (2 * f_size
        reals; Wilson/DWF [odd | even], Mobius [even | odd]), out updated in
        place.  inverter (CgArg.Inverter): INV_CG (out's CG checkerboard is the
        initial guess), INV_LOWMODEAPPROX (the low-mode approximation from
        the cache fname_eigen of neig vectors instead of CG) or
        INV_CG_LOWMODE_DEFL (that approximation as CG's initial guess)."""
        src = np.ascontiguousarray(src, dtype=np.float64)
        if src.size != 2 * self.f_size:
            raise ValueError(f"vectors must hold {2 * self.f_size} reals (both checkerboards)")
        if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                and out.size == src.size):
            raise TypeError("out must be a C-contiguous float64 array like src (updated in place)")
        a = self._cg_arg(stop_rsd, max_num_iter, 0.0, 0.0, precision, delta, chunk, use_graph)
        r = A.CgResult()
        if inverter == A.INV_CG:
            check(lib().cpsgpu_matinv(self._h, dptr(out), dptr(src), C.byref(a), C.byref(r)))
        else:
            check(lib().cpsgpu_matinv_lowmode(self._h, dptr(out), dptr(src), C.byref(a), inverter,
                                              fname_eigen.encode(), neig, C.byref(r)))
        return CgResult(r.iterations, r.status, r.true_res, r.reliable_updates, r.seconds, r.kernels)

    def EigenCacheLoad(self, name, evecs, evals):
        """fill the named eigenvector cache (EigenCache, eigen_container.h)
        on the device: evecs float32 vectors of f_size reals, evals float64"""
        evecs = [np.ascontiguousarray(v, dtype=np.float32) for v in evecs]
        for v in evecs:
            if v.size != self.f_size:
                raise ValueError(f"eigenvectors must hold {self.f_size} reals")
        evals = np.ascontiguousarray(evals, dtype=np.float64)
        if evals.size != len(evecs):
            raise ValueError("one eigenvalue per eigenvector")
        pv = (C.POINTER(C.c_float) * max(1, len(evecs)))(*[v.ctypes.data_as(C.POINTER(C.c_float)) for v in evecs])
        check(lib().cpsgpu_eigencache_load(self._h, name.encode(), len(evecs), pv, dptr(evals)))

    def InvLowModeApprox(self, out, src, fname_eigen, neig, ritz_mat_oper=A.RITZ_MATPCDAG_MATPC):
        """DiracOp::InvLowModeApprox (inv_lowmode_approx.C:272-512): out[i]
        (float64, in place) = sum_k <v_k, src[i]> / lambda_k v_k over the
        cache fname_eigen of neig vectors"""
        src = [self._vec(x) for x in src]
        for x in out:
            _inplace(x, self.f_size)
        if len(out) != len(src):
            raise ValueError("one output per source")
        po = (A._dp * max(1, len(out)))(*[dptr(x) for x in out])
        pi = (A._dp * max(1, len(src)))(*[dptr(x) for x in src])
        check(lib().cpsgpu_inv_lowmode_approx(self._h, po, pi, len(src), fname_eigen.encode(), neig, ritz_mat_oper))

    def CalcHmdForceVecs(self, chi):
        """DiracOp*::CalcHmdForceVecs: returns (f_out, f_in), full fields in
        WILSON order: (chi, D chi) and (-kappa^2 MatPc chi, D^dag of it)"""
        chi = self._vec(chi)
        f_out, f_in = np.empty(2 * self.f_size), np.empty(2 * self.f_size)
        check(lib().cpsgpu_calc_hmd_force_vecs(self._h, dptr(f_out), dptr(f_in), dptr(chi)))
        return f_out, f_in

    def EvolveMomFforce(self, mom, chi, dt):
        """Fwilson / FdwfBase::EvolveMomFforce: mom (CANONICAL Matrix field,
        4 * vol * 18 reals, updated in place) += the fermion force of chi;
        returns the reference's ForceArg as (L1, L2, Linf)"""
        chi = self._vec(chi)
        _inplace(mom, 4 * self.lat.vol * 18)
        fa = A.ForceArg()
        check(lib().cpsgpu_evolve_mom_fforce(self._h, dptr(mom), dptr(chi), dt, C.byref(fa)))
        return fa.L1, fa.L2, fa.Linf

    def RHMC_EvolveMomFforce(self, mom, sol, alpha, dt, force_measure=False):
        """Fwilson / FdwfBase::RHMC_EvolveMomFforce over the poles sol[k] with
        steps dt * alpha[k]; returns (L1, L2, Linf) of the summed force when
        force_measure, else zeros (as the reference)"""
        _inplace(mom, 4 * self.lat.vol * 18)
        sols = [self._vec(x) for x in sol]
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        if alpha.size != len(sols):
            raise ValueError("one alpha per pole")
        arr = (A._dp * max(1, len(sols)))(*[dptr(x) for x in sols])
        fa = A.ForceArg()
        check(lib().cpsgpu_rhmc_evolve_mom_fforce(self._h, dptr(mom), arr, len(sols), dptr(alpha), dt,
                                                  1 if force_measure else 0, C.byref(fa)))
        return fa.L1, fa.L2, fa.Linf

    def Ritz(self, psi_all, RsdR_a=1e-10, RsdR_r=1e-8, Rsdlam=1e-10, Cutl_zero=0.0, n_renorm=10, Kalk_Sim=0,
             N_min=0, N_max=1000, Cv_fact=0.0, MaxCG=10000, ProjApsiP=0, neg=False):
        """DiracOp::Ritz (ritz.C:152-532) on MatPcDagMatPc (its negative when
        neg): the last of psi_all (updated in place) becomes the eigenvector
        orthogonal to the others; returns (iterations, lambda).  Raises after
        MaxCG iterations, as the reference exits."""
        for x in psi_all:
            _inplace(x, self.f_size)
        a = A.RitzArg(RsdR_a, RsdR_r, Rsdlam, Cutl_zero, Cv_fact, n_renorm, Kalk_Sim, N_min, N_max, MaxCG,
                      ProjApsiP, 1 if neg else 0)
        pv = (A._dp * len(psi_all))(*[dptr(x) for x in psi_all])
        lam, k = C.c_double(), C.c_int()
        rc = lib().cpsgpu_ritz(self._h, pv, len(psi_all), C.byref(a), C.byref(lam), C.byref(k))
        if rc == A.MAX_ITER:
            raise A.CpsGpuError(f"too many CG/Ritz iterations: {k.value}")
        check(rc)
        return k.value, lam.value

    def RitzEig(self, psi, RsdR_a=1e-10, RsdR_r=1e-8, Rsdlam=1e-10, Cv_fact=0.1, n_renorm=10, Kalk_Sim=1,
                N_min=5, N_max=50, MaxCG=10000, ProjApsiP=0, N_KS_max=50, neg=False):
        """DiracOpWilsonTypes::RitzEig (eigen_wilson.C:89-586) with RitzMatOper
        MATPCDAG_MATPC (NEG_MATPCDAG_MATPC when neg): psi (start vectors,
        updated in place) become the len(psi) lowest eigenvectors; returns
        (total Ritz iterations, lambda_H, valid_eig) with lambda_H of
        2 len(psi) entries (eigenvalues, then the Ritz / Kalkreuter-Simma
        ones).  Raises when a Ritz call, the sweeps or a Jacobi call run out."""
        for x in psi:
            _inplace(x, self.f_size)
        a = A.RitzArg(RsdR_a, RsdR_r, Rsdlam, 0.0, Cv_fact, n_renorm, Kalk_Sim, N_min, N_max, MaxCG, ProjApsiP,
                      1 if neg else 0)
        pv = (A._dp * len(psi))(*[dptr(x) for x in psi])
        lam = np.zeros(2 * len(psi))
        valid = (C.c_int * len(psi))()
        k = C.c_int()
        rc = lib().cpsgpu_ritz_eig(self._h, pv, len(psi), C.byref(a), N_KS_max, dptr(lam), valid, C.byref(k))
        if rc == A.MAX_ITER:
            raise A.CpsGpuError(f"RitzEig stopped with code {k.value}")
        check(rc)
        return k.value, lam, np.array(valid[:])

    def ImpResLanczos(self, V, nk, nt, np_, Npol, params, stop_residual=1e-6, maxiters=100, conv_check=1,
                      eigen_shift=0.0, RitzMat_lanczos=A.RITZ_MATPCDAG_MATPC, RitzMat_convcheck=A.RITZ_MATPCDAG_MATPC):
        """DiracOp::ImpResLanczos (lanczos.C:193-745) with the Chebyshev filter
        T_Npol of DiracOpDwf / DiracOpMobius::RitzMat (d_op_dwf.C:852-960):
        V (nk + np float32 vectors, V[0] the start; updated in place) become
        the Ritz vectors; returns (restarts, alpha) with alpha[:nt] the
        eigenvalues of MatPcDagMatPc."""
        if len(V) != nk + np_:
            raise ValueError("V must hold nk + np vectors")
        for x in V:
            if not (isinstance(x, np.ndarray) and x.dtype == np.float32 and x.flags.c_contiguous
                    and x.size == self.f_size):
                raise TypeError("Lanczos vectors must be C-contiguous float32 arrays of the fermion size")
        a = A.LanczosArg(RitzMat_lanczos, RitzMat_convcheck, nk, nt, np_, eigen_shift, stop_residual, maxiters,
                         conv_check, Npol, (C.c_double * 2)(*params))
        pv = (C.POINTER(C.c_float) * len(V))(*[x.ctypes.data_as(C.POINTER(C.c_float)) for x in V])
        alpha = np.zeros(len(V))
        it = C.c_int()
        check(lib().cpsgpu_imp_res_lanczos(self._h, pv, dptr(alpha), C.byref(a), C.byref(it)))
        return it.value, alpha

    def Jacobi(self, psi, lam, off_diag, Toler=1e-10, N_max=50):
        """DiracOp::Jacobi (jacobi.C:48-268): psi and lam (float64, in place)
        rotated and sorted; off_diag: complex array of N(N-1)/2, zeroed in
        place; returns the sweep count"""
        for x in psi:
            _inplace(x, self.f_size)
        _inplace(lam, len(psi))
        if not (isinstance(off_diag, np.ndarray) and off_diag.dtype == np.complex128 and off_diag.flags.c_contiguous):
            raise TypeError("off_diag must be a C-contiguous complex128 array")
        pv = (A._dp * len(psi))(*[dptr(x) for x in psi])
        k = C.c_int()
        rc = lib().cpsgpu_jacobi(self._h, pv, len(psi), dptr(lam), off_diag.ctypes.data_as(A._dp), Toler, N_max,
                                 C.byref(k))
        if rc == A.MAX_ITER:
            raise A.CpsGpuError("too many Jacobi iterations")
        check(rc)
        return k.value

    def InvEigCg(self, sol, src, nev=0, m=0, stop_rsd=1e-8, max_num_iter=10000, U=None, invH=None, restart=()):
        """DiracOp::InvEigCg (inv_eig_cg.C:129-635): sol (in place) solves
        MatPcDagMatPc sol = src; returns (iterations, true_res, V, M) with V the
        m eigCG vectors (the first 2 nev: Ritz vectors) and M the 2 nev Ritz
        values.  U: deflation vectors (float32), invH their inverse projected
        matrix (complex, def_len x def_len); restart: the relative residuals of
        the deflated restarts."""
        src = self._vec(src)
        _inplace(sol, self.f_size)
        V = [np.empty(self.f_size) for _ in range(m if nev > 0 else 0)]
        M = np.zeros(max(2 * nev, 1))
        U = [np.ascontiguousarray(u, dtype=np.float32) for u in (U or [])]
        for u in U:
            if u.size != self.f_size:
                raise ValueError("deflation vector size")
        def_len = len(U)
        ih = np.ascontiguousarray(invH if invH is not None else np.zeros((max(def_len, 1),) * 2),
                                  dtype=np.complex128)
        if def_len and ih.shape != (def_len, def_len):
            raise ValueError("invH must be def_len x def_len")
        ihr = ih.view(np.float64).ravel()
        rs = np.ascontiguousarray(list(restart) or [0.0], dtype=np.float64)
        a = self._cg_arg(stop_rsd, max_num_iter, 0.0, 0.0, A.DOUBLE, 0.0, 8, True)
        pv = (A._dp * max(1, len(V)))(*([dptr(x) for x in V] or [None]))
        fp = C.POINTER(C.c_float)
        pu = (fp * max(1, def_len))(*([u.ctypes.data_as(fp) for u in U] or [None]))
        it, tr = C.c_int(), C.c_double()
        check(lib().cpsgpu_inveigcg(self._h, dptr(sol), dptr(src), C.byref(a), nev, m, pv, dptr(M), pu, dptr(ihr),
                                    def_len, dptr(rs), len(restart), C.byref(it), C.byref(tr)))
        return it.value, tr.value, V, M[:2 * nev]

    def MinResExt(self, psi, phi, v, vm):
        """DiracOp::MinResExt: psi (updated in place) = the chronological guess
        from the previous solutions v (orthonormalised in place); vm[i] =
        MatPcDagMatPc v[i]; returns |phi - A psi| / |phi|"""
        phi = self._vec(phi)
        _inplace(psi, self.f_size)
        for x in list(v) + list(vm):
            _inplace(x, self.f_size)
        if len(v) != len(vm):
            raise ValueError("v and vm must have the same length")
        n = max(1, len(v))
        pv = (A._dp * n)(*[dptr(x) for x in v])
        pm = (A._dp * n)(*[dptr(x) for x in vm])
        err = C.c_double()
        check(lib().cpsgpu_minresext(self._h, dptr(psi), dptr(phi), pv, pm, len(v), C.byref(err)))
        return err.value

    def FmatEvlInv(self, f_out, f_in, stop_rsd=1e-8, max_num_iter=10000, precision=A.DOUBLE):
        """Fwilson / FdwfBase::FmatEvlInv (f_dwf_base.C:189-214): InvCg of
        MatPcDagMatPc f_out = f_in from the guess in f_out; returns
        (iterations, true_res) as the reference returns iter and sets
        cg_arg->true_rsd"""
        r = self.InvCg(f_out, f_in, stop_rsd=stop_rsd, max_num_iter=max_num_iter, precision=precision)
        return r.iterations, r.true_res

    def FmatEvlMInv(self, f_out, f_in, shift, stop_rsd, type_=A.MS_MULTI, alpha=None, precision=A.DOUBLE):
        """FdwfBase::FmatEvlMInv (f_dwf_base.C:232-275): MInvCG with the source
        norm computed here and each shift's stop_rsd; returns (iterations,
        true_rsd per shift) as the reference writes cg_arg[s]->true_rsd"""
        f_in = self._vec(f_in)
        rs = np.array(stop_rsd, dtype=np.float64).copy()
        k = self.MInvCG(f_out, f_in, float(f_in @ f_in), shift, rs, type=type_, alpha=alpha, precision=precision)
        return k, rs

    def BiCGstab(self, psi, chi, n=1, chi_norm=0.0, stop_rsd=1e-8, max_num_iter=10000):
        """DiracOpWilsonTypes::BiCGstab(psi, chi, chi_norm, n, true_res) on MatPc:
        psi (initial guess) updated in place; returns (k, true_res) as the
        reference does (true_res absolute, 0 unless converged)"""
        chi = self._vec(chi)
        if not (isinstance(psi, np.ndarray) and psi.dtype == np.float64 and psi.flags.c_contiguous):
            raise TypeError("psi must be a C-contiguous float64 array (updated in place)")
        self._vec(psi)
        a = self._cg_arg(stop_rsd, max_num_iter, 0.0, 0.0, A.DOUBLE, 0.0, 8, True)
        k, tr = C.c_int(), C.c_double()
        check(lib().cpsgpu_bicgstab(self._h, dptr(psi), dptr(chi), chi_norm, n, C.byref(a), C.byref(k), C.byref(tr)))
        return k.value, tr.value

    def InvCgMulti(self, sols, srcs, stop_rsd=1e-8, max_num_iter=10000, precision=A.DOUBLE, delta=0.0,
                   chunk=8, use_graph=True):
        n = len(srcs)
        srcs = [self._vec(s) for s in srcs]
        for s in sols:
            self._vec(s)
        sp = (A._dp * n)(*[dptr(s) for s in sols])
        bp = (A._dp * n)(*[dptr(s) for s in srcs])
        a = self._cg_arg(stop_rsd, max_num_iter, 0.0, 0.0, precision, delta, chunk, use_graph)
        res = (A.CgResult * n)()
        check(lib().cpsgpu_invcg_multi(self._h, sp, bp, n, C.byref(a), res))
        return [CgResult(r.iterations, r.status, r.true_res, r.reliable_updates, r.seconds, r.kernels) for r in res]

    def MInvCG(self, psi, chi, chi_norm, shifts, rsdcg, type=A.MS_MULTI, alpha=None, max_num_iter=10000,
               precision=A.DOUBLE, refine=True):
        """DiracOp::MInvCG: psi list updated in place; rsdcg (np array) overwritten; returns k."""
        chi = self._vec(chi)
        n = len(shifts)
        sh = np.ascontiguousarray(shifts, dtype=np.float64)
        if not (isinstance(rsdcg, np.ndarray) and rsdcg.dtype == np.float64):
            raise TypeError("rsdcg must be a float64 array")
        al = np.ascontiguousarray(alpha if alpha is not None else np.ones(n), dtype=np.float64)
        pp = (A._dp * len(psi))(*[dptr(p) for p in psi])
        k = C.c_int()
        check(lib().cpsgpu_minvcg(self._h, pp, dptr(chi), chi_norm, dptr(sh), n, dptr(rsdcg), type, dptr(al),
                                  max_num_iter, precision, 1 if refine else 0, C.byref(k)))
        return k.value

    def minvcg_stats(self) -> dict:
        """phases of the last MInvCG: upload, recurrence, refine, download
        wall seconds and the refinement's iterations (max, sum)"""
        st = A.MInvCgStats()
        check(lib().cpsgpu_get_minvcg_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in A.MInvCgStats._fields_}

    def autotune(self, prec=A.DOUBLE, nrhs=1) -> int:
        t = C.c_int()
        check(lib().cpsgpu_autotune(self._h, prec, nrhs, C.byref(t)))
        return t.value

    def rhs_tile(self, prec=A.DOUBLE, nrhs=1) -> int:
        """right-hand sides per hop tile a batched launch of nrhs uses"""
        t = C.c_int()
        check(lib().cpsgpu_get_rhs_tile(self._h, prec, nrhs, C.byref(t)))
        return t.value

    def set_rhs_tile(self, prec: int, tile: int) -> None:
        check(lib().cpsgpu_set_rhs_tile(self._h, prec, tile))

    # block traversal orders of the hop launches (cpsgpu_set_hop_shape)
    ORDER_SLICES, ORDER_SITES = 0, 1

    def hop_shape(self, prec=A.DOUBLE) -> tuple:
        """(sites, slices, slices per thread, order) of the non-mixing hop launches"""
        a, b, c, o = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().cpsgpu_get_hop_shape(self._h, prec, C.byref(a), C.byref(b), C.byref(c), C.byref(o)))
        return a.value, b.value, c.value, o.value

    def set_hop_shape(self, prec: int, sites: int, slices: int, slices_per_thread: int = 1,
                      order: int = 0) -> None:
        check(lib().cpsgpu_set_hop_shape(self._h, prec, sites, slices, slices_per_thread, order))

    def close(self):
        if getattr(self, "_h", None):
            lib().cpsgpu_dirac_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DiracOpWilson(_DiracOp):
    kind = A.WILSON

    def __init__(self, lat: Lattice, mass: float):
        super().__init__(lat, mass, ls=1)


class DiracOpDwf(_DiracOp):
    kind = A.DWF

    def __init__(self, lat: Lattice, mass: float, ls: int, m5: float = 1.8, a5_inv: float = 1.0):
        super().__init__(lat, mass, ls=ls, m5=m5, a5_inv=a5_inv)


class DiracOpMobius(_DiracOp):
    kind = A.MOBIUS
    # GJP.ZMobius_PC_Type values (enum ZMobiusPCType, dwf.h:42-48)
    PC_ORIG, PC_SYM1, PC_SYM2, PC_SYM1_MIT, PC_SYM2_MIT, PC_SYM3 = range(6)

    def __init__(self, lat: Lattice, mass: float, ls: int, m5: float = 1.8, b: float = 1.5, c: float = 0.5,
                 a5_inv: float = 1.0, pc_type: int = 2):
        super().__init__(lat, mass, ls=ls, m5=m5, b=b, c=c, a5_inv=a5_inv)
        if pc_type != self.PC_SYM2:
            self.set_pc_type(pc_type)

    def set_pc_type(self, pc_type: int) -> None:
        """the preconditioning of MatPc (GJP.ZMobius_PC_Type; SYM2 the default)"""
        check(lib().cpsgpu_dirac_set_pc_type(self._h, pc_type))

    @property
    def pc_type(self) -> int:
        v = C.c_int()
        check(lib().cpsgpu_dirac_get_pc_type(self._h, C.byref(v)))
        return v.value

    MIX_DEFAULT, MIX_TENSOR_CORES, MIX_SHARED, MIX_REG = 0, 1, 2, 3
    MIX_BULK = MIX_DEFAULT  # FP16 fields: staged by bulk copies where it applies

    def set_mix_impl(self, impl) -> None:
        """the kernel of the standalone Ls x Ls mixings: MIX_DEFAULT (0: FP16
        fields the register-tiled arithmetic on input tiles staged by bulk
        asynchronous copies, else as MIX_REG), MIX_TENSOR_CORES (1, FP16
        fields on the tensor cores), MIX_SHARED (2, the shared-memory
        CUDA-core kernel) or MIX_REG (3, register-tiled CUDA cores);
        True / False mean 1 / 0"""
        impl = int(impl) if not isinstance(impl, bool) else (1 if impl else 0)
        check(lib().cpsgpu_set_mix_impl(self._h, impl))

    def MatPcDagMatPcShift(self, inp, mu: float, prec: int = A.DOUBLE):
        """DiracOpMobius::MatPcDagMatPcShift (eigen_shift mu): returns
        (M^+ M in - 2 mu R g5 M in + mu^2 in, |M in|^2)"""
        inp = self._vec(inp)
        out = np.empty_like(inp)
        dot = C.c_double()
        check(lib().cpsgpu_matpc_dag_matpc_shift(self._h, dptr(out), dptr(inp), mu, C.byref(dot), prec))
        return out, dot.value

    def Dslash(self, inp, cb, dag=0, prec=A.DOUBLE):
        raise NotImplementedError("Mobius: use Dslash4 (zmobius_dslash_4)")

    def set_zmobius(self, b, c) -> None:
        """complex per-slice b_s, c_s (DiracOpZMobius)"""
        b = np.ascontiguousarray(np.asarray(b, dtype=np.complex128).view(np.float64))
        c = np.ascontiguousarray(np.asarray(c, dtype=np.complex128).view(np.float64))
        if b.size != 2 * self.ls or c.size != 2 * self.ls:
            raise ValueError("b and c need Ls complex values")
        check(lib().cpsgpu_dirac_set_zmobius(self._h, dptr(b), dptr(c)))

    def Dslash4(self, inp, cb: int, dag: int = 0, prec: int = A.DOUBLE) -> np.ndarray:
        inp = self._vec(inp)
        out = np.empty_like(inp)
        check(lib().cpsgpu_mobius_dslash_4(self._h, dptr(out), dptr(inp), cb, dag, prec))
        return out

    def M5inv(self, inp, dag: int = 0, prec: int = A.DOUBLE) -> np.ndarray:
        inp = self._vec(inp)
        out = np.empty_like(inp)
        check(lib().cpsgpu_mobius_m5inv(self._h, dptr(out), dptr(inp), dag, prec))
        return out


def solve_batch(items, stop_rsd=1e-8, max_num_iter=10000, precision=A.DOUBLE, delta=0.0, chunk=8):
    """Independent InvCg solves of different operators in one graph launch
    (cpsgpu_solve_batch).  items: (DiracOp, sol, src) with host vectors, sol
    the initial guess, updated in place.  Returns one CgResult per item; the
    device time of each is the whole batch's."""
    fields, ops, sols, srcs, args = [], [], [], [], []
    for D, sol, src in items:
        src = D._vec(src)
        if not (isinstance(sol, np.ndarray) and sol.dtype == np.float64 and sol.flags.c_contiguous):
            raise TypeError("sol must be a C-contiguous float64 array (updated in place)")
        D._vec(sol)
        fs, fb = C.c_void_p(), C.c_void_p()
        check(lib().cpsgpu_field_create(D._h, A.DOUBLE, 1, C.byref(fs)))
        check(lib().cpsgpu_field_create(D._h, A.DOUBLE, 1, C.byref(fb)))
        fields += [fs, fb]
        check(lib().cpsgpu_field_upload(fs, dptr(sol)))
        check(lib().cpsgpu_field_upload(fb, dptr(src)))
        ops.append(D._h)
        sols.append(fs)
        srcs.append(fb)
        args.append(D._cg_arg(stop_rsd, max_num_iter, 0.0, 0.0, precision, delta, chunk, True))
    n = len(items)
    try:
        res = (A.CgResult * n)()
        VP = C.c_void_p * n
        check(lib().cpsgpu_solve_batch(n, VP(*[o.value for o in ops]), VP(*[f.value for f in sols]),
                                       VP(*[f.value for f in srcs]), (A.CgArg * n)(*args), res))
        for (D, sol, _), fs in zip(items, sols):
            check(lib().cpsgpu_field_download(fs, dptr(sol)))
        return [CgResult(r.iterations, r.status, r.true_res, r.reliable_updates, r.seconds, r.kernels) for r in res]
    finally:
        for f in fields:
            lib().cpsgpu_field_destroy(f)
