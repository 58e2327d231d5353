"""Generate the golden fixtures from the reference's own kernels.

Runs the reference's noarch kernels (compiled unchanged from the reference
sources by ``make -C oracle ref``) on small seeded inputs and stores inputs
and outputs in ``tests/golden/ref_kernels.npz``.  The gauge field is stored
without boundary signs; the reference is called with the signs applied as
its BondCond applies them.  Re-run only when the fixture set changes:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.loader import apply_bc_signs, load_reference, p  # noqa: E402

OUT = Path(__file__).resolve().parent / "ref_kernels.npz"


def su3_field(L, rng):
    """Random SU(3) links by QR of complex Gaussians, det fixed to 1."""
    vol = int(np.prod(L))
    a = rng.normal(size=(vol * 4, 3, 3)) + 1j * rng.normal(size=(vol * 4, 3, 3))
    q, r = np.linalg.qr(a)
    q = q * (np.diagonal(r, axis1=1, axis2=2) / np.abs(np.diagonal(r, axis1=1, axis2=2)))[:, None, :]
    det = np.linalg.det(q)
    q[:, 2, :] /= det[:, None]
    # WILSON order element (row, col) at 2*(row + 3*col): store the transpose
    out = np.empty((vol * 4, 18))
    qt = np.transpose(q, (0, 2, 1)).reshape(vol * 4, 9)
    out[:, 0::2] = qt.real
    out[:, 1::2] = qt.imag
    return out.reshape(-1)


def main():
    R = load_reference()
    rng = np.random.default_rng(20261203)
    data = {}
    cases = [
        ("w44", (4, 4, 4, 4), 1, (1, 1, 1, -1)),
        ("w2468", (2, 4, 6, 8), 1, (1, 1, 1, -1)),
        ("d4", (2, 4, 4, 4), 4, (1, 1, 1, -1)),
        ("d2", (2, 2, 4, 4), 6, (1, 1, 1, -1)),
    ]
    mass = 0.05
    for name, L, ls, bc in cases:
        vol = int(np.prod(L))
        vh = vol // 2
        u = su3_field(L, rng)
        us = apply_bc_signs(u, L, bc)
        R.ref_init(*L, max(ls, 1) if ls > 1 else 2, 1.8, 1.5, 0.5, -1 if bc[3] < 0 else 1)
        data[f"{name}_L"] = np.array(L)
        data[f"{name}_ls"] = np.array(ls)
        data[f"{name}_u"] = u
        n = 24 * vh * ls
        psi = rng.normal(size=n)
        data[f"{name}_psi"] = psi
        if ls == 1:
            for cb in (0, 1):
                for dag in (0, 1):
                    y = np.zeros(n)
                    R.ref_wilson_dslash(p(y), p(us), p(psi), cb, dag)
                    data[f"{name}_dslash_{cb}{dag}"] = y
            y = np.zeros(n)
            d = C.c_double()
            R.ref_wilson_mdagm(p(y), p(us), p(psi), C.byref(d), 0.12)
            data[f"{name}_mdagm"] = y
            data[f"{name}_mdagm_dot"] = np.array(d.value)
            for dag, fn in ((0, R.ref_wilson_m), (1, R.ref_wilson_mdag)):
                y = np.zeros(n)
                fn(p(y), p(us), p(psi), 0.12)
                data[f"{name}_m_{dag}"] = y
        else:
            for cb in (0, 1):
                for dag in (0, 1):
                    y = np.zeros(n)
                    R.ref_dwf_dslash(p(y), p(us), p(psi), mass, cb, dag)
                    data[f"{name}_dwf_dslash_{cb}{dag}"] = y
                    y = np.zeros(n)
                    R.ref_zmobius_dslash_4(p(y), p(us), p(psi), cb, dag, mass)
                    data[f"{name}_mob_dslash4_{cb}{dag}"] = y
            d = C.c_double()
            y = np.zeros(n)
            R.ref_dwf_mdagm(p(y), p(us), p(psi), C.byref(d), mass)
            data[f"{name}_dwf_mdagm"] = y
            data[f"{name}_dwf_mdagm_dot"] = np.array(d.value)
            for dag in (0, 1):
                y = psi.copy()
                R.ref_zmobius_m5inv(p(y), mass, dag)
                data[f"{name}_mob_m5inv_{dag}"] = y
                y = np.zeros(n)
                (R.ref_zmobius_mdag if dag else R.ref_zmobius_m)(p(y), p(us), p(psi), mass)
                data[f"{name}_mob_m_{dag}"] = y
            y = np.zeros(n)
            R.ref_zmobius_mdagm(p(y), p(us), p(psi), C.byref(d), mass)
            data[f"{name}_mob_mdagm"] = y
            data[f"{name}_mob_mdagm_dot"] = np.array(d.value)
    data["mass"] = np.array(mass)
    np.savez_compressed(OUT, **data)
    print(OUT, OUT.stat().st_size)


if __name__ == "__main__":
    main()
