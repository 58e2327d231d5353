"""The C-ABI library without a GPU: it loads, exports every symbol declared
in include/cpsgpu.h, generates the seeded inputs deterministically, and
reports errors instead of crashing."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import gen_gauge, gen_gaussian

HEADER = Path(__file__).resolve().parents[1] / "include" / "cpsgpu.h"


def test_library_exports_every_declared_symbol():
    lib = A.lib()
    names = A.declared_symbols(HEADER)
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_version_and_error_string():
    lib = A.lib()
    assert b"sm_100a" in lib.cpsgpu_version()
    rc = lib.cpsgpu_dirac_create(None, None, None)
    assert rc == -1
    assert b"null" in lib.cpsgpu_last_error()


def test_bad_lattice_arguments_rejected():
    lib = A.lib()
    h = C.c_void_p()
    rc = lib.cpsgpu_lattice_create(A.ints([4, 4, 3, 4]), A.ints([1, 1, 1, -1]), C.byref(h))
    assert rc != 0
    rc = lib.cpsgpu_lattice_create(A.ints([4, 4, 4, 4]), A.ints([1, 1, 1, 0]), C.byref(h))
    assert rc == -1


def _links(u, vol):
    m = u.reshape(vol * 4, 18)
    z = m[:, 0::2] + 1j * m[:, 1::2]
    return np.transpose(z.reshape(vol * 4, 3, 3), (0, 2, 1))  # element (row, col) at 2*(row+3*col)


def test_gauge_generator_su3_and_deterministic():
    L = (4, 2, 2, 4)
    vol = int(np.prod(L))
    u1 = gen_gauge(L, seed=7)
    u2 = gen_gauge(L, seed=7)
    u3 = gen_gauge(L, seed=8)
    assert np.array_equal(u1, u2) and not np.array_equal(u1, u3)
    U = _links(u1, vol)
    eye = np.eye(3)
    err = np.abs(U @ np.conj(np.transpose(U, (0, 2, 1))) - eye).max()
    assert err < 1e-14
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-14
    # width 0.3: links close to, but not at, the identity
    dist = np.abs(U - eye).mean()
    assert 0.05 < dist < 0.6


def test_gaussian_generator_moments():
    x = gen_gaussian(400000, seed=3)
    assert abs(x.mean()) < 0.01 and abs(x.std() - 1) < 0.01
    assert np.array_equal(gen_gaussian(1000, seed=3), x[:1000])
    assert not np.array_equal(gen_gaussian(1000, seed=3, stream=1), x[:1000])
