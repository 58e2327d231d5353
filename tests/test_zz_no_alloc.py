"""The allocation-free MatPcDagMatPc (cpsgpu_matpc_dag_matpc_noalloc).

It exists for callers that cannot call cudaMalloc while they apply the
operator (their device memory is owned by their own pool allocator, or they
cannot afford the synchronisation an allocation implies): the caller passes
device buffers it already owns, and every temporary lives in the library's
fixed scratch array.  Here its output is checked against the ordinary
cpsgpu_matpc_dag_matpc on two calls in a row (the scratch keeps the previous
call's contents, which must not leak into the next result), and an operator
too large for the scratch must be rejected.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import DiracOpDwf, DiracOpWilson, Lattice, gen_gauge, gen_gaussian
from helpers import rel

pytestmark = pytest.mark.gpu


def to_device_layout(x, ls, vh):
    """CPS order [s][site][24] -> the library's FP64 layout [s][group][site][2]."""
    return np.ascontiguousarray(x.reshape(ls, vh, 12, 2).transpose(0, 2, 1, 3))


def from_device_layout(y, ls, vh):
    return np.ascontiguousarray(y.reshape(ls, 12, vh, 2).transpose(0, 2, 1, 3)).reshape(-1)


def _check(D, seed):
    import torch

    ls, vh = D.ls, D.lat.vol // 2
    x = gen_gaussian(D.f_size, seed=seed)
    ref, ref_dot = D.MatPcDagMatPc(x)
    xin = torch.from_numpy(to_device_layout(x, ls, vh)).to("cuda")
    for call in range(2):  # two calls in a row through the shared scratch
        out = torch.full((D.f_size,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        dot = C.c_double()
        A.check(A.lib().cpsgpu_matpc_dag_matpc_noalloc(D._h, C.c_void_p(out.data_ptr()),
                                                        C.c_void_p(xin.data_ptr()), C.byref(dot)))
        y = from_device_layout(out.cpu().numpy(), ls, vh)
        assert rel(y, ref) < 1e-13, f"call {call}"
        assert abs(dot.value / ref_dot - 1) < 1e-13, f"call {call}"


def test_noalloc_wilson_matches():
    L = (8, 8, 8, 8)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=201))
    _check(DiracOpWilson(lat, mass=0.1), seed=202)


def test_noalloc_dwf_matches():
    L = (4, 4, 4, 8)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=203))
    _check(DiracOpDwf(lat, mass=0.05, ls=8), seed=204)


def test_noalloc_rejects_operator_too_large_for_scratch():
    L = (16, 16, 16, 16)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=205))
    D = DiracOpDwf(lat, mass=0.05, ls=8)  # 262144 5D sites: two FP64 fields are 96 MiB
    dummy = C.c_void_p(1 << 20)  # never dereferenced: the size check comes first
    rc = A.lib().cpsgpu_matpc_dag_matpc_noalloc(D._h, dummy, dummy, None)
    assert rc == -1
    assert b"scratch" in A.lib().cpsgpu_last_error()
