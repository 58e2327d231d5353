"""The storage-order conversions on device memory (cpsgpu_fconvert_device,
_gconvert_device, _four2five_device, _five2four_device) against the host
routines (pinned to the reference's site and component tables by
tests/test_convert.py): permutations, so bit for bit, both directions, 4D
and 5D fermions, odd and even Ls, the links, and the wall placement with
one and two checkerboards."""
import numpy as np
import pytest
import torch

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import Lattice

pytestmark = pytest.mark.gpu
CAN, WIL = 0, 2


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (6, 4, 2, 8), (2, 2, 2, 2)])
@pytest.mark.parametrize("ls", [1, 5, 8])
def test_fconvert_device(L, ls):
    A.check(A.lib().cpsgpu_set_device(0))
    torch.cuda.set_device(0)
    lat = Lattice(L)
    vol = int(np.prod(L))
    rng = np.random.default_rng(ls + vol)
    f = rng.normal(size=24 * ls * vol)
    ns = (A.C.c_int * 4)(*L)
    for to, frm in ((WIL, CAN), (CAN, WIL)):
        host = f.copy()
        A.check(A.lib().cpsgpu_fconvert(ns, ls, A.dptr(host), to, frm))
        src, dst = _dev(f), torch.empty(f.size, dtype=torch.float64, device="cuda")
        A.check(A.lib().cpsgpu_fconvert_device(lat._h, ls, dst.data_ptr(), src.data_ptr(), to, frm))
        A.check(A.lib().cpsgpu_synchronize(lat._h))
        np.testing.assert_array_equal(dst.cpu().numpy(), host)


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (6, 4, 2, 8)])
def test_gconvert_device(L):
    A.check(A.lib().cpsgpu_set_device(0))
    lat = Lattice(L)
    u = np.random.default_rng(9).normal(size=72 * int(np.prod(L)))
    ns = (A.C.c_int * 4)(*L)
    for to, frm in ((WIL, CAN), (CAN, WIL)):
        host = u.copy()
        A.check(A.lib().cpsgpu_gconvert(ns, A.dptr(host), to, frm))
        src, dst = _dev(u), torch.empty(u.size, dtype=torch.float64, device="cuda")
        A.check(A.lib().cpsgpu_gconvert_device(lat._h, dst.data_ptr(), src.data_ptr(), to, frm))
        A.check(A.lib().cpsgpu_synchronize(lat._h))
        np.testing.assert_array_equal(dst.cpu().numpy(), host)


@pytest.mark.parametrize("ncb", [1, 2])
@pytest.mark.parametrize("ls,s_u,s_l", [(8, 0, 7), (5, 2, 2), (4, 3, 1)])
def test_four2five_device(ncb, ls, s_u, s_l):
    A.check(A.lib().cpsgpu_set_device(0))
    L = (4, 4, 2, 6)
    lat = Lattice(L)
    v4 = int(np.prod(L)) * ncb // 2
    four = np.random.default_rng(ls).normal(size=24 * v4)
    ns = (A.C.c_int * 4)(*L)
    five_h = np.full(24 * ls * v4, np.nan)
    A.check(A.lib().cpsgpu_four2five(ns, ls, A.dptr(five_h), A.dptr(four), s_u, s_l, ncb))
    src, five = _dev(four), torch.full((24 * ls * v4,), float("nan"), dtype=torch.float64, device="cuda")
    A.check(A.lib().cpsgpu_four2five_device(lat._h, ls, five.data_ptr(), src.data_ptr(), s_u, s_l, ncb))
    A.check(A.lib().cpsgpu_synchronize(lat._h))
    np.testing.assert_array_equal(five.cpu().numpy(), five_h)
    back_h = np.zeros(24 * v4)
    A.check(A.lib().cpsgpu_five2four(ns, ls, A.dptr(back_h), A.dptr(five_h), s_u, s_l, ncb))
    back = torch.zeros(24 * v4, dtype=torch.float64, device="cuda")
    A.check(A.lib().cpsgpu_five2four_device(lat._h, ls, back.data_ptr(), five.data_ptr(), s_u, s_l, ncb))
    A.check(A.lib().cpsgpu_synchronize(lat._h))
    np.testing.assert_array_equal(back.cpu().numpy(), back_h)
    np.testing.assert_array_equal(back_h, four)


def test_device_conversions_refuse_bad_arguments():
    A.check(A.lib().cpsgpu_set_device(0))
    lat = Lattice((4, 4, 4, 4))
    t = torch.zeros(24 * 256, dtype=torch.float64, device="cuda")
    assert A.lib().cpsgpu_fconvert_device(lat._h, 1, t.data_ptr(), t.data_ptr(), WIL, CAN) != 0  # in place
    u = torch.zeros(24 * 256, dtype=torch.float64, device="cuda")
    assert A.lib().cpsgpu_fconvert_device(lat._h, 1, u.data_ptr(), t.data_ptr(), 1, CAN) != 0  # other orders
    assert A.lib().cpsgpu_four2five_device(lat._h, 4, u.data_ptr(), t.data_ptr(), 4, 0, 2) != 0  # s_u out of range
