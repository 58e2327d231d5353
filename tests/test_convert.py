"""Host storage-order conversions (cpsgpu_fconvert / gconvert / four2five /
five2four) against numpy restatements of the reference's routines
(oracle/convert.py), and their round trips.  CPU only."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import StrOrd, fconvert, five2four, four2five, gconvert, gen_gauge, gen_gaussian
from oracle import convert as OC

GEOMS = [(4, 4, 4, 4), (2, 4, 6, 2), (6, 2, 2, 4)]


@pytest.mark.parametrize("L", GEOMS)
def test_fconvert_4d_matches_reference_table(L):
    f = gen_gaussian(24 * int(np.prod(L)), seed=1)
    w = f.copy()
    fconvert(L, 1, w, StrOrd.WILSON, StrOrd.CANONICAL)
    assert np.array_equal(w, OC.fcanon_to_wilson_4d(f, L))
    fconvert(L, 1, w, StrOrd.CANONICAL, StrOrd.WILSON)
    assert np.array_equal(w, f)


@pytest.mark.parametrize("L", GEOMS)
@pytest.mark.parametrize("ls", [2, 3, 4])
def test_fconvert_dwf_matches_reference(L, ls):
    f = gen_gaussian(24 * ls * int(np.prod(L)), seed=2)
    w = f.copy()
    fconvert(L, ls, w, StrOrd.WILSON, StrOrd.CANONICAL)
    assert np.array_equal(w, OC.fconvert_dwf(f, L, ls))
    fconvert(L, ls, w, StrOrd.CANONICAL, StrOrd.WILSON)
    assert np.array_equal(w, f)


@pytest.mark.parametrize("L", GEOMS)
def test_gconvert_matches_reference(L):
    u = gen_gaussian(72 * int(np.prod(L)), seed=3)
    w = u.copy()
    gconvert(L, w, StrOrd.WILSON, StrOrd.CANONICAL)
    assert np.array_equal(w, OC.gcanon_to_wilson(u, L))
    gconvert(L, w, StrOrd.CANONICAL, StrOrd.WILSON)
    assert np.array_equal(w, u)


def test_gconvert_of_library_gauge_is_consistent():
    """The generator writes WILSON order: converting to CANONICAL and back is
    the identity, and CANONICAL holds each link row-major."""
    L = (4, 2, 2, 4)
    u = gen_gauge(L, seed=4)
    c = u.copy()
    gconvert(L, c, StrOrd.CANONICAL, StrOrd.WILSON)
    w = c.copy()
    gconvert(L, w, StrOrd.WILSON, StrOrd.CANONICAL)
    assert np.array_equal(w, u)
    # site (0,0,0,0) is the first even site; its mu=0 link (row 0, col 1)
    assert c[2 * (3 * 0 + 1)] == u[2 * (0 + 3 * 1)]


@pytest.mark.parametrize("ncb", [1, 2])
def test_four2five_five2four(ncb):
    L, ls = (4, 2, 2, 4), 6
    v4 = int(np.prod(L)) * ncb // 2
    four = gen_gaussian(24 * v4, seed=5)
    for s_u, s_l in ((0, ls - 1), (2, 2), (ls - 1, 0)):
        five = four2five(L, ls, four, s_u, s_l, ncb)
        assert np.array_equal(five, OC.four2five(four, v4, ls, s_u, s_l))
        back = five2four(L, ls, five, s_u, s_l, ncb)
        assert np.array_equal(back, OC.five2four(five, v4, ls, s_u, s_l))
        assert np.array_equal(back, four)


def test_conversion_arguments_are_checked():
    L = (4, 4, 4, 4)
    f = np.zeros(24 * 256)
    with pytest.raises(A.CpsGpuError):
        fconvert(L, 1, f, 5, StrOrd.CANONICAL)  # only CANONICAL <-> WILSON
    with pytest.raises(A.CpsGpuError):
        four2five(L, 4, np.zeros(24 * 256), 4, 0)  # s_u outside [0, ls)
    with pytest.raises(TypeError):
        fconvert(L, 2, f, StrOrd.WILSON, StrOrd.CANONICAL)  # wrong size
