"""The device plaquette and loading a NERSC archive into a lattice
(ReadLatticeParallel::read with its plaquette check)."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import Lattice, StrOrd, gconvert, gen_gauge, nersc_write
from oracle import nersc as ON

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (8, 4, 6, 2), (16, 16, 16, 32)])
def test_plaquette_matches_oracle(L):
    u = gen_gauge(L, seed=311)
    lat = Lattice(L)
    lat.import_gauge(u)
    uc = u.copy()
    gconvert(L, uc, StrOrd.CANONICAL, StrOrd.WILSON)
    plaq, ltr = ON.plaquette(uc, L)
    p, t = lat.plaquette()
    assert abs(p - plaq) < 1e-13 * abs(plaq) and abs(t - ltr) < 1e-13 * abs(ltr)


def test_load_nersc_into_lattice(tmp_path):
    L = (8, 4, 4, 8)
    u = gen_gauge(L, seed=312)
    uc = u.copy()
    gconvert(L, uc, StrOrd.CANONICAL, StrOrd.WILSON)
    path = tmp_path / "conf.nersc"
    hw = nersc_write(path, L, uc, recon_row_3=True, floating_point="IEEE64BIG")
    lat = Lattice(L)
    p, h = lat.load_nersc(path)
    assert abs(p - hw["plaquette"]) < 1e-13 and h["checksum"] == hw["checksum"]
    ref = Lattice(L)
    ref.import_gauge(u)
    assert abs(ref.plaquette()[0] - p) < 1e-13
    # a header plaquette off by more than the check precision is refused
    raw = path.read_bytes()
    line = next(x for x in raw.split(b"\n") if x.startswith(b"PLAQUETTE"))
    bad = tmp_path / "bad.nersc"
    bad.write_bytes(raw.replace(line, b"PLAQUETTE  = 0.1234567890"[:len(line)].ljust(len(line))))
    with pytest.raises(A.CpsGpuError, match="plaquette"):
        lat.load_nersc(bad)
