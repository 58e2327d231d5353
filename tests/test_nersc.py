"""NERSC gauge archives (cpsgpu_nersc_read / _write) against numpy
restatements of the reference's reader, writer and checksum
(oracle/nersc.py), with the checksum pinned to the reference's own
FPConv::checksum.  CPU only (host code of the library)."""
import numpy as np
import pytest

from cps_veloc_b200 import _abi as A
from cps_veloc_b200.dirac import StrOrd, gconvert, gen_gauge, gen_gaussian, nersc_read, nersc_write
from oracle import nersc as ON

L = (4, 4, 2, 6)


def canonical_gauge(L, seed):
    u = gen_gauge(L, seed=seed)
    gconvert(L, u, StrOrd.CANONICAL, StrOrd.WILSON)
    return u


@pytest.mark.parametrize("fmt", ["IEEE32BIG", "IEEE32LITTLE", "IEEE64BIG", "IEEE64LITTLE"])
def test_checksum_vs_reference(reference, fmt):
    x = gen_gaussian(1000, seed=301)
    dtype = ON.FORMATS[fmt]
    raw = x.astype(dtype).tobytes()
    ref = reference.ref_fp_checksum(raw, x.size, A.FP_FORMATS[fmt])
    assert ON.checksum(raw, dtype) == ref


@pytest.mark.parametrize("recon", [True, False])
@pytest.mark.parametrize("fmt", ["IEEE64BIG", "IEEE32BIG", "IEEE64LITTLE"])
def test_library_writer_matches_reference_format(tmp_path, recon, fmt):
    u = canonical_gauge(L, 302)
    path = tmp_path / "conf.nersc"
    hw = nersc_write(path, L, u, recon_row_3=recon, floating_point=fmt, ensemble_id="ens", sequence_number=7)
    uo, ho = ON.read(path, L)
    plaq, ltr = ON.plaquette(u, L)
    assert int(ho["CHECKSUM"], 16) == hw["checksum"]
    assert ho["DATATYPE"] == ("4D_SU3_GAUGE" if recon else "4D_SU3_GAUGE_3x3") and ho["FLOATING_POINT"] == fmt
    assert [int(ho[f"DIMENSION_{k + 1}"]) for k in range(4)] == list(L)
    assert abs(float(ho["PLAQUETTE"]) - plaq) < 1e-9 and abs(float(ho["LINK_TRACE"]) - ltr) < 1e-9
    assert abs(hw["plaquette"] - plaq) < 1e-13 and abs(hw["link_trace"] - ltr) < 1e-13
    assert ho["ENSEMBLE_ID"] == "ens" and ho["SEQUENCE_NUMBER"] == "7"
    tol = 1e-6 if "32" in fmt else 1e-15
    assert np.abs(uo - u).max() < tol


@pytest.mark.parametrize("recon", [True, False])
@pytest.mark.parametrize("fmt", ["IEEE64BIG", "IEEE32BIG", "IEEE32LITTLE"])
def test_library_reader_reads_reference_format(tmp_path, recon, fmt):
    u = canonical_gauge(L, 303)
    path = tmp_path / "conf.nersc"
    cs, plaq, ltr = ON.write(path, u, L, recon_row_3=recon, fmt=fmt, ensemble_label="lbl", seq=3)
    ul, h = nersc_read(path, L)
    uo, _ = ON.read(path, L)
    assert h["checksum"] == cs and h["recon_row_3"] == recon and h["floating_point"] == fmt
    assert h["ensemble_label"] == "lbl" and h["sequence_number"] == 3
    assert abs(h["plaquette"] - plaq) < 1e-6  # parsed with %f as the reference does
    assert np.abs(ul - uo).max() < 1e-14
    assert np.abs(ul - u).max() < (1e-6 if "32" in fmt else 1e-14)


def test_reader_rejects_bad_files(tmp_path):
    u = canonical_gauge(L, 304)
    path = tmp_path / "conf.nersc"
    nersc_write(path, L, u)
    raw = bytearray(path.read_bytes())
    raw[-100] ^= 0x01  # one flipped bit in the data
    bad = tmp_path / "bad.nersc"
    bad.write_bytes(bytes(raw))
    with pytest.raises(A.CpsGpuError, match="checksum"):
        nersc_read(bad, L)
    with pytest.raises(A.CpsGpuError):
        nersc_read(path, (4, 4, 2, 8))  # dimensions differ from the header
    short = tmp_path / "short.nersc"
    short.write_bytes(path.read_bytes()[:-8])
    with pytest.raises(A.CpsGpuError):
        nersc_read(short, L)
