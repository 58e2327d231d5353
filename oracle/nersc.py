"""Test infrastructure only: numpy restatements of the reference's NERSC
archive handling, to check the library's reader and writer
(cps_veloc_b200/csrc/nersc.cpp) and the device plaquette against.

* ``checksum``   FPConv::checksum (fpconv.C:320-360): the data as 32-bit
  words in host order, summed modulo 2^32.
* ``write``      WriteLatticeParallel::write (WriteLatticePar.C) with the
  header of LatticeHeader::write (latheader.C:195-260): sites in
  lexicographic order, links mu = 0..3, first two rows or all three,
  row-major (re, im).
* ``read``       ReadLatticeParallel::read (ReadLatticePar.C): header map,
  checksum, third row rebuilt as conj(row0 x row1).
* ``plaquette``  Lattice::SumReTrPlaq / (18 V) (lattice_base.C:2878-3060) and
  the link trace sum Re tr U / (12 V) of a CANONICAL field.
"""
import numpy as np

FORMATS = {"IEEE32": ">f4", "IEEE32BIG": ">f4", "IEEE32LITTLE": "<f4",
           "IEEE64": ">f8", "IEEE64BIG": ">f8", "IEEE64LITTLE": "<f8"}


def checksum(raw: bytes, dtype: str) -> int:
    """sum of the 32-bit words of the file data, each read in the file's byte order"""
    order = ">" if dtype.startswith(">") else "<"
    return int(np.frombuffer(raw, dtype=order + "u4").astype(np.uint64).sum() % (1 << 32))


def links(u, L):
    """CANONICAL field as complex [t][z][y][x][mu][row][col]"""
    a = np.asarray(u).reshape(L[3], L[2], L[1], L[0], 4, 3, 3, 2)
    return a[..., 0] + 1j * a[..., 1]


def plaquette(u, L):
    U = links(u, L)
    vol = int(np.prod(L))
    axis = {0: 3, 1: 2, 2: 1, 3: 0}  # lattice direction -> array axis
    sp = 0.0
    for mu in range(3):
        for nu in range(mu + 1, 4):
            Um, Un = U[..., mu, :, :], U[..., nu, :, :]
            Un_pm = np.roll(Un, -1, axis=axis[mu])  # U_nu(x + mu)
            Um_pn = np.roll(Um, -1, axis=axis[nu])  # U_mu(x + nu)
            m1 = Um @ Un_pm
            m2 = Un @ Um_pn
            sp += float(np.sum((m1 * np.conj(m2)).real))
    lt = float(np.sum(np.trace(U, axis1=-2, axis2=-1).real))
    return sp / (18.0 * vol), lt / (12.0 * vol)


def write(path, u, L, recon_row_3=True, fmt="IEEE64BIG", ensemble_id="", ensemble_label="", seq=0):
    plaq, ltr = plaquette(u, L)
    per = 12 if recon_row_3 else 18
    data = np.asarray(u).reshape(-1, 18)[:, :per].astype(FORMATS[fmt]).tobytes()
    cs = checksum(data, FORMATS[fmt])
    lines = ["BEGIN_HEADER", "HDR_VERSION = 1.0",
             "DATATYPE = " + ("4D_SU3_GAUGE" if recon_row_3 else "4D_SU3_GAUGE_3x3"), "STORAGE_FORMAT = 1.0"]
    lines += [f"DIMENSION_{k + 1} = {L[k]}" for k in range(4)]
    lines += [f"LINK_TRACE = {ltr:.10g}", f"PLAQUETTE  = {plaq:.10g}"]
    lines += [f"BOUNDARY_{k + 1} = PERIODIC" for k in range(4)]
    lines += [f"CHECKSUM = {cs:8x}", f"ENSEMBLE_ID = {ensemble_id}", f"ENSEMBLE_LABEL = {ensemble_label}",
              f"SEQUENCE_NUMBER = {seq}", "CREATOR = oracle", "CREATOR_HARDWARE = none",
              "CREATION_DATE = none", "ARCHIVE_DATE = none", f"FLOATING_POINT = {fmt}", "END_HEADER"]
    with open(path, "wb") as f:
        f.write(("\n".join(lines) + "\n").encode())
        f.write(data)
    return cs, plaq, ltr


def read(path, L):
    raw = open(path, "rb").read()
    end = raw.index(b"END_HEADER")
    nl = raw.index(b"\n", end)
    hdr = {}
    for line in raw[:end].decode().splitlines():
        if "=" in line:
            k, v = line.split("=", 1)
            hdr.setdefault(k.strip(), v.strip())
    dtype = FORMATS[hdr["FLOATING_POINT"]]
    per = 12 if hdr["DATATYPE"] == "4D_SU3_GAUGE" else 18
    vol = int(np.prod(L))
    data = raw[nl + 1:nl + 1 + vol * 4 * per * np.dtype(dtype).itemsize]
    if checksum(data, dtype) != int(hdr["CHECKSUM"], 16):
        raise ValueError("checksum")
    vals = np.frombuffer(data, dtype=dtype).astype(np.float64).reshape(-1, per)
    out = np.zeros((vals.shape[0], 18))
    out[:, :per] = vals
    if per == 12:
        m = out[:, 0:12:2] + 1j * out[:, 1:12:2]  # rows 0, 1 as 6 complex
        r0, r1 = m[:, 0:3], m[:, 3:6]
        r2 = np.conj(np.cross(r0, r1))
        out[:, 12::2], out[:, 13::2] = r2.real, r2.imag
    return out.ravel(), hdr
