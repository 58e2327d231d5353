"""Test and baseline infrastructure only: the seeded synthetic inputs in numpy.

The same counter-based streams as the library's generator (every random
number a pure function of (seed, stream, index) through a SplitMix64-style
hash, Steele, Lea and Flood, OOPSLA 2014; Gaussians by Box-Muller), so the
reference's CPU arm of the benchmark builds the benchmarked gauge field and
sources without loading the library under test.

    gen_gauge(L, seed, width)   U = exp(i width H), H = (A + A^+)/2 - tr/3,
                                 A a 3x3 matrix of unit complex Gaussians;
                                 the exponential by scaling and squaring of an
                                 18-term Taylor series, then Gram-Schmidt on
                                 rows 0, 1 and row 2 = conj(r0 x r1), det U = 1.
                                 WILSON order [parity][cb site][mu][col][row]
                                 (order="wilson") or CANONICAL [site][mu][row][col].
    gen_gaussian(n, seed, stream)

Values agree with the library's generator to rounding (the transcendental
functions of numpy and of the C++ runtime may differ in the last place).
"""
from __future__ import annotations

import numpy as np

_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix64(z):
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _uniform(seed, stream, idx):
    with np.errstate(over="ignore"):
        h = _mix64(np.uint64(seed) ^ _mix64(np.uint64(stream) * np.uint64(0x632BE59BD9B4E019) ^ _mix64(idx)))
    return ((h >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def _gaussian(seed, stream, idx):
    idx = np.asarray(idx, dtype=np.uint64)
    pair = idx >> np.uint64(1)
    with np.errstate(over="ignore"):
        u1 = _uniform(seed, stream, np.uint64(2) * pair)
        u2 = _uniform(seed, stream, np.uint64(2) * pair + np.uint64(1))
    r = np.sqrt(-2.0 * np.log(u1))
    th = 6.283185307179586476925286766559 * u2
    return np.where((idx & np.uint64(1)) == 1, r * np.sin(th), r * np.cos(th))


def gen_gaussian(n: int, seed: int = 20261203, stream: int = 0) -> np.ndarray:
    return _gaussian(seed, 1000 + stream, np.arange(n, dtype=np.uint64))


def _su3(seed, keys, width):
    nk = keys.size
    base = keys.astype(np.uint64) * np.uint64(18)
    comp = np.arange(18, dtype=np.uint64)
    with np.errstate(over="ignore"):
        g = _gaussian(seed, 1, base[:, None] + comp[None, :])
    a = (g[:, 0::2] + 1j * g[:, 1::2]).reshape(nk, 3, 3)
    h = 0.5 * (a + np.conj(np.transpose(a, (0, 2, 1))))
    tr = (h[:, 0, 0] + h[:, 1, 1] + h[:, 2, 2]) / 3.0
    for i in range(3):
        h[:, i, i] -= tr
    x = 1j * width * h
    nrm = np.sqrt(np.sum(np.abs(x) ** 2, axis=(1, 2)))
    k = np.zeros(nk, dtype=np.int64)
    while True:
        big = nrm > 0.25
        if not big.any():
            break
        nrm = np.where(big, nrm * 0.5, nrm)
        k += big
    x = x * np.ldexp(1.0, -k)[:, None, None]
    e = np.broadcast_to(np.eye(3, dtype=np.complex128), (nk, 3, 3)).copy()
    term = e.copy()
    for n in range(1, 19):
        term = (term @ x) / float(n)
        e = e + term
    for s in range(int(k.max(initial=0))):
        sq = e @ e
        e = np.where((k > s)[:, None, None], sq, e)
    u = np.empty_like(e)
    u[:, 0] = e[:, 0] / np.sqrt(np.sum(np.abs(e[:, 0]) ** 2, axis=1))[:, None]
    pr = np.sum(np.conj(u[:, 0]) * e[:, 1], axis=1)
    u1 = e[:, 1] - pr[:, None] * u[:, 0]
    u[:, 1] = u1 / np.sqrt(np.sum(np.abs(u1) ** 2, axis=1))[:, None]
    u[:, 2, 0] = np.conj(u[:, 0, 1] * u[:, 1, 2] - u[:, 0, 2] * u[:, 1, 1])
    u[:, 2, 1] = np.conj(u[:, 0, 2] * u[:, 1, 0] - u[:, 0, 0] * u[:, 1, 2])
    u[:, 2, 2] = np.conj(u[:, 0, 0] * u[:, 1, 1] - u[:, 0, 1] * u[:, 1, 0])
    return u


def gen_gauge(L, seed: int = 20261203, width: float = 0.3, order: str = "wilson") -> np.ndarray:
    """Seeded SU(3) field, no boundary signs; the stream of link (site, mu) is
    keyed by the canonical site x + Lx (y + Ly (z + Lz t)) and mu."""
    lx, ly, lz, lt = L
    vol = lx * ly * lz * lt
    out = np.empty((vol, 4, 18))
    chunk = 1 << 15
    for b in range(0, vol * 4, chunk):
        keys = np.arange(b, min(vol * 4, b + chunk), dtype=np.uint64)
        u = _su3(seed, keys, width)
        site, mu = keys // np.uint64(4), keys % np.uint64(4)
        if order == "canonical":
            m = u  # [row][col]
        else:
            m = np.transpose(u, (0, 2, 1))  # element (row, col) at 2 (row + 3 col)
        flat = np.empty((keys.size, 18))
        flat[:, 0::2] = m.reshape(-1, 9).real
        flat[:, 1::2] = m.reshape(-1, 9).imag
        out[site.astype(np.int64), mu.astype(np.int64)] = flat
    if order == "canonical":
        return out.reshape(-1)
    s = np.arange(vol)
    x, r = s % lx, s // lx
    y, r = r % ly, r // ly
    z, t = r % lz, r // lz
    par = (x + y + z + t) & 1
    cb = x // 2 + (lx // 2) * (y + ly * (z + lz * t))
    w = np.empty((2, vol // 2, 4, 18))
    w[par, cb] = out
    return w.reshape(-1)
