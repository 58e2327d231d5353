"""Test infrastructure only: numpy restatements of the reference's storage-
order conversions, step for step, to check the library's host conversions
(cps_veloc_b200/csrc/convert.cpp) against.

* ``fcanon_to_wilson_4d``   FcanonToWilson's site table, convert_func.C:429-494
  (new position (x - x%2 + Lx*(y + Ly*(z + Lz*t)) + V*((x+y+z+t+1)%2)) / 2).
* ``fconvert_dwf``          FdwfBase::Fconvert CANONICAL -> WILSON, convert.C:704-760:
  every 4D slice through FcanonToWilson, then the odd part gathered from
  slice s's half (s+1)%2 and the even part from half s%2, moving the read
  pointer by (2*parity + 1) half volumes as the reference does.
* ``gcanon_to_wilson``      the WILSON gauge order of convert.C:258-336 (its
  site and link tables, read in the CANONICAL -> WILSON direction).
* ``four2five`` / ``five2four``  f_dwf_base.C:961-1140.
"""
import numpy as np


def _coords(L):
    lx, ly, lz, lt = L
    t, z, y, x = np.meshgrid(np.arange(lt), np.arange(lz), np.arange(ly), np.arange(lx), indexing="ij")
    return x.ravel(), y.ravel(), z.ravel(), t.ravel()  # lexicographic order, x fastest


def fcanon_to_wilson_4d(f, L):
    """one 4D fermion volume, canonical -> WILSON (new array)"""
    lx, ly, lz, lt = L
    vol = lx * ly * lz * lt
    x, y, z, t = _coords(L)
    new = (x - x % 2 + lx * (y + ly * (z + lz * t)) + vol * ((x + y + z + t + 1) % 2)) // 2
    f = np.asarray(f).reshape(vol, 24)
    out = np.empty_like(f)
    out[new] = f
    return out.ravel()


def fconvert_dwf(f, L, ls):
    """5D fermion, canonical -> WILSON (DWF even-odd), as convert.C:704-760"""
    vol = int(np.prod(L))
    stride, half = 24 * vol, 12 * vol
    tmp = np.concatenate([fcanon_to_wilson_4d(f[s * stride:(s + 1) * stride], L) for s in range(ls)])
    out = np.empty_like(tmp)
    o, src = 0, 0
    for s in range(ls):  # odd part
        parity = (s + 1) % 2
        out[o:o + half] = tmp[src:src + half]
        o += half
        src += (2 * parity + 1) * half
    src = half
    for s in range(ls):  # even part
        parity = s % 2
        out[o:o + half] = tmp[src:src + half]
        o += half
        src += (2 * parity + 1) * half
    return out


def gcanon_to_wilson(u, L):
    """gauge field, canonical [site][mu][row][col] -> WILSON [parity][cb site][mu][col][row]"""
    lx, ly, lz, lt = L
    vol = lx * ly * lz * lt
    u = np.asarray(u).reshape(vol, 4, 3, 3, 2)
    out = np.empty((vol, 4, 3, 3, 2))
    idx = 0
    for cb in range(2):  # convert.C:281-299: WILSON site order
        for t in range(lt):
            for z in range(lz):
                for y in range(ly):
                    for x in range(lx):
                        if (x + y + z + t) % 2 == cb:
                            canon = x + lx * (y + ly * (z + lz * t))
                            out[idx] = u[canon].transpose(0, 2, 1, 3)  # (mu, col, row, re/im)
                            idx += 1
    return out.ravel()


def four2five(four, vol4, ls, s_u, s_l):
    five = np.zeros((ls, vol4, 24))
    four = np.asarray(four).reshape(vol4, 24)
    five[s_u, :, :12] = four[:, :12]
    five[s_l, :, 12:] = four[:, 12:]
    return five.ravel()


def five2four(five, vol4, ls, s_u, s_l):
    five = np.asarray(five).reshape(ls, vol4, 24)
    four = np.zeros((vol4, 24))
    four[:, :12] = five[s_u, :, :12]
    four[:, 12:] = five[s_l, :, 12:]
    return four.ravel()
