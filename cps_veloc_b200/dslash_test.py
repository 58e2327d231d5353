"""Time the hop kernel (Dslash) and MatPcDagMatPc of one operator, per
precision, from HBM (the launches rotate over fields larger than L2):

    python -m cps_veloc_b200.dslash_test --lattice 16x16x16x32 --ls 16 --kind dwf --prec 0,1,2 [--reps 40]

Prints one line per precision: ms per Dslash, GB/s of its algorithmic bytes,
ms per MatPcDagMatPc and its GB/s.  Under a profiler, --reps 1 and
--no-mdagm keep the launch count small.  --force times the HMC fermion force
instead (CalcHmdForceVecs + the force kernel, FP64; Wilson, DWF, Mobius).
"""
from __future__ import annotations

import argparse
import ctypes as C

from . import _abi as A
from .dirac import DiracOpDwf, DiracOpMobius, DiracOpWilson, Lattice, gen_gauge


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--lattice", default="16x16x16x32")
    ap.add_argument("--ls", type=int, default=16)
    ap.add_argument("--kind", default="dwf", choices=["wilson", "dwf", "mobius"])
    ap.add_argument("--mass", type=float, default=0.01)
    ap.add_argument("--prec", default="0,1,2", help="comma list: 0 FP64, 1 FP32, 2 FP16")
    ap.add_argument("--reps", type=int, default=40)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-mdagm", action="store_true")
    ap.add_argument("--force", action="store_true", help="time the HMC fermion force instead")
    ap.add_argument("--link-reals", type=int, default=0,
                    help="link form of the FP32/FP16 operators (12, 18, 112, 118; 0: default or autotuned)")
    args = ap.parse_args(argv)
    L = tuple(int(x) for x in args.lattice.split("x"))
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=20261203))
    if args.kind == "wilson":
        D = DiracOpWilson(lat, mass=args.mass)
    elif args.kind == "dwf":
        D = DiracOpDwf(lat, mass=args.mass, ls=args.ls)
    else:
        D = DiracOpMobius(lat, mass=args.mass, ls=args.ls)
    if args.force:
        tot, ker, by = C.c_double(), C.c_double(), C.c_double()
        A.check(A.lib().cpsgpu_time_fforce(D._h, args.reps, C.byref(tot), C.byref(ker), C.byref(by)))
        print(f"force: {tot.value:.4f} ms per call; force kernel {ker.value:.4f} ms "
              f"{by.value / ker.value / 1e6:.0f} GB/s ({by.value:.0f} B)", flush=True)
        return 0
    for prec in (int(p) for p in args.prec.split(",")):
        if not args.no_autotune:
            D.autotune(prec)
        if args.link_reals and prec != A.DOUBLE:
            lat.set_link_reals(prec, args.link_reals)
        ms, by = C.c_double(), C.c_double()
        A.check(A.lib().cpsgpu_time_dslash(D._h, prec, 1, 0, args.reps, C.byref(ms), C.byref(by)))
        line = f"prec {prec}: dslash {ms.value:.4f} ms {by.value / ms.value / 1e6:.0f} GB/s ({by.value:.0f} B)"
        if not args.no_mdagm:
            m2, b2 = C.c_double(), C.c_double()
            A.check(A.lib().cpsgpu_time_mdagm(D._h, prec, max(1, args.reps // 4), C.byref(m2), C.byref(b2)))
            line += f"; mdagm {m2.value:.4f} ms {b2.value / m2.value / 1e6:.0f} GB/s"
        print(line, flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
