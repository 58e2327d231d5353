"""Time the hop kernel (Dslash) and MatPcDagMatPc of one operator, per
precision, from HBM (the launches rotate over fields larger than L2):

    python -m cps_veloc_b200.dslash_test --lattice 16x16x16x32 --ls 16 --kind dwf --prec 0,1,2 [--reps 40]

Prints one line per precision: ms per Dslash, GB/s of its algorithmic bytes,
ms per MatPcDagMatPc and its GB/s.  Under a profiler, --reps 1 and
--no-mdagm keep the launch count small.  --force times the HMC fermion force
instead (CalcHmdForceVecs + the force kernel, FP64; Wilson, DWF, Mobius).
--dd N times the t-slab decomposed dslash (Wilson, DWF; FP64, FP32).
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
    ap.add_argument("--shape", default="",
                    help="sites,slices,slices_per_thread[,order] of the hop launches (overrides the autotuner; "
                         "order 0 slices first, 1 sites first)")
    ap.add_argument("--m5inv", action="store_true",
                    help="time the Mobius M5^-1 (the standalone Ls x Ls mixing) instead of the hop")
    ap.add_argument("--mix-impl", type=int, default=0,
                    help="Mobius mixing kernel: 0 default (FP16: bulk-staged), 1 tensor cores (FP16), "
                         "2 shared memory, 3 register-tiled")
    ap.add_argument("--dd", type=int, default=0,
                    help="time the t-slab decomposed dslash over this many slabs (one process; see time_dd)")
    args = ap.parse_args(argv)
    L = tuple(int(x) for x in args.lattice.split("x"))
    if args.dd:
        return time_dd(args, L)
    lat = Lattice(L)
    lat.import_gauge(gen_gauge(L, seed=20261203))
    if args.kind == "wilson":
        D = DiracOpWilson(lat, mass=args.mass)
    elif args.kind == "dwf":
        D = DiracOpDwf(lat, mass=args.mass, ls=args.ls)
    else:
        D = DiracOpMobius(lat, mass=args.mass, ls=args.ls)
    if args.m5inv:
        if args.kind != "mobius":
            raise SystemExit("--m5inv needs --kind mobius")
        D.set_mix_impl(args.mix_impl)
        for prec in (int(p) for p in args.prec.split(",")):
            ms, by = C.c_double(), C.c_double()
            A.check(A.lib().cpsgpu_time_m5inv(D._h, prec, args.reps, C.byref(ms), C.byref(by)))
            print(f"prec {prec} mix kernel {args.mix_impl}: m5inv {ms.value:.4f} ms "
                  f"{by.value / ms.value / 1e6:.0f} GB/s ({by.value:.0f} B)", flush=True)
        return 0
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
        if args.shape:
            D.set_hop_shape(prec, *(int(x) for x in args.shape.split(",")))
        ms, by = C.c_double(), C.c_double()
        A.check(A.lib().cpsgpu_time_dslash(D._h, prec, 1, 0, args.reps, C.byref(ms), C.byref(by)))
        line = f"prec {prec} shape {D.hop_shape(prec)}: dslash {ms.value:.4f} ms {by.value / ms.value / 1e6:.0f} GB/s ({by.value:.0f} B)"
        if not args.no_mdagm:
            m2, b2 = C.c_double(), C.c_double()
            A.check(A.lib().cpsgpu_time_mdagm(D._h, prec, max(1, args.reps // 4), C.byref(m2), C.byref(b2)))
            line += f"; mdagm {m2.value:.4f} ms {b2.value / m2.value / 1e6:.0f} GB/s"
        print(line, flush=True)
    return 0


def time_dd(args, L) -> int:
    """The t-slab decomposed dslash with N slabs played by one process: per
    repetition every slab packs its faces, the faces move by device copies
    (what NCCL does between GPUs), and every slab runs its halo hop; against
    the same loop of whole-lattice dslashes on device fields.  Both are host
    clocked with a device synchronize after every call, so the ratio shows
    the decomposition's overhead (pack, copies, halo reads), not a
    multi-GPU time (the slabs here run one after another)."""
    import time

    import numpy as np
    import torch

    from . import dd
    from .dirac import gen_gaussian

    n = args.dd
    u = gen_gauge(L, seed=20261203)
    mk = (lambda lat: DiracOpWilson(lat, mass=args.mass)) if args.kind == "wilson" else \
        (lambda lat: DiracOpDwf(lat, mass=args.mass, ls=args.ls))
    ls = 1 if args.kind == "wilson" else args.ls
    vh = int(np.prod(L)) // 2
    face, lt = vh // L[3], L[3] // n
    for prec in [int(p) for p in args.prec.split(",") if int(p) in (0, 1)]:
        full = Lattice(L)
        full.import_gauge(u)
        Df = mk(full)
        x = gen_gaussian(Df.f_size, seed=7)
        fi, fo = dd.DeviceField(Df, prec), dd.DeviceField(Df, prec)
        fi.upload(x)
        slabs = []
        for r in range(n):
            lat = Lattice((L[0], L[1], L[2], lt))
            lat.import_gauge(np.ascontiguousarray(u.reshape(2, vh, 72)[:, r * lt * face:(r + 1) * lt * face]).ravel())
            dd.set_t_partition(lat, n, r)
            D = mk(lat)
            a, b = dd.DeviceField(D, prec), dd.DeviceField(D, prec)
            a.upload(np.ascontiguousarray(x.reshape(ls, vh, 24)[:, r * lt * face:(r + 1) * lt * face]).ravel())
            slabs.append((lat, D, a, b, dd.Faces(D, prec)))

        def one_dd():
            for lat, D, a, b, f in slabs:
                dd.pack(D, a, 0, 0, f)
            for r in range(n):
                slabs[r][4].from_next.copy_(slabs[(r + 1) % n][4].to_prev)
                slabs[r][4].from_prev.copy_(slabs[(r - 1) % n][4].to_next)
            torch.cuda.synchronize()
            for lat, D, a, b, f in slabs:
                dd.dslash(D, b, a, 0, 0, f)

        def one_dd_overlap():
            for lat, D, a, b, f in slabs:
                dd.pack(D, a, 0, 0, f)
                dd.dslash_interior(D, b, a, 0, 0)
            for r in range(n):
                slabs[r][4].from_next.copy_(slabs[(r + 1) % n][4].to_prev)
                slabs[r][4].from_prev.copy_(slabs[(r - 1) % n][4].to_next)
            torch.cuda.current_stream().synchronize()
            for lat, D, a, b, f in slabs:
                dd.dslash_boundary(D, b, a, 0, 0, f)

        def one_full():
            A.check(A.lib().cpsgpu_dslash_field(Df._h, fo._h, fi._h, 0, 0))
            torch.cuda.synchronize()

        res = {}
        for name, fn in (("whole", one_full), ("dd", one_dd), ("dd_overlap", one_dd_overlap)):
            for _ in range(3):
                fn()
            t0 = time.perf_counter()
            for _ in range(args.reps):
                fn()
            res[name] = (time.perf_counter() - t0) / args.reps * 1e3
        nbytes = slabs[0][4].to_prev.numel()
        print(f"prec {prec}: {n} slabs, whole-lattice dslash {res['whole']:.4f} ms, decomposed {res['dd']:.4f} ms "
              f"(ratio {res['dd'] / res['whole']:.2f}), interior / boundary split {res['dd_overlap']:.4f} ms, "
              f"{4 * nbytes * n} face bytes moved per dslash")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

