"""Worker for test_gpu_dd_dist.py, run under torch.distributed.run: each
rank holds one t slab of the lattice (its own Lattice, links and fields),
and the decomposed CG (dd.cg over dd.DistRing: faces and global sums
between the processes through gloo, faces staged through host memory)
solves MatPcDagMatPc x = b.  Rank 0 gathers the solution and compares it
with the whole lattice's device CG.  Every rank uses GPU 0; no kernel waits
on another process (the exchange is on the host)."""
import datetime
import os
import sys
from pathlib import Path

import numpy as np
import torch
import torch.distributed as dist

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE))
from cps_veloc_b200 import _abi as A  # noqa: E402
from cps_veloc_b200 import dd  # noqa: E402
from cps_veloc_b200.dirac import Lattice, gen_gauge, gen_gaussian  # noqa: E402
from test_gpu_dd import _join, _make, _slab_gauge, _slab_vec  # noqa: E402


def main():
    kind, L, ls = sys.argv[1], tuple(int(v) for v in sys.argv[2].split("x")), int(sys.argv[3])
    rank, size = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    A.check(A.lib().cpsgpu_set_device(0))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    mass = 0.1
    u = gen_gauge(L, seed=511)
    lat = Lattice((L[0], L[1], L[2], L[3] // size))
    lat.import_gauge(_slab_gauge(u, L, size, rank))
    dd.set_t_partition(lat, size, rank)
    D = _make(kind, lat, mass, ls)
    op = dd.DDOperator([D], dd.DistRing())
    vh = int(np.prod(L)) // 2
    b = gen_gaussian(24 * ls * vh, seed=512)
    fb, fx = dd.DeviceField(D), dd.DeviceField(D)
    fb.upload(_slab_vec(b, L, ls, size, rank))
    fx.upload(np.zeros(D.f_size))
    it, tr = dd.cg(op, [fx], [fb], stop_rsd=1e-11)
    part = torch.from_numpy(fx.download())
    parts = [torch.empty_like(part) for _ in range(size)]
    dist.all_gather(parts, part)
    if rank == 0:
        y = _join([q.numpy() for q in parts], L, ls)
        full = Lattice(L)
        full.import_gauge(u)
        Dfull = _make(kind, full, mass, ls)
        x = np.zeros(Dfull.f_size)
        r = Dfull.InvCg(x, b, stop_rsd=1e-11)
        err = float(np.linalg.norm(y - x) / np.linalg.norm(x))
        ok = abs(it - r.iterations) <= 1 and tr < 1e-11 and err < 1e-9
        print(f"{'OK' if ok else 'FAIL'} iterations {it} whole-lattice {r.iterations} true_res {tr:.3e} rel {err:.3e}",
              flush=True)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
