"""The decomposed CG's host recurrences and DistRing's global sums among 2
and 3 gloo ranks on the CPU (cps_veloc_b200.dd.cg, DistRing.allreduce).

Each rank holds one slab of a block-diagonal symmetric positive definite
system (a numpy stand-in for the slab's MatPcDagMatPc): the slabs share
nothing but the global sums, which is what the ring must provide.  Every
rank must take the iteration count and reach the solution of a CG on the
whole system computed in one process with the same recurrences."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

N = 48  # unknowns per slab


def _system(size, seed=7):
    rng = np.random.default_rng(seed)
    blocks, rhs = [], []
    for _ in range(size):
        m = rng.normal(size=(N, N))
        blocks.append(m @ m.T + 0.5 * np.eye(N))
        rhs.append(rng.normal(size=N))
    return blocks, rhs


class SlabOp:
    """one rank's slab: fields are numpy vectors, dot products go through
    the ring"""

    def __init__(self, A, ring):
        self.A, self.ring = A, ring

    def field(self):
        return [np.zeros(N)]

    def dot(self, a, b):
        return self.ring.allreduce(complex(sum(float(x @ y) for x, y in zip(a, b))))

    def mdagm(self, out, inp):
        out[0][:] = self.A @ inp[0]
        return self.dot(inp, out).real

    @staticmethod
    def axpby(out, a, x, y):
        out[:] = a * x + y


def _whole_system_cg(blocks, rhs, stop_rsd, max_num_iter):
    """the same recurrences on the whole block-diagonal system"""
    from scipy.linalg import block_diag

    A, b = block_diag(*blocks), np.concatenate(rhs)
    x = np.zeros_like(b)
    r = b - A @ x
    p = r.copy()
    rr, stop, k = r @ r, stop_rsd ** 2 * (b @ b), 0
    while k < max_num_iter - 1 and rr > stop:
        ap = A @ p
        alpha = rr / (p @ ap)
        x += alpha * p
        r -= alpha * ap
        rr_new = r @ r
        p = (rr_new / rr) * p + r
        rr = rr_new
        k += 1
    return k + 1, x


def _rank(rank, size, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=60))
    try:
        from cps_veloc_b200 import dd

        ring = dd.DistRing()
        s = ring.allreduce(complex(rank + 1, -rank))
        # the device-resident solver's all-reduce and exchange need NCCL: gloo is refused
        import torch
        refused = 0
        try:
            ring.allreduce_device(torch.zeros(2, dtype=torch.float64))
        except RuntimeError:
            refused += 1
        try:
            ring.exchange([None], sync=False)
        except RuntimeError:
            refused += 1
        blocks, rhs = _system(size)
        op = SlabOp(blocks[rank], ring)
        x = [np.zeros(N)]
        it, tr = dd.cg(op, x, [rhs[rank]], stop_rsd=1e-10, max_num_iter=500)
        q.put((rank, s, it, tr, x[0], refused))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("size", [2, 3])
def test_dist_ring_cg(size):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, size, port, q)) for r in range(size)]
    for pr in procs:
        pr.start()
    res = {}
    for _ in range(size):
        rank, s, it, tr, x, refused = q.get(timeout=120)
        res[rank] = (s, it, tr, x)
        assert refused == 2
    for pr in procs:
        pr.join(timeout=60)
    blocks, rhs = _system(size)
    it_ref, x_ref = _whole_system_cg(blocks, rhs, 1e-10, 500)
    total = complex(sum(r + 1 for r in range(size)), -sum(range(size)))
    for r in range(size):
        s, it, tr, x = res[r]
        assert s == total
        assert it == it_ref
        assert tr <= 1e-10
        assert np.linalg.norm(x - x_ref[r * N:(r + 1) * N]) <= 1e-9 * np.linalg.norm(x_ref)
