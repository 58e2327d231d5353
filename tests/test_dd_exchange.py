"""The face exchange of the t-slab decomposition (cps_veloc_b200.dd.
exchange_faces) among 2 and 3 gloo ranks on the CPU: every rank's to_prev
arrives in the previous rank's from_next and its to_next in the next rank's
from_prev, around the periodic ring."""
import os
import socket
from types import SimpleNamespace

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cps_veloc_b200 import dd


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, size, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        n = 64
        f = SimpleNamespace(to_prev=torch.full((n,), 10 * rank + 1, dtype=torch.uint8),
                            to_next=torch.full((n,), 10 * rank + 2, dtype=torch.uint8),
                            from_next=torch.zeros(n, dtype=torch.uint8), from_prev=torch.zeros(n, dtype=torch.uint8))
        dd.exchange_faces(f)
        nxt, prev = (rank + 1) % size, (rank - 1) % size
        ok = bool((f.from_next == 10 * nxt + 1).all() and (f.from_prev == 10 * prev + 2).all())
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size", [2, 3])
def test_exchange_faces_ring(size):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, size, port, q)) for r in range(size)]
    for pr in procs:
        pr.start()
    res = dict(q.get(timeout=120) for _ in range(size))
    for pr in procs:
        pr.join(timeout=60)
    assert res == {r: True for r in range(size)}
