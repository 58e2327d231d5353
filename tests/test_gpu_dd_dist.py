"""The decomposed CG across processes: dd.cg over dd.DistRing with one t
slab per process (2 and 3 ranks, gloo, faces staged through host memory),
all on one GPU (tests/dd_dist_worker.py), against the whole lattice's
device CG: the same iteration count within one and the same solution.
This runs the cross-process path of the decomposition (the face exchange
and the global sums between ranks) on real slabs; with NCCL on several
GPUs the same code moves the device faces directly."""
import socket
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
WORKER = Path(__file__).resolve().parent / "dd_dist_worker.py"


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("kind,L,ls,ranks", [("wilson", "4x4x4x8", 1, 2), ("dwf", "4x4x2x12", 4, 3)])
def test_dd_cg_across_processes(kind, L, ls, ranks):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", str(ranks),
           "--master-addr", "127.0.0.1", "--master-port", str(_port()), str(WORKER), kind, L, str(ls)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "OK iterations" in r.stdout, r.stdout[-3000:] + r.stderr[-3000:]
