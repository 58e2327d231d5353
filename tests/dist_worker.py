"""Worker for test_bench_dist.py: run under torch.distributed.run with two
CPU ranks (gloo).  Exercises the benchmark's multi-rank plumbing: process
group setup, the max-over-ranks timing reduction, and the reference arm's
rank-0-only rule."""
import io
import os
import sys
from contextlib import redirect_stdout
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402


def main():
    ws, rank, local = bench.dist_env()
    assert ws == 2 and rank in (0, 1) and local == rank
    dist = bench.init_dist(ws)
    # each rank reports its own time; every rank must get the slowest one
    t = bench.max_over_ranks(dist, 1.0 + rank)
    assert t == 2.0, t
    dist.barrier()
    if rank == 1:
        # the reference arm runs on rank 0 only: rank 1 returns at once, silently
        buf = io.StringIO()
        with redirect_stdout(buf):
            rc = bench.run_reference_arm(bench.argparse.Namespace(gpus=2, steps=1, warmup=0))
        assert rc == 0 and buf.getvalue() == ""
    dist.barrier()
    dist.destroy_process_group()
    print(f"rank {rank} ok", flush=True)


if __name__ == "__main__":
    main()
