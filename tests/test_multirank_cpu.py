"""Multi-rank plumbing of bench.py on CPU: two gloo ranks, no GPU.

The batched path shards by independent read sets: each rank draws its own
sets (seed + rank) and there is no exchange on the data path; the only
collectives are the timing max and the cell-count sum that make the job's
aggregate value. These tests run that host logic as two processes.
"""
import hashlib
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as tmp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "minipoa-rs_b200"))
    import bench
    from minipoa_b200 import workloads

    w, r, _, pg = bench.dist_setup(None)
    assert (w, r) == (world, rank) and pg is not None
    # per-rank device time and cells, as the timed region produces them
    t_ms = 100.0 + 50.0 * rank
    cells = 1000.0 * (rank + 1)
    bench.barrier(pg)
    mx = bench.reduce_max(pg, t_ms)
    total = bench.reduce_sum(pg, cells)
    sets = workloads.batched_sets(8, seed=1003 + rank, lmax=400, dmax=12)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        digest = hashlib.sha256(b"|".join(b",".join(s) for s in sets)).hexdigest()
        f.write(f"{mx} {total} {digest}\n")
    pg.destroy_process_group()


def test_two_gloo_ranks_reduce_time_and_cells(tmp_path):
    port = _free_port()
    tmp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    lines = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(2)]
    for mx, total, _ in lines:
        assert float(mx) == 150.0  # the slowest rank's device time
        assert float(total) == 3000.0  # every rank's cells
    # weak scaling: each rank aligns its own, different read sets
    assert lines[0][2] != lines[1][2]


def test_single_process_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench

    world, rank, _, pg = bench.dist_setup(None)
    assert (world, rank, pg) == (1, 0, None)
    assert bench.reduce_max(pg, 7.0) == 7.0 and bench.reduce_sum(pg, 7.0) == 7.0
