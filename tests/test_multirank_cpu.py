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


def _split_main(rank: int, world: int, port: int, out_dir: str) -> None:
    # one list of read sets split over the ranks by estimated work; each rank
    # aligns its share (the oracle stands in for the GPU), rank 0 gathers
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    for sub in ("", "minipoa-rs_b200", "oracle"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import torch.distributed as dist

    import oracle
    from minipoa_b200 import shard, workloads
    from minipoa_b200.params import Params

    dist.init_process_group("gloo")
    sets = workloads.batched_sets(24, seed=77, lmax=500, dmax=10)
    shares = shard.partition([shard.set_work(s) for s in sets], world)
    mine = [sets[s] for s in shares[rank]]
    _, hashes = oracle.batch_run(Params(), mine, kernel=oracle.AUTO_AVX2, threads=1, out_format=2)
    got = [None] * world
    dist.all_gather_object(got, hashes)
    if rank == 0:
        merged = shard.gather(len(sets), shares, got)
        with open(os.path.join(out_dir, "split.txt"), "w") as f:
            f.write(" ".join(str(h) for h in merged) + "\n")
            f.write(" ".join(str(len(x)) for x in shares) + "\n")
    dist.destroy_process_group()


def test_split_batch_over_two_ranks_equals_single_process(tmp_path):
    port = _free_port()
    tmp.start_processes(_split_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    merged, sizes = open(tmp_path / "split.txt").read().splitlines()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from minipoa_b200 import workloads
    from minipoa_b200.params import Params

    sets = workloads.batched_sets(24, seed=77, lmax=500, dmax=10)
    _, whole = oracle.batch_run(Params(), sets, kernel=oracle.AUTO_AVX2, threads=1, out_format=2)
    assert [int(x) for x in merged.split()] == whole
    assert all(int(n) > 0 for n in sizes.split())


def test_partition_balances_work_and_covers_every_set():
    sys.path.insert(0, os.path.join(ROOT, "minipoa-rs_b200"))
    from minipoa_b200 import shard

    works = [float(w) for w in (100, 90, 80, 70, 60, 50, 40, 30, 20, 10, 5, 5)]
    for n in (1, 2, 3, 4, 8):
        sh = shard.partition(works, n)
        assert sorted(s for x in sh for s in x) == list(range(len(works)))
        loads = [sum(works[s] for s in x) for x in sh]
        # LPT: no rank exceeds the best possible by more than the largest set
        assert max(loads) <= sum(works) / n + max(works)
    assert shard.partition(works, 3) == shard.partition(works, 3)
