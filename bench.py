#!/usr/bin/env python3
"""Benchmark: batched independent partial-order alignments on B200.

Workload (default): 4,096 independent read sets, ancestor length log-uniform
in 200-5,000 bp, depth uniform in 10-60 reads, per-set error uniform in
2-15% split 60/20/20 among substitution / insertion / deletion (seed 1003);
default Params (static band b=100, f=40), i32 DP. A step is one full pass
of the read loop over every set (Graph::new, then align -> add_path ->
toposort for each read), all resident on the GPU.

Metric: GCUPS = 8-aligned band cells computed (retries included) / s / 1e9.
`value` is device time of the batched run with inputs already in HBM; `e2e`
goes through the C ABI from host buffers (upload, run, download and render
every set's consensus). The CPU baseline is the oracle's 8-lane AVX2 kernel
on the host's threads over a bounded sample of the same sets.

Multi-GPU: one process per GPU, each aligning its own 4,096 sets (weak
scaling, no collective on the data path); value = all ranks' cells / the
slowest rank's time.
"""
import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "minipoa-rs_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOAD = ("batched independent POA: 4096 read sets, ancestor 200-5000 bp log-uniform, depth 10-60, "
            "error 2-15% (60/20/20 sub/ins/del), default Params, consensus output")
METRIC = "GCUPS (batched POA, bit-exact)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--sets", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=1003)
    ap.add_argument("--lmax", type=int, default=5000, help="largest ancestor length (smaller for profiling runs)")
    ap.add_argument("--dmax", type=int, default=60, help="largest read depth (smaller for profiling runs)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-sets", type=int, default=64, help="sets timed in the plain per-read form")
    ap.add_argument("--mem-budget-gb", type=float, default=0.0,
                    help="device memory budget of the context (0: 90%% of free memory)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (small profiling runs)")
    ap.add_argument("--no-extra", action="store_true", help="skip the single-set and protein configurations")
    ap.add_argument("--split", action="store_true",
                    help="N>1: split one list of --sets sets over the ranks (strong scaling) instead of "
                         "--sets sets per rank (weak scaling)")
    ap.add_argument("--serve-jobs", type=int, default=1024, help="jobs of the serving loop's saturation run (0: skip)")
    ap.add_argument("--serve-seconds", type=float, default=12.0, help="length of the serving run at 80%% load")
    ap.add_argument("--autotune", type=int, default=1,
                    help="1: tune the batch's launch settings before the timed steps (0: defaults)")
    ap.add_argument("--c4a-only", type=int, default=0,
                    help="run only the protein-family configuration with this many families and print its "
                         "key (a small case for profiling the wide kernel form)")
    ap.add_argument("--c4b-reads", type=int, default=3,
                    help="reads per set of the int64 run (8 sets x 100 kbp, match 1000; 0: skip)")
    ap.add_argument("--seeded-reads", type=int, default=100,
                    help="reads of the seeded-window run (16.5 kbp ancestor, ~5%% error; 0: skip)")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value: float) -> float:
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(pg, value: float) -> float:
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def set_work(reads, params) -> float:
    """Estimated band cells of one read set (for sampling): reads x rows x band."""
    if not reads:
        return 0.0
    L = max(len(r) for r in reads)
    w = min(2.0 * (params.b + (L / params.f if params.f else L)) + 16.0, L + 16.0)
    return sum(len(r) for r in reads) * w * (1.0 + 0.03 * len(reads))


def cpu_sample(sets, params, seconds: float, threads: int, rate_per_thread: float = 0.12e9):
    """A fixed, size-stratified sample of the sets for the CPU leg: the 8
    largest sets, then every k-th set of the size-ordered list, with k chosen
    so the estimated work is about `seconds` on `threads` threads at
    `rate_per_thread` cells/s. Returned largest first, so the oracle's atomic
    queue keeps every thread busy until the end."""
    order = sorted(range(len(sets)), key=lambda s: -set_work(sets[s], params))
    budget = seconds * threads * rate_per_thread
    total = sum(set_work(sets[s], params) for s in order)
    k = max(1, int(total / max(1.0, budget)))
    pick = order[:8] + order[8::k]
    out, acc = [], 0.0
    for s in pick:
        if acc > budget and len(out) >= 8:
            break
        out.append(s)
        acc += set_work(sets[s], params)
    return out


def cpu_baseline(sets, params, seconds: float, threads: int = 0):
    """The oracle's 8-lane AVX2 i32 kernel over a fixed sample of the same
    sets (cpu_sample) in ONE call on `threads` host threads (default: all),
    largest set first, so the atomic work queue keeps every thread busy.
    Returns the measurement plus the sample's consensus hashes."""
    import oracle

    threads = threads or os.cpu_count() or 1
    sample = cpu_sample(sets, params, seconds, threads)
    part = [sets[s] for s in sample]
    t0 = time.perf_counter()
    cells, hashes = oracle.batch_run(params, part, kernel=oracle.AUTO_AVX2, threads=threads, out_format=0)
    elapsed = time.perf_counter() - t0
    return {
        "value": cells / elapsed / 1e9 if elapsed > 0 else None,
        "unit": "GCUPS",
        "cores": threads,
        "kind": "port",
        "sample": f"{len(sample)} of the {len(sets)} sets (the 8 largest, then every k-th by size; "
                  f"{cells / 1e9:.2f} G cells, {elapsed:.1f} s), 8-lane AVX2 i32 kernel, one call, "
                  f"largest first over {threads} threads",
    }, dict(zip(sample, hashes))


def cpu_single_thread(sets, params, seconds: float):
    """The same kernel on one thread over a small stratified sample (the
    reference's unseeded runs are single-threaded whatever -t is)."""
    import oracle

    order = sorted(range(len(sets)), key=lambda s: -set_work(sets[s], params))
    budget = seconds * 0.12e9
    total = sum(set_work(sets[s], params) for s in order)
    k = max(1, int(total / budget))
    sample = order[k // 2::k] or order[-1:]
    t0 = time.perf_counter()
    cells, _ = oracle.batch_run(params, [sets[s] for s in sample], kernel=oracle.AUTO_AVX2, threads=1, out_format=-1)
    dt = time.perf_counter() - t0
    return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": 1,
            "sample": f"{len(sample)} sets, every k-th by size ({cells / 1e9:.2f} G cells, {dt:.1f} s)"}


def consensus_parity(gpu_text: bytes, hashes: dict):
    """Compares the GPU's consensus of the sampled sets (from the all-sets
    output, split per set) with the oracle's hashes of the same sets."""
    import oracle

    head = b">consensus sequence\n"
    parts = gpu_text.split(head)[1:]
    bad = [s for s, h in hashes.items() if s >= len(parts) or oracle.fnv1a(head + parts[s]) != h]
    return {"sets_checked": len(hashes), "mismatches": len(bad), "output": "consensus FASTA bytes (FNV-1a)",
            "mismatched_sets": bad[:16]}


def serving_jobs(mp, params, ctx, n_jobs: int, seed: int = 1006):
    """Jobs drawn like the batched workload (ancestor 200-5000 bp log-uniform,
    error 2-15% split 60/20/20); 20% of them bring an initial graph: the GFA
    of 10-40 prior reads (aligned here in one batched launch and written with
    Graph::gfa) plus 5-20 new reads to extend it; the others are plain read
    sets of depth 10-60."""
    import numpy as np

    from minipoa_b200 import workloads

    rng = np.random.default_rng(seed)
    jobs, prior_sets, gfa_jobs = [], [], []
    for k in range(n_jobs):
        L = int(np.exp(rng.uniform(np.log(200), np.log(5000))))
        e = float(rng.uniform(0.02, 0.15))
        if rng.random() < 0.2:
            k0, k1 = int(rng.integers(10, 41)), int(rng.integers(5, 21))
            reads = workloads.read_set(rng, L, k0 + k1, 0.6 * e, 0.2 * e, 0.2 * e)
            prior_sets.append(reads[:k0])
            gfa_jobs.append(k)
            jobs.append([None, reads[k0:]])
        else:
            jobs.append([None, workloads.read_set(rng, L, int(rng.integers(10, 61)), 0.6 * e, 0.2 * e, 0.2 * e)])
    if prior_sets:
        pb = mp.Batch(params, prior_sets, ctx)
        pb.run(0)
        for k, s in zip(gfa_jobs, range(len(prior_sets))):
            jobs[k][0] = pb.output(s, 2)
        del pb
    return jobs


def serving_bench(mp, params, ctx, n_jobs: int, seconds: float, seed: int = 1006, pool_gb: float = 120.0):
    """Serving loop (continuous batching) on serving_jobs: saturated
    throughput (all jobs submitted at once), then Poisson arrivals at 80% of
    it, with each job's latency from submission to completion (measured by
    the server), split into queueing and running time, per job-size bucket."""
    import random

    jobs = serving_jobs(mp, params, ctx, n_jobs, seed)
    server = mp.Server(params, ctx=ctx, pool_bytes=int(pool_gb * 1e9) // 256 * 256)
    t0 = time.perf_counter()
    ids = [server.submit(r, gfa=g) for g, r in jobs]
    cells = 0
    for i in ids:
        server.wait(i, 300000.0)
        cells += server.info(i).cells
    sat_s = time.perf_counter() - t0
    print(f"[bench] serving: {n_jobs} jobs at once in {sat_s:.2f} s", file=sys.stderr, flush=True)
    for i in ids:
        server.release(i)
    sat_rate = n_jobs / sat_s
    rate = 0.8 * sat_rate
    rng = random.Random(seed)
    submitted, recs = [], []
    done = threading.Event()

    def reaper():
        k = 0
        while not (done.is_set() and k >= len(submitted)):
            if k >= len(submitted):
                time.sleep(0.0005)
                continue
            j, kind = submitted[k]
            server.wait(j, 300000.0)
            info = server.info(j)
            recs.append((info.latency_ms, info.queued_ms, info.cells, kind))
            server.release(j)
            k += 1

    th = threading.Thread(target=reaper)
    th.start()
    t0 = time.perf_counter()
    t_next = t0
    while t_next - t0 < seconds:
        now = time.perf_counter()
        if now < t_next:
            time.sleep(min(t_next - now, 0.002))
            continue
        g, r = jobs[rng.randrange(n_jobs)]
        submitted.append((server.submit(r, gfa=g), "gfa" if g is not None else "plain"))
        t_next += rng.expovariate(rate)
    done.set()
    th.join()
    span = time.perf_counter() - t0
    print(f"[bench] serving: {len(submitted)} Poisson arrivals at {rate:.0f}/s, drained in {span:.2f} s",
          file=sys.stderr, flush=True)
    server.close()

    def pct(v, q):
        v = sorted(v)
        return v[min(len(v) - 1, int(q * len(v)))] if v else None

    def summary(rows):
        return {"jobs": len(rows), "p50_ms": pct([r[0] for r in rows], 0.50), "p99_ms": pct([r[0] for r in rows], 0.99),
                "queued_p50_ms": pct([r[1] for r in rows], 0.50), "queued_p99_ms": pct([r[1] for r in rows], 0.99),
                "run_p50_ms": pct([r[0] - r[1] for r in rows], 0.50),
                "run_p99_ms": pct([r[0] - r[1] for r in rows], 0.99)}

    buckets = {"small (<10 M cells)": [r for r in recs if r[2] < 10e6],
               "medium (10-100 M cells)": [r for r in recs if 10e6 <= r[2] < 100e6],
               "large (>=100 M cells)": [r for r in recs if r[2] >= 100e6]}
    lat = [r[0] for r in recs]
    return {"workload": f"{n_jobs} jobs drawn like the batched workload, 20% extending a GFA graph of 10-40 prior "
                        f"reads with 5-20 new reads (seed {seed}); pool {pool_gb:g} GB",
            "saturated_jobs_per_s": sat_rate, "saturated_gcups": cells / sat_s / 1e9,
            "load": "Poisson arrivals at 80% of the saturated job rate", "arrival_jobs_per_s": rate,
            "jobs": len(recs), "gcups": sum(r[2] for r in recs) / span / 1e9,
            "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99), "max_ms": max(lat) if lat else None,
            "all": summary(recs), "by_size": {k: summary(v) for k, v in buckets.items()},
            "gfa_jobs": summary([r for r in recs if r[3] == "gfa"])}


def cpu_seeded(mp, params, reads, threads: int):
    """The seeded read loop on the CPU (the CPU baseline of the seeded
    workload): per read, the oracle graph's consensus, the seed windows from
    the same host function the GPU path uses (a shared input: the reference's
    own minimizer crate is not available), each window aligned with the
    oracle's poa on a pool of `threads` host threads (the reference's
    map_ordered over windows, src/align.rs:186) and the anchor nodes added as
    align::align does; then add_path and toposort. Returns (graph, windows)."""
    from concurrent.futures import ThreadPoolExecutor

    import oracle

    og = oracle.OracleGraph(params)
    n_win = 0
    with ThreadPoolExecutor(max_workers=threads) as ex:
        for r, q in enumerate(reads):
            if og.n_nodes() <= 2:
                items = [(0, params.encode("N"), None)] + [(None, params.encode(c), None) for c in q]
            else:
                cons, ids, _ = og.consensus(params)
                anchors, tail = mp.anchor_windows(params, q, cons)
                windows, beg, qbeg, prev, ok = [], 0, 0, None, bool(anchors)
                for a in anchors:
                    ts, qs = a.target_end + 1 - a.span, a.query_end + 1 - a.span
                    if not (a.span > 0 and a.target_end < len(ids) and a.query_end < len(q) and qs >= qbeg
                            and (prev is None or ts > prev)
                            and all(params.encode(cons[ts + o]) == params.encode(q[qs + o]) for o in range(a.span))):
                        ok = False
                        break
                    windows.append((beg, ids[ts], qbeg, qs, a.adaptive_before, ids[ts:a.target_end]))
                    beg, qbeg, prev = ids[a.target_end], a.query_end + 1, a.target_end
                if ok:
                    windows.append((beg, 1, qbeg, len(q), tail, []))
                    base = og.dump(len(params.alphabet))["base"]
                    parts = list(ex.map(lambda w: og.poa(params, w[0], w[1], q[w[2]:w[3]], w[4],
                                                         params.b if w[4] else params.win_band,
                                                         kernel=oracle.AUTO_AVX2), windows))
                    items = []
                    for w, part in zip(windows, parts):
                        items += part + [(i, base[i], None) for i in w[5]]
                    n_win += len(windows)
                else:
                    items = og.poa(params, 0, 1, q, True, params.b, kernel=oracle.AUTO_AVX2)
            og.add_path(params, r, items)
            og.toposort()
    return og, n_win


def seeded_bench(mp, ctx, n_reads: int, plain_reads: int = 20, seed: int = 1002, threads: int = 0):
    """Seeded windowed POA (-S -B -r1) on a 16.5 kbp ancestor with 100 reads at
    about 5% error (3/1/1% sub/ins/del, indel lengths geometric with mean
    1.5): windows/s with all windows of a read in one launch (one warp per
    window) on every read; the same with one launch per window on the first
    `plain_reads` reads (the batched/plain ratio is taken on those); and the
    CPU loop (cpu_seeded) on all host threads, with MSA bytes compared."""
    from minipoa_b200 import workloads
    from minipoa_b200.params import Params

    threads = threads or os.cpu_count() or 1
    reads = workloads.seeded_window_set(seed)[:n_reads]
    params = Params(seeding=True, adaptive=True, result=1)
    recs = [mp.Sequence(name=f"read{i}", seq=r) for i, r in enumerate(reads)]
    out = {"workload": f"16,500 bp ancestor, {len(reads)} reads (seed {seed}), -S -B -r1"}

    def gpu(rs, plain):
        ctx.tune_windows(plain)
        w0 = ctx.window_stats()
        t0 = time.perf_counter()
        g = mp.align_sequences(params, rs, ctx=ctx)
        dt = time.perf_counter() - t0
        w1 = ctx.window_stats()
        ctx.tune_windows(False)
        return g, {"reads": len(rs), "windows": w1[0] - w0[0], "launches": w1[1] - w0[1],
                   "fallback_reads": w1[2] - w0[2], "seconds": dt, "windows_per_s": (w1[0] - w0[0]) / dt,
                   "reads_per_s": len(rs) / dt}

    g_all, out["batched"] = gpu(reads, False)
    gp_b, out["batched_first"] = gpu(reads[:plain_reads], False)
    gp_p, out["plain_first"] = gpu(reads[:plain_reads], True)
    sub = recs[:plain_reads]
    out["identical_msa_batched_plain"] = gp_b.msa(params, sub) == gp_p.msa(params, sub)
    out["batched_over_plain"] = out["batched_first"]["windows_per_s"] / out["plain_first"]["windows_per_s"]
    t0 = time.perf_counter()
    og, n_win = cpu_seeded(mp, params, reads, threads)
    dt = time.perf_counter() - t0
    out["cpu"] = {"threads": threads, "seconds": dt, "windows": n_win, "windows_per_s": n_win / dt,
                  "kind": "oracle poa per window on a thread pool, windows from the same host seeding"}
    out["identical_msa_gpu_cpu"] = g_all.msa(params, recs) == og.msa(params, recs)
    return out


def c1_bench(mp, ctx, params, reps: int = 5):
    """One 1,000 bp x 20-read set (seed 1001; 1% sub, 0.5% ins, 0.5% del),
    consensus output, through the single-graph API (align_sequences: every
    read of the set in one launch, graph resident on the device), against the
    oracle's AVX2 kernel on one thread (the reference's unseeded runs are
    single-threaded whatever -t is). Latency per set and GCUPS; consensus
    bytes compared."""
    import oracle
    from minipoa_b200 import workloads

    reads = workloads.unseeded_consensus_set(1001)
    mp.align_sequences(params, reads, ctx).consensus(params)  # warm-up
    ts, cons = [], None
    for _ in range(reps):
        t0 = time.perf_counter()
        g = mp.align_sequences(params, reads, ctx)
        cons = g.consensus(params)[0]
        ts.append(time.perf_counter() - t0)
    oracle.reset_cells()
    t0 = time.perf_counter()
    o = oracle.align_sequences(params, reads, kernel=oracle.AUTO_AVX2)
    tc = time.perf_counter() - t0
    cells = oracle.cells()
    t = statistics.median(ts)
    return {"workload": "1,000 bp ancestor x 20 reads (seed 1001), -r0, default Params",
            "cells": cells, "gpu_ms_per_set": t * 1e3, "gpu_gcups": cells / t / 1e9,
            "timing": f"host wall clock through the C ABI (upload, all reads, download, consensus), median of {reps}",
            "cpu_1thread_ms": tc * 1e3, "cpu_1thread_gcups": cells / tc / 1e9,
            "consensus_identical": cons == o.consensus(params)[0]}


def c4a_bench(mp, ctx, n_fam: int = 1000, threads: int = 0):
    """Protein families (-f0 full DP, 20-letter alphabet, symmetric integer
    matrix): 1,000 families x 30 members of 300-800 residues at 20%
    divergence, in one batched launch; the oracle's AVX2 kernel on all host
    threads over a stratified sample of the families; consensus bytes of the
    sample compared."""
    import oracle
    from minipoa_b200 import workloads
    from minipoa_b200.params import Params

    threads = threads or os.cpu_count() or 1
    fams = workloads.protein_families(n_fam)
    params = Params(alphabet=workloads.PROTEIN_ALPHABET, matrix=workloads.protein_matrix(), f=0)
    b = mp.Batch(params, fams, ctx)
    b.run(0)
    st = b.run(0)
    out = b.output_all(0)
    sample = list(range(0, n_fam, max(1, n_fam // (4 * threads))))
    t0 = time.perf_counter()
    cells, hashes = oracle.batch_run(params, [fams[s] for s in sample], kernel=oracle.AUTO_AVX2, threads=threads,
                                     out_format=0)
    tc = time.perf_counter() - t0
    par = consensus_parity(out, dict(zip(sample, hashes)))
    del b
    return {"workload": f"{n_fam} protein families x 30 (300-800 aa, 15% sub + 5% indels), -f0, 20x20 matrix",
            "cells": st.cells, "gpu_ms": st.device_ms, "gpu_gcups": st.cells / st.device_ms / 1e6,
            "rows_generic": st.rows_generic,
            "cpu": {"gcups": cells / tc / 1e9, "cores": threads, "sample": f"{len(sample)} families"},
            "parity": par}


def c4b_bench(mp, ctx, reads_per_set: int, threads: int = 0):
    """DNA sets whose scores overflow int32 (match score 1000, as -M1000):
    8 sets of a 100,000 bp ancestor (seed 1005) x 20 reads at 1% error; the
    score guard (align.rs:493-529) selects the exact int64 kernel on the GPU
    as in the reference. Bounded: the first `reads_per_set` reads of every set
    in one batched launch (about 0.6 G band cells per alignment); the oracle's
    scalar int64 kernel on host threads over the first two sets with the same
    reads; consensus bytes of those sets compared."""
    import numpy as np

    import oracle
    from minipoa_b200 import workloads
    from minipoa_b200.params import Params

    threads = threads or os.cpu_count() or 1
    rng = np.random.default_rng(1005)
    full = [workloads.read_set(rng, 100000, 20, 0.006, 0.002, 0.002) for _ in range(8)]
    sets = [s[:reads_per_set] for s in full]
    params = Params.from_cli_scores(match=1000)
    o_probe = oracle.align_sequences(params, sets[0][:1])
    i64 = not o_probe.i32_scores_safe(params, 0, 1, len(sets[0][1]))
    b = mp.Batch(params, sets, ctx)
    st = b.run(0)
    out = b.output_all(0)
    del b
    sample = [0, 1]
    t0 = time.perf_counter()
    cells, hashes = oracle.batch_run(params, [sets[s] for s in sample], kernel=oracle.AUTO_AVX2,
                                     threads=min(threads, len(sample)), out_format=0)
    tc = time.perf_counter() - t0
    par = consensus_parity(out, dict(zip(sample, hashes)))
    return {"workload": f"8 sets x 100,000 bp ancestor (seed 1005), 1% error, match 1000 (-M1000): "
                        f"the first {reads_per_set} of 20 reads per set",
            "int64_kernel": i64, "cells": st.cells, "gpu_ms": st.device_ms,
            "gpu_gcups": st.cells / st.device_ms / 1e6, "relaunch_passes": st.relaunches,
            "cpu": {"gcups": cells / tc / 1e9, "cores": min(threads, len(sample)),
                    "kind": "oracle scalar int64 kernel (the score guard's choice), one set per thread",
                    "sample": f"sets {sample} with the same reads"},
            "parity": par}


def load_traffic():
    """DRAM bytes per launch of the batched kernel from the committed ncu
    summary, scaled to this run's cells (null when absent)."""
    path = os.path.join(ROOT, "profiles", "k_batch_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def main():
    args = parse()
    if args.c4a_only:
        import minipoa_b200 as mp

        ctx = mp.Context(0, mem_budget=int(args.mem_budget_gb * (1 << 30)))
        print(json.dumps({"c4a_protein": c4a_bench(mp, ctx, args.c4a_only)}))
        return
    world, rank, local, pg = dist_setup(args)
    from minipoa_b200 import workloads
    from minipoa_b200.params import Params

    params = Params()
    if args.split and world > 1:
        # strong scaling: one list of sets split over the ranks by estimated
        # work (minipoa_b200.shard), the same split computed on every rank
        from minipoa_b200 import shard

        every = workloads.batched_sets(args.sets, seed=args.seed, lmax=args.lmax, dmax=args.dmax)
        share = shard.partition([shard.set_work(x) for x in every], world)[rank]
        sets = [every[s] for s in share]
        del every
    else:
        sets = workloads.batched_sets(args.sets, seed=args.seed + rank, lmax=args.lmax, dmax=args.dmax)

    if args.impl == "reference":
        if rank != 0:
            return
        t_steps = []
        cb = None
        for k in range(args.warmup + args.steps):
            cb, _ = cpu_baseline(sets, params, max(2.0, args.cpu_seconds / max(1, args.steps)))
            if k >= args.warmup:
                t_steps.append(cb)
        vals = [c["value"] for c in t_steps]
        v = statistics.median(vals)
        line = {
            "impl": "reference", "metric": METRIC, "value": v, "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "sets": args.sets, "seed": args.seed,
                       "sample": "bounded per step", "l2": "inputs larger than L2"},
            "cpu_baseline": {**t_steps[-1], "value": v},
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import minipoa_b200 as mp

    ctx = mp.Context(local, mem_budget=int(args.mem_budget_gb * (1 << 30)))
    batch = mp.Batch(params, sets, ctx)
    warm = None
    for _ in range(args.warmup):
        warm = batch.run(0)
    tuning = None
    if args.autotune:
        # launch settings per size bucket (warps per SM, giant threshold):
        # every candidate runs the whole batch once; the fastest is applied
        # and cached (the end-to-end leg's batch picks it up from the cache)
        t = batch.autotune()
        tuning = {"warps_per_sm": t.warps_per_sm, "giant_factor": t.giant_factor, "giant_alone": t.giant_alone,
                  "trials": t.trials,
                  "tuned_ms": t.device_ms, "default_ms": warm.device_ms if warm else None}
    barrier(pg)
    clocks = ClockSampler(local)
    clocks.start()
    steps = []
    for _ in range(args.steps):
        steps.append(batch.run(0))
        s = steps[-1]
        print(f"[bench] rank {rank} step: {s.cells / 1e9:.2f} G cells, {s.device_ms:.1f} ms device, "
              f"{s.kernel_ms:.1f} ms kernel, {s.cells / s.device_ms / 1e6:.1f} GCUPS, passes {1 + s.relaunches}, "
              f"slots {s.slots}", file=sys.stderr, flush=True)
    clock_info = clocks.stop()
    barrier(pg)
    dev_ms = sum(s.device_ms for s in steps)
    kern_ms = sum(s.kernel_ms for s in steps)
    cells = sum(s.cells for s in steps)
    dp_bytes = sum(s.dp_bytes for s in steps)
    launches = sum(s.launches for s in steps)
    max_ms = reduce_max(pg, dev_ms)
    all_cells = reduce_sum(pg, float(cells))
    value = all_cells / (max_ms / 1e3) / 1e9
    reads = sum(s.reads for s in steps)
    first_slots, first_passes = steps[0].slots, steps[0].relaunches
    del batch  # releases its DP arena pool before the end-to-end leg
    gc.collect()

    # end to end through the C ABI from host buffers
    e2e_vals, h2d, d2h = [], 0, 0
    e2e_parts = []
    out = None
    for _ in range(0 if args.no_e2e else max(1, min(args.steps, 2))):
        t0 = time.perf_counter()
        b2 = mp.Batch(params, sets, ctx)
        t1 = time.perf_counter()
        st = b2.run(0)
        t2 = time.perf_counter()
        out = b2.output_all(0)
        t3 = time.perf_counter()
        h2d, d2h = b2.transfer_bytes()
        del b2
        dt = time.perf_counter() - t0
        e2e_vals.append(st.cells / dt / 1e9)
        e2e_parts.append({"create_s": t1 - t0, "run_s": t2 - t1, "run_device_s": st.device_ms / 1e3,
                          "output_s": t3 - t2, "release_s": t0 + dt - t3})
        assert out.count(b">consensus sequence\n") == len(sets)
    e2e_v = None
    if e2e_vals:
        e2e_v = reduce_sum(pg, statistics.median(e2e_vals)) if pg else statistics.median(e2e_vals)

    # plain form (one launch per read) on a prefix of the sets
    plain = None
    if args.plain_sets > 0 and rank == 0:
        sub = sets[: args.plain_sets]
        bp = mp.Batch(params, sub, ctx)
        bp.run(0)
        sb = bp.run(0)
        sp = bp.run(1)
        plain = {"sets": len(sub), "plain_gcups": sp.cells / (sp.device_ms / 1e3) / 1e9,
                 "batched_gcups": sb.cells / (sb.device_ms / 1e3) / 1e9,
                 "plain_reads_per_s": sp.reads / (sp.device_ms / 1e3),
                 "batched_reads_per_s": sb.reads / (sb.device_ms / 1e3), "plain_launches": sp.launches}
        del bp

    peak, peak_kind = measured_peaks()
    avg_launch_ms = kern_ms / max(1, sum(1 + s.relaunches for s in steps))
    bytes_per_launch = dp_bytes / max(1, sum(1 + s.relaunches for s in steps))
    achieved = bytes_per_launch / (avg_launch_ms / 1e3) / 1e9
    traffic = load_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "algorithmic_bytes": "12 B/cell: the int32 M, D, I states stored per band cell for the traceback",
                "kernel": "k_batch",
                "traffic": None if traffic is None else traffic.get("bytes_per_cell", 0) * cells / max(
                    1, sum(1 + s.relaunches for s in steps))}

    serving = None
    if rank == 0 and args.serve_jobs > 0:
        try:
            serving = serving_bench(mp, params, ctx, args.serve_jobs, args.serve_seconds)
        except Exception as e:  # the throughput line above stands on its own
            serving = {"error": str(e)}

    c1 = c4a = c4b = None
    if rank == 0 and not args.no_extra and args.c4b_reads > 1:
        try:
            c4b = c4b_bench(mp, ctx, args.c4b_reads)
        except Exception as e:
            c4b = {"error": str(e)}
    if rank == 0 and not args.no_extra:
        try:
            c1 = c1_bench(mp, ctx, params)
        except Exception as e:
            c1 = {"error": str(e)}
        try:
            c4a = c4a_bench(mp, ctx)
        except Exception as e:
            c4a = {"error": str(e)}

    seeded = None
    if rank == 0 and args.seeded_reads > 0:
        try:
            seeded = seeded_bench(mp, ctx, args.seeded_reads)
        except Exception as e:
            seeded = {"error": str(e)}

    cb, parity = None, None
    if rank == 0 and not args.no_cpu_baseline:
        cb, hashes = cpu_baseline(sets, params, args.cpu_seconds)
        cb["single_thread"] = cpu_single_thread(sets, params, max(3.0, args.cpu_seconds / 3))
        if out is not None:
            parity = consensus_parity(out, hashes)
            print(f"[bench] parity: {parity['sets_checked']} sets checked, {parity['mismatches']} mismatches",
                  file=sys.stderr, flush=True)

    # integer-ALU roofline: (6 + 5 P) adds and maxes per cell, P the in-band
    # predecessors (counted as predecessor-cell updates), against the measured
    # integer throughput of this GPU
    int_roof = None
    try:
        peaks = mp.int_peak(local)
        int_peak = max(peaks)
        pred_cells = sum(s.pred_cells for s in steps)
        ops = 6.0 * cells + 5.0 * pred_cells
        ach = ops / (kern_ms / 1e3)
        int_roof = {"bound": "int32 ALU", "achieved": ach / 1e12, "peak": int_peak / 1e12, "unit": "Tops/s",
                    "frac": ach / int_peak, "ops_per_cell": ops / max(1, cells),
                    "preds_per_cell": pred_cells / max(1, cells),
                    "peak_source": "measured on this GPU (poa_probe_int_peak): add, max, fused add-max = "
                                   + ", ".join(f"{x / 1e12:.1f}" for x in peaks) + " Tops/s; the largest is the peak",
                    "kernel": "k_batch"}
    except Exception as e:
        int_roof = {"error": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if (args.split and world > 1) else "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD.replace("200-5000", f"200-{args.lmax}").replace("10-60", f"10-{args.dmax}"),
                       "sets": args.sets, "seed": args.seed, "reads_per_step": reads // args.steps,
                       "cells_per_step": cells // args.steps, "l2": "inputs larger than L2 (no flush needed)",
                       "parallelism": f"{world} independent GPU(s)", "slots": first_slots,
                       "relaunch_passes": first_passes, "reads_per_s": reads / (dev_ms / 1e3),
                       "paths": {"giant_jobs_with_helpers": steps[0].coop_jobs, "rows_4_stripe": steps[0].rows_g4,
                                 "rows_generic": steps[0].rows_generic,
                                 "pred_rows_from_arena": steps[0].far_preds},
                       "tuning": tuning},
            "roofline": roofline,
            "roofline_int": int_roof,
            "parity": parity,
            "cpu_baseline": cb,
            "e2e": {"value": e2e_v, "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "breakdown": e2e_parts[-1] if e2e_parts else None},
            "gpu_launches": launches,
            "clocks": clock_info,
            "plain_vs_batched": plain,
            "serving": serving,
            "seeded": seeded,
            "c1_single_set": c1,
            "c4a_protein": c4a,
            "c4b_int64": c4b,
        }
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
