"""GPU parity on the code paths the benchmark times, against the CPU oracle.

The batched benchmark launches thousands of read sets, so every block of the
persistent kernel has its full eight warps and the largest sets run as
"giants" with three helper warps computing their DP rows (cooperative rows).
Sets of 3.6 kbp and more have bands of 385-512 columns (the 4-stripe row
tile), and high-error sets have predecessor rows that left the shared-memory
ring. A small batch reaches none of these, so these tests build batches that
do, assert from the run's counters that each path ran, and compare every
set's output with the oracle.

Static-band reads run their DP either row at a time (striped rows, the ring,
giants with helper warps; the default) or as a row wavefront (a lane per
row). The static-band tests run the batch once with each form forced
(MINIPOA_DP_ROWS, read when the batch is created), once with each read's own
choice ("auto") and once with the default.

Also here: protein families with full DP (-f0, bands wider than 512 columns:
the generic row) and an i64 set whose reads are longer than the query bytes
kept in shared memory.
"""
import contextlib
import os

import numpy as np
import pytest

import refcases as rc
from minipoa_b200.params import Params, Sequence

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def mp():
    import minipoa_b200 as m

    m.default_context()
    return m


def _full_machine_sets(seed, n_giants, giant_len, giant_depth, n_small):
    """n_giants large high-error sets first, then many small ones, so that a
    launch has one slot per warp of every SM and the giants are marked."""
    rng = np.random.default_rng(seed)
    sets = []
    for g in range(n_giants):
        e = 0.08 + 0.02 * g
        sets.append(rc.synthetic_reads(rng, giant_len + 150 * g, giant_depth, 0.6 * e, 0.2 * e, 0.2 * e))
    for _ in range(n_small):
        L = int(rng.integers(40, 140))
        e = rng.uniform(0.02, 0.15)
        sets.append(rc.synthetic_reads(rng, L, int(rng.integers(3, 7)), 0.6 * e, 0.2 * e, 0.2 * e))
    return sets


@contextlib.contextmanager
def _env(name, value):
    old = os.environ.get(name)
    if value is None:
        os.environ.pop(name, None)
    else:
        os.environ[name] = value
    try:
        yield
    finally:
        if old is None:
            os.environ.pop(name, None)
        else:
            os.environ[name] = old


@contextlib.contextmanager
def _dp_rows(mode, wide=None):
    """Sets the static-band DP form of batches created inside the block:
    "rows" (row at a time), "wave" (row wavefront), "auto" (each read's
    choice) or None (the default); and the batched kernel's row form: wide
    "1" (bands up to 2048 columns in striped segments), "0" (the narrow
    form) or None (the default for the parameters)."""
    with _env("MINIPOA_DP_ROWS", mode), _env("MINIPOA_WIDE_ROWS", wide):
        yield


def _gfa_hashes_match(oracle, batch, params, sets):
    _, want = oracle.batch_run(params, sets, kernel=oracle.AUTO_AVX2, threads=THREADS, out_format=2)
    bad = [s for s in range(len(sets)) if oracle.fnv1a(batch.output(s, 2)) != want[s]]
    return bad


@pytest.mark.parametrize("adaptive,dp,wide", [(False, "rows", None), (False, "wave", None), (False, "auto", None),
                                             (True, None, None), (False, "rows", "1"), (True, None, "1")])
def test_full_machine_batch_with_giants_matches_oracle(mp, oracle, adaptive, dp, wide):
    params = Params(adaptive=adaptive)
    sets = _full_machine_sets(2024 + int(adaptive), 4, 4200, 30, 1180)
    with _dp_rows(dp, wide):
        batch = mp.Batch(params, sets)
    batch.tune(8)  # full 8-warp blocks: the giant runs on warp 4 with warps 0-2 as helpers
    st = batch.run(0)
    # one slot per resident warp of every SM in the first pass: full 8-warp
    # blocks (an adaptive giant may outgrow its arena and finish in a second
    # pass, which the comparison below covers too)
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert st.slots == min(len(sets), sms * 8)
    if wide is None:
        # (the wide form keeps every row of these sets in the ring: its
        # predecessors leave the ring only by distance, which these graphs'
        # edges rarely reach; the wide-band tests cover its arena reads)
        assert st.far_preds > 0, "no predecessor state was read back from the arena"
    if adaptive or dp == "rows":
        assert st.wave_reads == 0
        assert st.rows_g4 > 0, "no 4-stripe rows ran"
    if not adaptive and dp != "wave":
        assert st.coop_jobs >= 1, "no giant ran cooperative rows"
    if dp == "wave":
        # every static-band read but the giants' (their helper warps run rows)
        assert st.wave_reads > 0, "the row wavefront did not run"
    for s in range(len(sets)):
        assert batch.status(s) is None
    # every set: GFA bytes (graph, edges in order, paths) against the oracle
    assert _gfa_hashes_match(oracle, batch, params, sets) == []
    # the giants and a sample of small sets: whole graphs and MSA bytes
    rng = np.random.default_rng(7)
    sample = list(range(4)) + sorted(rng.choice(np.arange(4, len(sets)), 12, replace=False).tolist())
    for s in sample:
        reads = sets[s]
        o = oracle.align_sequences(params, reads, kernel=oracle.AUTO_AVX2)
        recs = [Sequence(name=f"read{i}", seq=x) for i, x in enumerate(reads)]
        assert batch.graph(s).dump() == o.dump(5), f"set {s}"
        assert batch.output(s, 0) == ">consensus sequence\n" + o.consensus(params)[0].decode() + "\n"
        assert batch.output(s, 1, recs) == o.msa(params, recs)
    # consensus of every set through the all-sets call
    allc = batch.output_all(0).decode()
    _, want0 = oracle.batch_run(params, sets, kernel=oracle.AUTO_AVX2, threads=THREADS, out_format=0)
    parts = allc.split(">consensus sequence\n")[1:]
    assert len(parts) == len(sets)
    assert [oracle.fnv1a(">consensus sequence\n" + p) for p in parts] == want0


def test_protein_families_full_dp_wide_rows_match_oracle(mp, oracle):
    # 20-letter alphabet, symmetric matrix (diagonal 4..11, off-diagonal
    # -4..2), -f0: every row spans the whole query (600-800 columns)
    rng = np.random.default_rng(1004)
    alpha = b"ACDEFGHIKLMNPQRSTVWYX"
    k = len(alpha)
    m = [0] * (k * k)
    for i in range(k - 1):
        for j in range(i, k - 1):
            v = int(rng.integers(4, 12)) if i == j else int(rng.integers(-4, 3))
            m[i * k + j] = m[j * k + i] = v
    m[k * k - 1] = 5
    params = Params(alphabet=alpha, matrix=m, f=0)
    fams = []
    for L in (640, 780):
        anc = rng.integers(0, 20, size=L)
        fam = []
        for _ in range(30):
            s = []
            for a in anc:
                u = rng.random()
                if u < 0.025:
                    continue  # deletion
                s.append(int(rng.integers(0, 20)) if rng.random() < 0.15 else int(a))
                if rng.random() < 0.025:
                    s.append(int(rng.integers(0, 20)))  # insertion
            fam.append(bytes(alpha[x] for x in s))
        fams.append(fam)
    for dp, wide in (("rows", None), ("rows", "0"), ("wave", None)):
        with _dp_rows(dp, wide):
            batch = mp.Batch(params, fams)
        st = batch.run(0)
        if dp == "rows" and wide == "0":
            assert st.rows_generic > 0, "no generic (wide) rows ran"
        elif dp == "rows":
            # -f0 selects the wide kernel form: rows of 600-800 columns in
            # striped segments, none on the generic row
            assert st.rows_g4 > 0 and st.rows_generic < st.rows_g4, (st.rows_g4, st.rows_generic)
        else:
            assert st.wave_reads > 0, "the row wavefront did not run"
        for f, reads in enumerate(fams):
            o = oracle.align_sequences(params, reads, kernel=oracle.AUTO_AVX2)
            assert batch.graph(f).dump() == o.dump(k)
            recs = [Sequence(name=f"read{i}", seq=x) for i, x in enumerate(reads)]
            assert batch.output(f, 1, recs) == o.msa(params, recs)
        del batch


def test_i64_reads_longer_than_shared_query_match_oracle(mp, oracle):
    # match 10,000: the score guard selects the i64 kernel; 6 kbp reads do not
    # fit the shared-memory query bytes, so the query is read from the arena
    params = Params.from_cli_scores(match=10000)
    reads = rc.synthetic_reads(np.random.default_rng(1005), 6000, 3, 0.01, 0.005, 0.005)
    o = oracle.align_sequences(params, reads)
    assert not o.i32_scores_safe(params, 0, 1, len(reads[-1]))
    g = mp.align_sequences(params, reads)
    assert g.dump() == o.dump(5)
    batch = mp.Batch(params, [reads])
    st = batch.run(0)
    assert st.rows_generic > 0
    assert batch.graph(0).dump() == o.dump(5)
