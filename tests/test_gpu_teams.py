"""Small batches (at most one read set per SM) run as teams: one 4-warp
block per set, the set on warp 0 and three helper warps on its DP rows. The
int32 rows are split by stripes, the int64 kernel's generic rows by quarters
of the band with the insertion state composed across them; graphs, ranks and
outputs must be the oracle's (src/align.rs:588-1162, src/lib.rs:177-204).
"""
import numpy as np
import pytest

import refcases as rc
from minipoa_b200.params import Params, Sequence

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mp():
    import minipoa_b200 as m

    m.default_context()
    return m


def test_small_int64_batch_runs_cooperative_generic_rows_like_the_oracle(mp, oracle):
    # match 30,000: the score guard selects the int64 kernel for these sizes
    params = Params.from_cli_scores(match=30000)
    rng = np.random.default_rng(1007)
    sets = [rc.synthetic_reads(rng, int(rng.integers(1500, 3200)), 4, 0.03, 0.01, 0.01) for _ in range(5)]
    probe = oracle.align_sequences(params, sets[0][:1])
    assert not probe.i32_scores_safe(params, 0, 1, len(sets[0][1]))
    batch = mp.Batch(params, sets)
    st = batch.run(0)
    assert st.slots == 4 * len(sets), "not a team launch"
    assert st.coop_jobs == len(sets), "a set ran without its helpers"
    assert st.rows_generic > 0
    for s, reads in enumerate(sets):
        assert batch.status(s) is None
        o = oracle.align_sequences(params, reads)
        assert batch.graph(s).dump() == o.dump(5), f"set {s}"
        recs = [Sequence(name=f"r{i}", seq=x) for i, x in enumerate(reads)]
        assert batch.output(s, 1, recs) == o.msa(params, recs)


@pytest.mark.parametrize("adaptive", [False, True])
def test_small_int32_batch_teams_match_the_oracle(mp, oracle, adaptive):
    params = Params(adaptive=adaptive)
    rng = np.random.default_rng(1008 + int(adaptive))
    sets = [rc.synthetic_reads(rng, int(rng.integers(400, 4200)), int(rng.integers(3, 9)), 0.06, 0.02, 0.02)
            for _ in range(12)]
    batch = mp.Batch(params, sets)
    st = batch.run(0)
    assert st.slots == 4 * len(sets)
    if not adaptive:
        assert st.coop_jobs > 0
    for s, reads in enumerate(sets):
        o = oracle.align_sequences(params, reads)
        assert batch.graph(s).dump() == o.dump(5), f"set {s}"
        assert batch.output(s, 0) == ">consensus sequence\n" + o.consensus(params)[0].decode() + "\n"


def test_empty_batch_and_tiny_sets(mp, oracle):
    # no sets at all: nothing runs, nothing is output
    empty = mp.Batch(Params(), [])
    st = empty.run(0)
    assert st.cells == 0
    assert empty.output_all(0) == b""
    del empty
    # one-read sets and an empty read (src/graph.rs: a path of the unknown
    # base only) as teams
    params = Params()
    sets = [[b"ACGTACGTTGCA"], [b""], [b"ACGT", b"ACGA", b""]]
    batch = mp.Batch(params, sets)
    batch.run(0)
    for s, reads in enumerate(sets):
        o = oracle.align_sequences(params, reads)
        assert batch.graph(s).dump() == o.dump(5), f"set {s}"
        assert batch.output(s, 0) == ">consensus sequence\n" + o.consensus(params)[0].decode() + "\n"
