"""Progressive guide order (-p, src/lib.rs:190-194, src/minimizer.rs:505-578)
on the GPU paths, against the oracle. The order comes from minimizer
sketches, which are this library's own, so it is a shared input: the oracle
adds the reads in the order the library computes (mp.guide_order) and the
graphs (paths keep each read's own index), MSA and GFA bytes must match."""
import numpy as np
import pytest

from minipoa_b200 import workloads
from minipoa_b200.params import Params, Sequence

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mp():
    import minipoa_b200 as m

    m.default_context()
    return m


def _sets(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(rng.integers(150, 900))
        e = float(rng.uniform(0.02, 0.12))
        reads = workloads.read_set(rng, L, int(rng.integers(4, 12)), 0.6 * e, 0.2 * e, 0.2 * e)
        # reads in a shuffled order, so the guide order is not the input order
        perm = rng.permutation(len(reads))
        out.append([reads[int(k)] for k in perm])
    return out


def _check(mp, oracle, params, reads, graph_dump, msa, gfa):
    order = mp.guide_order(params, reads)
    o = oracle.align_sequences_in_order(params, reads, order)
    recs = [Sequence(name=f"read{i}", seq=x) for i, x in enumerate(reads)]
    assert graph_dump == o.dump(5)
    assert msa(recs) == o.msa(params, recs)
    assert gfa(recs) == o.gfa(params, recs)
    return order


def test_single_graph_progressive_matches_oracle(mp, oracle):
    params = Params(progressive=True)
    moved = 0
    for reads in _sets(190, 6):
        g = mp.align_sequences(params, reads)
        order = _check(mp, oracle, params, reads, g.dump(), lambda r: g.msa(params, r), lambda r: g.gfa(params, r))
        moved += order != list(range(len(reads)))
    assert moved > 0, "every guide order was the input order"


def test_batched_and_served_progressive_match_oracle(mp, oracle):
    params = Params(progressive=True)
    sets = _sets(578, 24)
    batch = mp.Batch(params, sets)
    batch.run(0)
    server = mp.Server(params)
    ids = [server.submit(r) for r in sets]
    for s, reads in enumerate(sets):
        _check(mp, oracle, params, reads, batch.graph(s).dump(), lambda r: batch.output(s, 1, r),
               lambda r: batch.output(s, 2, r))
        assert server.wait(ids[s]) == mp._lib.POA_SERVER_DONE
        assert server.output(ids[s], 2) == batch.output(s, 2)
    server.close()
