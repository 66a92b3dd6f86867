"""Seeded alignment (-S, src/align.rs:99-164) on the GPU against the oracle.

The seed windows come from one host function (the library's
poa_seed_anchor_windows, restating src/minimizer.rs) and are a shared input:
the oracle side recomputes them from its own graph's consensus with that
function, aligns each window with the oracle's poa (src/align.rs:192-211)
and adds the anchor nodes, exactly as align::align does; the GPU side runs
the same read loop through poa_align_sequences with params.seeding set.
Graphs (ranks included), consensus, MSA and GFA must be identical.
"""
import numpy as np
import pytest

from minipoa_b200.params import Params, Sequence

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mp():
    import minipoa_b200 as m

    m.default_context()
    return m


def seeded_path(mp, og, params, q):
    cons, ids, _ = og.consensus(params)
    anchors, tail = mp.anchor_windows(params, q, cons)
    whole = lambda: og.poa(params, 0, 1, q, True, params.b)  # noqa: E731
    if not anchors:
        return whole()
    windows, beg, qbeg, prev = [], 0, 0, None
    for a in anchors:
        ts, qs = a.target_end + 1 - a.span, a.query_end + 1 - a.span
        valid = (a.span > 0 and a.target_end < len(ids) and a.query_end < len(q) and qs >= qbeg
                 and (prev is None or ts > prev)
                 and all(params.encode(cons[ts + o]) == params.encode(q[qs + o]) for o in range(a.span)))
        if not valid:
            return whole()
        windows.append((beg, ids[ts], qbeg, qs, a.adaptive_before, ids[ts:a.target_end]))
        beg, qbeg, prev = ids[a.target_end], a.query_end + 1, a.target_end
    windows.append((beg, 1, qbeg, len(q), tail, []))
    base = og.dump(len(params.alphabet))["base"]
    out = []
    for b, e, qb, qe, ad, anchor in windows:
        out += og.poa(params, b, e, q[qb:qe], ad, params.b if ad else params.win_band)
        out += [(i, base[i], None) for i in anchor]
    return out


def oracle_seeded(mp, oracle, params, reads):
    og = oracle.OracleGraph(params)
    for r, q in enumerate(reads):
        if og.n_nodes() <= 2:
            items = [(0, params.encode("N"), None)] + [(None, params.encode(c), None) for c in q]
        else:
            items = seeded_path(mp, og, params, q)
        og.add_path(params, r, items)
        og.toposort()
    return og


@pytest.mark.parametrize("adaptive", [False, True])
def test_seeded_read_loop_matches_oracle_on_shared_windows(mp, oracle, adaptive):
    from minipoa_b200 import workloads

    rng = np.random.default_rng(1002)
    reads = workloads.read_set(rng, 2500, 6, 0.03, 0.01, 0.01, indel_mean=1.5)
    params = Params(seeding=True, adaptive=adaptive, result=1)
    g = mp.align_sequences(params, reads)
    o = oracle_seeded(mp, oracle, params, reads)
    assert g.dump() == o.dump(5)
    recs = [Sequence(name=f"read{i}", seq=x) for i, x in enumerate(reads)]
    assert g.msa(params, recs) == o.msa(params, recs)
    assert g.gfa(params, recs) == o.gfa(params, recs)
    # the windows were used: a read aligned through anchors, not the fallback
    cons, _, _ = o.consensus(params)
    assert mp.anchor_windows(params, reads[-1], cons)[0]


def test_seeded_align_of_one_query_matches_oracle(mp, oracle):
    from minipoa_b200 import workloads

    rng = np.random.default_rng(7)
    reads = workloads.read_set(rng, 1800, 4, 0.02, 0.01, 0.01)
    params = Params(seeding=True)
    g = mp.align_sequences(params, reads[:3])
    o = oracle_seeded(mp, oracle, params, reads[:3])
    got = [(a.node, a.base, a.aligned) for a in mp.align(params, g, reads[3])]
    assert got == seeded_path(mp, o, params, reads[3])
    # a query with no usable seeds takes the whole graph with an adaptive band
    short = reads[3][:30]
    got = [(a.node, a.base, a.aligned) for a in mp.align(params, g, short)]
    assert got == seeded_path(mp, o, params, short)


def test_windows_in_one_launch_equal_one_launch_per_window(mp):
    from minipoa_b200 import workloads

    rng = np.random.default_rng(11)
    reads = workloads.read_set(rng, 4000, 5, 0.03, 0.01, 0.01, indel_mean=1.5)
    params = Params(seeding=True, adaptive=True)
    ctx = mp.default_context()
    w0 = ctx.window_stats()
    ctx.tune_windows(False)
    batched = mp.align_sequences(params, reads).dump()
    w1 = ctx.window_stats()
    ctx.tune_windows(True)
    try:
        plain = mp.align_sequences(params, reads).dump()
    finally:
        ctx.tune_windows(False)
    w2 = ctx.window_stats()
    assert batched == plain
    # same windows both ways; far fewer launches in the batched form
    assert w1[0] - w0[0] == w2[0] - w1[0] > 4
    assert w1[1] - w0[1] < w2[1] - w1[1]
