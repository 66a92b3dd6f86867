"""GPU parity: the CUDA path against the CPU oracle, through the C ABI.

Every comparison is exact (integer DP, byte outputs): alignment paths, error
messages, whole graphs (nodes, edges in insertion order, weights, ranks,
column groups, paths) and consensus / MSA / GFA bytes. Case streams are the
reference's own (same LCG seeds as src/align.rs and tests/avx512.rs), plus
seeded synthetic read sets at the configured workload shapes.
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


def tup(path):
    return [(a.node, a.base, a.aligned) if hasattr(a, "node") else tuple(a) for a in path]


def res(fn):
    try:
        return ("ok", tup(fn()))
    except Exception as e:
        return ("err", str(e))


def linear_pair(mp, oracle, params, reference):
    g = mp.align_sequences(params, [reference])
    o = oracle.align_sequences(params, [reference])
    return g, o


def test_known_answers_through_the_gpu(mp):
    # tests/io_cli.rs:422-451, 542-561, 612-630
    p = Params.from_cli_scores()
    reads = [Sequence(name="a", seq=b"ACGT"), Sequence(name="b", seq=b"ACGT")]
    assert mp.run(p.copy(result=0), reads) == ">consensus sequence\nACGT\n"
    assert mp.run(p.copy(result=1), reads) == ">a \nACGT\n>b \nACGT\n"
    gfa = mp.run(p.copy(result=2), reads)
    assert gfa.startswith("H\tVN:Z:1.0\n") and "P\ta\t1+,2+,3+,4+\t*" in gfa
    assert mp.run(p, [Sequence(name="rna", seq=b"acgu")]) == ">consensus sequence\nACGU\n"
    out = mp.run(p.copy(result=1), [Sequence(name="a", seq=b"ACGT"), Sequence(name="empty", seq=b"")])
    assert out == ">a \nACGT\n>empty \n----\n"


def test_weights_consensus_ties_and_cycles(mp):
    # graph.rs:344-392
    p = Params()
    g = mp.Graph(p)
    g.add_path(0, [(0, 4, None), (None, 0, None), (None, 1, None)])
    g.add_path(1, [(0, 4, None), (2, 0, None), (None, 2, 3)])
    g.add_path(2, [(0, 4, None), (2, 0, None), (4, 2, None)])
    g.toposort(False)
    seq, ids, cov = g.consensus(p)
    assert seq == b"AG" and cov == [3, 2]
    d = g.dump()
    assert d["coverage"][2] == 3 and d["aligned"][3][2] == 4
    g = mp.Graph(p)
    a = g.add_node(0)
    b = g.add_node(1)
    g.add_edge(0, a)
    g.add_edge(a, b)
    g.add_edge(b, a)
    g.add_edge(b, 1)
    with pytest.raises(mp.PoaError, match="cycle"):
        g.toposort(False)


def test_regressions(mp):
    # tests/regressions.rs:15-67
    p = Params()
    reads = [Sequence(name="r0", seq=b"ACGT"), Sequence(name="r1", seq=b"ACCT")]
    g = mp.align_sequences(p, reads)
    before = g.dump()
    assert "ACCT" in g.msa(p, reads)
    after = g.dump()
    assert after["rank"] == before["rank"] and after["rank_of"] == before["rank_of"]
    g.add_path(2, mp.align(p, g, b"ACGT"))
    g.toposort(False)
    assert g.consensus(p)[0] == b"ACGT"
    p2 = Params.from_cli_scores(match=5, mismatch=-1, gap_open=0, gap_ext=-1, f=0)
    reads2 = [Sequence(name="r0", seq=b"GCANCCTTG"), Sequence(name="r1", seq=b"CTTCA")]
    msa = mp.align_sequences(p2, reads2).msa(p2, reads2)
    assert [s.replace("-", "") for s in msa.splitlines() if not s.startswith(">")] == ["GCANCCTTG", "CTTCA"]
    with pytest.raises(mp.PoaError, match="matrix"):
        mp.align_sequences(Params(alphabet=b"", matrix=[]), reads)


@pytest.mark.parametrize("which", ["pairwise", "zero_gap"])
def test_paths_match_oracle_on_reference_case_streams(mp, oracle, which):
    # align.rs:1426-1492 case streams; the GPU path must equal the oracle's
    if which == "pairwise":
        groups = [(Params(f=0), rc.pairwise_cases())]
    else:
        groups = rc.zero_gap_cases()
    for params, cases in groups:
        for ref, q in cases:
            g, o = linear_pair(mp, oracle, params, ref)
            assert tup(mp.align(params, g, q)) == tup(o.align(params, q)), (ref, q)


def test_branched_graphs_i32_and_i64_match_oracle(mp, oracle):
    # align.rs:1603-1669: both GPU kernels against both oracle kernels
    n = 0
    for case, params, template, reads in rc.branched_cases():
        g, o = linear_pair(mp, oracle, params, template)
        for rid, query in enumerate(reads, start=1):
            for f, adaptive, band in rc.BRANCHED_BANDS:
                params.f = f
                params.adaptive = adaptive
                want32 = res(lambda: o.poa(params, 0, 1, query, adaptive, band, 3, retry=False))
                want64 = res(lambda: o.poa(params, 0, 1, query, adaptive, band, 4, retry=False))
                got32 = res(lambda: mp.poa(params, g, 0, 1, query, adaptive, band, kernel=1, retry=False))
                got64 = res(lambda: mp.poa(params, g, 0, 1, query, adaptive, band, kernel=2, retry=False))
                assert got32 == want32 and got64 == want64, (case, rid, f, adaptive, band)
                n += 1
            params.f = 0
            path = o.poa(params, 0, 1, query, False, 100, 4, retry=False)
            assert tup(mp.poa(params, g, 0, 1, query, False, 100, kernel=2, retry=False)) == tup(path)
            o.add_path(params, rid, path)
            o.toposort(False)
            g.add_path(rid, path)
            g.toposort(False)
        assert g.dump() == o.dump(5)
    assert n == 560


def test_band_and_lane_edges_match_oracle(mp, oracle):
    # align.rs:1802-1871 (1080 cases, both kernels)
    template = rc.edge_template()
    cases = 0
    for length in rc.EDGE_LENGTHS:
        params = rc.edge_params(length)
        reference = template[:length]
        g, o = linear_pair(mp, oracle, params, reference)
        alternate = rc.edge_alternate(reference)
        alt = o.poa(params, 0, 1, alternate, False, 100, 4, retry=False)
        o.add_path(params, 1, alt)
        o.toposort(False)
        g.add_path(1, alt)
        g.toposort(False)
        for query in rc.edge_queries(reference, alternate):
            for f, adaptive, band in rc.EDGE_BANDS:
                params.f = f
                params.adaptive = adaptive
                for gk, ok in ((1, 3), (2, 4)):
                    got = res(lambda: mp.poa(params, g, 0, 1, query, adaptive, band, kernel=gk, retry=False))
                    want = res(lambda: o.poa(params, 0, 1, query, adaptive, band, ok, retry=False))
                    assert got == want, (length, len(query), f, adaptive, band, gk)
                cases += 1
    assert cases == 1080


def test_retry_and_score_guard_match_oracle(mp, oracle):
    # poa's full-DP retry (align.rs:192-211) and the guard (align.rs:1671-1692)
    params = Params()
    g, o = linear_pair(mp, oracle, params, b"ACGTACGTACGT")
    extreme = params.copy(matrix=[2 ** 31 - 1] * 25)
    got = res(lambda: mp.poa(extreme, g, 0, 1, b"ACGTACCTACGT", False, 100, kernel=0, retry=False))
    want = res(lambda: o.poa(extreme, 0, 1, b"ACGTACCTACGT", False, 100, 4, retry=False))
    assert got == want
    with pytest.raises(mp.PoaError, match="topologically ordered"):
        mp.poa(params, g, 1, 0, b"A", False, 100, kernel=1, retry=False)
    # a band of 0 forces the retry on an indel-heavy read
    tight = Params(b=0, f=1000)
    g, o = linear_pair(mp, oracle, tight, b"ACGTACGTTTTTTTTTTACGTACGTACGGGGGGGGGGGGT")
    q = b"ACGTACGTACGTACGTACGGGGGGGGGGGGGGGGGGGGGGGT"
    assert res(lambda: mp.align(tight, g, q)) == res(lambda: o.align(tight, q))


@pytest.mark.parametrize("adaptive", [False, True])
def test_lane_boundary_workflows_match_oracle_bytes(mp, oracle, adaptive):
    # tests/avx512.rs:115-143, compared byte for byte with the oracle
    for length in rc.LANE_LENGTHS:
        reads = rc.lane_reads(length)
        recs = [Sequence(name=f"read{i}", seq=s) for i, s in enumerate(reads)]
        params = Params(b=1, f=40, adaptive=adaptive)
        g = mp.align_sequences(params, reads)
        o = oracle.align_sequences(params, reads)
        assert g.dump() == o.dump(5)
        assert g.msa(params, recs) == o.msa(params, recs)
        assert g.gfa(params, recs) == o.gfa(params, recs)
        assert g.consensus(params) == o.consensus(params)
        rc.validate_msa(g.msa(params, recs), [r.name for r in recs], reads)


@pytest.mark.parametrize("adaptive", [False, True])
def test_unseeded_workload_matches_oracle(mp, oracle, adaptive):
    # 1,000 bp ancestor, 20 reads, 1% sub / 0.5% ins / 0.5% del (seed 1001)
    rng = np.random.default_rng(1001)
    reads = rc.synthetic_reads(rng, 1000, 20, 0.01, 0.005, 0.005)
    recs = [Sequence(name=f"read{i}", seq=s) for i, s in enumerate(reads)]
    params = Params(adaptive=adaptive)
    g = mp.align_sequences(params, reads)
    o = oracle.align_sequences(params, reads)
    assert g.dump() == o.dump(5)
    for r in (0, 1, 2):
        assert mp.run(params.copy(result=r), recs) == _oracle_run(oracle, params.copy(result=r), recs)


def _oracle_run(oracle, params, recs):
    g = oracle.align_sequences(params, [r.seq for r in recs])
    if params.result == 0:
        return ">consensus sequence\n" + g.consensus(params)[0].decode() + "\n"
    return g.msa(params, recs) if params.result == 1 else g.gfa(params, recs)


def test_protein_matrix_and_i64_workloads_match_oracle(mp, oracle):
    # 20-letter alphabet with a symmetric integer matrix, full DP (-f0); and a
    # DNA set with match 1000 so the score guard selects the i64 kernel
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
    anc = rng.integers(0, 20, size=120)
    reads = []
    for _ in range(6):
        s = [int(a) if rng.random() > 0.15 else int(rng.integers(0, 20)) for a in anc if rng.random() > 0.03]
        reads.append(bytes(alpha[x] for x in s))
    g = mp.align_sequences(params, reads)
    o = oracle.align_sequences(params, reads)
    assert g.dump() == o.dump(k)
    big = Params.from_cli_scores(match=100000, mismatch=-100000, gap_open=-100000, gap_ext=-50000)
    reads = rc.synthetic_reads(np.random.default_rng(1005), 1000, 4, 0.01, 0.005, 0.005)
    ob = oracle.align_sequences(big, reads)
    gb = mp.align_sequences(big, reads)
    assert not ob.i32_scores_safe(big, 0, 1, 1000)
    assert gb.dump() == ob.dump(5)


def _batch_sets(seed, n_sets, lmin, lmax, dmin, dmax):
    rng = np.random.default_rng(seed)
    sets = []
    for _ in range(n_sets):
        L = int(np.exp(rng.uniform(np.log(lmin), np.log(lmax))))
        d = int(rng.integers(dmin, dmax + 1))
        e = rng.uniform(0.02, 0.15)
        sets.append(rc.synthetic_reads(rng, L, d, 0.6 * e, 0.2 * e, 0.2 * e))
    return sets


@pytest.mark.parametrize("adaptive", [False, True])
def test_batched_and_plain_runs_match_oracle(mp, oracle, adaptive):
    # independent read sets of uneven sizes in one persistent launch
    params = Params(adaptive=adaptive)
    sets = _batch_sets(1003, 24, 60, 600, 3, 8)
    batch = mp.Batch(params, sets)
    st = batch.run(0)
    assert st.cells > 0 and st.reads == sum(len(s) for s in sets)
    outs = {}
    for s, reads in enumerate(sets):
        assert batch.status(s) is None
        o = oracle.align_sequences(params, reads)
        recs = [Sequence(name=f"read{i}", seq=x) for i, x in enumerate(reads)]
        assert batch.graph(s).dump() == o.dump(5)
        outs[s] = [batch.output(s, r, recs) for r in (0, 1, 2)]
        assert outs[s][0] == ">consensus sequence\n" + o.consensus(params)[0].decode() + "\n"
        assert outs[s][1] == o.msa(params, recs)
        assert outs[s][2] == o.gfa(params, recs)
    # a second run resets the graphs and reproduces the same bytes
    st2 = batch.run(0)
    assert st2.cells == st.cells
    # the plain form (one launch per read) gives the same graphs
    st3 = batch.run(1)
    assert st3.cells == st.cells and st3.launches > st.launches
    for s in range(len(sets)):
        assert [batch.output(s, r) for r in (0, 2)] == [outs[s][0], outs[s][2]]
    allc = batch.output_all(0).decode()
    assert allc == "".join(outs[s][0] for s in range(len(sets)))


def test_batch_arena_overflow_parks_and_finishes(mp, oracle):
    # a tiny per-slot arena forces jobs to park and resume in later passes
    params = Params()
    sets = _batch_sets(77, 12, 200, 800, 3, 6)
    batch = mp.Batch(params, sets)
    batch.tune(warps_per_sm=16, arena_bytes_per_slot=1 << 20)
    st = batch.run(0)
    assert st.relaunches >= 1
    for s, reads in enumerate(sets):
        assert batch.graph(s).dump() == oracle.align_sequences(params, reads).dump(5)


def test_deep_high_error_sets_match_oracle(mp, oracle):
    # many reads at high error: the path often reaches existing column
    # siblings out of rank order, so the device repairs its rank order between
    # reads; the finished graphs, ranks included, must be the oracle's
    params = Params()
    rng = np.random.default_rng(4242)
    sets = [rc.synthetic_reads(rng, int(rng.integers(300, 700)), int(rng.integers(25, 40)), 0.09, 0.03, 0.03)
            for _ in range(6)]
    batch = mp.Batch(params, sets)
    batch.run(0)
    for s, reads in enumerate(sets):
        assert batch.status(s) is None
        o = oracle.align_sequences(params, reads, kernel=oracle.AUTO_AVX2)
        assert batch.graph(s).dump() == o.dump(5)
