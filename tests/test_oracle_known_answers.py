"""Pins the CPU oracle to the reference's known answers.

Each test restates a minipoa-rs test that holds an exact expected output:
graph.rs:344-392, tests/regressions.rs:15-67 and the executable known answers
of tests/io_cli.rs (the workflow of lib.rs:207-242 without file I/O).
"""
import pytest

from minipoa_b200.params import Params, Sequence


def run_workflow(orc, params: Params, reads, result: int, kernel=0) -> str:
    """lib.rs:207-242 without the file reading: is_rna detection, the read
    loop, then the selected output."""
    params = params.copy(result=result)
    assert orc.validate(params) is None
    params.is_rna = len(params.alphabet) <= 5 and any(b"U" in r.seq.upper() for r in reads)
    g = orc.align_sequences(params, [r.seq for r in reads], kernel)
    if result == 0:
        return ">consensus sequence\n" + g.consensus(params)[0].decode() + "\n"
    if result == 1:
        return g.msa(params, reads)
    return g.gfa(params, reads)


def seqs(*items):
    return [Sequence(name=n, seq=s) for n, s in items]


@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_executable_consensus_msa_and_gfa_modes(oracle, kernel):
    # tests/io_cli.rs:422-451
    reads = seqs(("a", b"ACGT"), ("b", b"ACGT"))
    p = Params.from_cli_scores()
    assert run_workflow(oracle, p, reads, 0, kernel) == ">consensus sequence\nACGT\n"
    assert run_workflow(oracle, p, reads, 1, kernel) == ">a \nACGT\n>b \nACGT\n"
    gfa = run_workflow(oracle, p, reads, 2, kernel)
    assert gfa.startswith("H\tVN:Z:1.0\n")
    assert "P\ta\t1+,2+,3+,4+\t*" in gfa


def test_executable_reads_stdin_and_normalizes_rna(oracle):
    # tests/io_cli.rs:542-561
    out = run_workflow(oracle, Params.from_cli_scores(), seqs(("rna", b"acgu")), 0)
    assert out == ">consensus sequence\nACGU\n"


def test_executable_gzip_stdin_and_empty_record(oracle):
    # tests/io_cli.rs:612-630 (after decompression: ">a\nACGT\n>empty\n")
    out = run_workflow(oracle, Params.from_cli_scores(), seqs(("a", b"ACGT"), ("empty", b"")), 1)
    assert out == ">a \nACGT\n>empty \n----\n"


def test_weights_and_consensus_ties(oracle):
    # graph.rs:344-380
    p = Params()
    g = oracle.OracleGraph(p)
    g.add_path(p, 0, [(0, 4, None), (None, 0, None), (None, 1, None)])
    g.add_path(p, 1, [(0, 4, None), (2, 0, None), (None, 2, 3)])
    g.add_path(p, 2, [(0, 4, None), (2, 0, None), (4, 2, None)])
    g.toposort(False)
    seq, ids, cov = g.consensus(p)
    assert seq == b"AG"
    assert cov == [3, 2]
    d = g.dump(5)
    assert d["coverage"][2] == 3
    assert d["aligned"][3][2] == 4


def test_rejects_cycles(oracle):
    # graph.rs:381-392
    p = Params()
    g = oracle.OracleGraph(p)
    a = g.add_node(0)
    b = g.add_node(1)
    g.add_edge(0, a)
    g.add_edge(a, b)
    g.add_edge(b, a)
    g.add_edge(b, 1)
    with pytest.raises(oracle.OracleError, match="cycle"):
        g.toposort(False)


def test_rendering_msa_keeps_graph_ready_for_further_alignment(oracle):
    # tests/regressions.rs:15-32
    p = Params()
    reads = seqs(("r0", b"ACGT"), ("r1", b"ACCT"))
    g = oracle.align_sequences(p, [r.seq for r in reads])
    before = g.dump(5)
    assert "ACCT" in g.msa(p, reads)
    after = g.dump(5)
    assert after["rank"] == before["rank"]
    assert after["rank_of"] == before["rank_of"]
    path = g.align(p, b"ACGT")
    g.add_path(p, 2, path)
    g.toposort(False)
    assert g.consensus(p)[0] == b"ACGT"


def test_zero_gap_open_traceback_regression(oracle):
    # tests/regressions.rs:34-55
    p = Params.from_cli_scores(match=5, mismatch=-1, gap_open=0, gap_ext=-1, f=0)
    reads = seqs(("r0", b"GCANCCTTG"), ("r1", b"CTTCA"))
    g = oracle.align_sequences(p, [r.seq for r in reads])
    msa = g.msa(p, reads)
    rows = [s.replace("-", "") for s in msa.splitlines() if not s.startswith(">")]
    assert rows == ["GCANCCTTG", "CTTCA"]


def test_invalid_library_matrix_is_rejected_before_encoding(oracle):
    # tests/regressions.rs:57-67
    p = Params(alphabet=b"", matrix=[])
    err = oracle.validate(p)
    assert err is not None and "matrix" in err
    with pytest.raises(oracle.OracleError, match="matrix"):
        oracle.align_sequences(p, [b"ACGT", b"ACCT"])


def test_cli_score_normalization_and_matrix_rule():
    # tests/io_cli.rs:89-132 (score part) and cli.rs:166-199
    p = Params.from_cli_scores(match=3, mismatch=5, gap_open=7, gap_ext=1)
    assert (p.match_score, p.mismatch, p.gap_open, p.gap_ext) == (3, -5, -7, -1)
    assert p.score(0, 0) == 3
    assert p.score(0, 1) == -5
    assert p.score(4, 0) == 0
    assert p.score(4, 4) == 3


def test_encode_rules(oracle):
    # lib.rs:110-126: lowercase, U->T for <=5 letters, unknown -> N
    p = Params()
    for c in b"acgtnuACGTNU?*":
        assert oracle.lib().orc_encode(oracle._params(p)[0], c) == p.encode(c)
    assert p.encode(ord("U")) == p.encode(ord("T"))
    assert p.encode(ord("?")) == p.encode(ord("N"))
