"""Pins the oracle's GFA reader to the reference's GFA tests.

The reference's reader (io::read_gfa) lives in src/io.rs, which its source
tree does not contain; the oracle restates the behaviour the reference's
tests pin, and these tests restate those tests (tests/io_cli.rs) on it.
"""
import pytest

from minipoa_b200.params import Params, Sequence


def recs(records):
    return [Sequence(name=n, seq=s) for n, s in records]


def test_paths_include_single_base_segments_and_roundtrip(oracle):
    # tests/io_cli.rs:374-389
    text = "H\tVN:Z:1.0\nS\tone\tA\nS\ttwo\tCG\nL\tone\t+\ttwo\t+\t0M\nP\tread\tone+,two+\t*\n"
    p = Params()
    g, records = oracle.read_gfa(p, text)
    assert records[0][1] == b"ACG"
    d = g.dump(5)
    assert len(d["paths"][0][1]) == 3
    assert g.consensus(p)[0] == b"ACG"
    out = g.gfa(p, recs(records))
    again, seqs2 = oracle.read_gfa(p, out)
    assert again.consensus(p)[0] == b"ACG"
    assert seqs2[0][1] == b"ACG"


def test_links_without_paths_still_initialize_a_graph(oracle):
    # tests/io_cli.rs:391-399
    g, records = oracle.read_gfa(Params(), "S\ta\tAC\nS\tb\tGT\nL\ta\t+\tb\t+\t0M\n")
    assert records == []
    assert g.consensus(Params())[0] == b"ACGT"


@pytest.mark.parametrize("text", [
    "S\ta\tA\nS\ta\tC\n",
    "S\ta\tA\nP\tx\tb+\t*\n",
    "S\ta\tA\nP\tx\ta-\t*\n",
    "S\ta\tA\nL\ta\t+\ta\t+\t0M\n",
    "S\ta\tA\nS\tb\tC\nL\ta\t+\tb\t+\t0M\nL\tb\t+\ta\t+\t0M\n",
    "S\ta\tA\nL\ta\t+\ta\t-\t0M\n",
    "S\ta\tA\nL\ta\t+\ta\t+\t1M\n",
    "S\ta\t*\n",
])
def test_rejects_invalid_references_cycles_or_orientation(oracle, text):
    # tests/io_cli.rs:401-419
    with pytest.raises(oracle.OracleError):
        oracle.read_gfa(Params(), text)


def test_incremental_graph_alignment(oracle):
    # tests/io_cli.rs:563-581: -i graph.gfa -r1 with one new read; the
    # reference disables progressive ordering for incremental runs
    p = Params()
    g, records = oracle.read_gfa(p, "S\ta\tACGT\nP\told\ta+\t*\n")
    allrecs = recs(records) + [Sequence(name="new", seq=b"ACGT")]
    oracle.extend_graph(p, g, [r.seq for r in allrecs], len(records))
    assert g.msa(p, allrecs) == ">old \nACGT\n>new \nACGT\n"


@pytest.mark.parametrize("text", [
    "H\tVN:Z:1.0\nP\tempty\t*\t*\n",
    "H\tVN:Z:1.0\nS\ta\tAC\nP\tempty\t*\t*\nP\tnonempty\ta+\t*\n",
])
def test_empty_paths_export_and_reimport(oracle, text):
    # tests/io_cli.rs:583-602
    p = Params()
    g, records = oracle.read_gfa(p, text)
    assert records[0] == ("empty", b"")
    assert g.dump(5)["paths"][0][1] == []
    out = g.gfa(p, recs(records))
    assert "P\tempty\t*\t*\n" in out
    loaded, again = oracle.read_gfa(p, out)
    assert again == records
    assert loaded.consensus(p)[0] == g.consensus(p)[0]


def test_paths_revisiting_a_single_base_segment_fail(oracle):
    # tests/io_cli.rs:604-610
    with pytest.raises(oracle.OracleError, match="revisits"):
        oracle.read_gfa(Params(), "S\ta\tA\nP\tcycle\ta+,a+\t*\n")


def test_graph_written_by_gfa_reimports_with_the_same_consensus(oracle):
    # a POA graph of several reads, written with Graph::gfa and read back:
    # the same consensus and path sequences (column groups are not part of GFA)
    import numpy as np

    import refcases as rc

    p = Params()
    reads = rc.synthetic_reads(np.random.default_rng(5), 300, 8, 0.03, 0.01, 0.01)
    g = oracle.align_sequences(p, reads)
    seqs = [Sequence(name=f"r{i}", seq=s) for i, s in enumerate(reads)]
    back, records = oracle.read_gfa(p, g.gfa(p, seqs))
    assert [r[0] for r in records] == [s.name for s in seqs]
    assert [r[1] for r in records] == reads
    assert back.consensus(p)[0] == g.consensus(p)[0]
