"""GFA input on the GPU against the oracle, through the C ABI: the reference's
GFA known answers (tests/io_cli.rs), whole imported graphs, and graphs
extended with new reads after import (the -i workflow, lib.rs:214-231)."""
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


def test_gfa_known_answers(mp):
    p = Params()
    # tests/io_cli.rs:374-389
    g, recs = mp.read_gfa(p, "H\tVN:Z:1.0\nS\tone\tA\nS\ttwo\tCG\nL\tone\t+\ttwo\t+\t0M\nP\tread\tone+,two+\t*\n")
    assert recs[0].seq == b"ACG" and g.consensus(p)[0] == b"ACG"
    again, recs2 = mp.read_gfa(p, g.gfa(p, recs))
    assert again.consensus(p)[0] == b"ACG" and recs2[0].seq == b"ACG"
    # :391-399
    g, recs = mp.read_gfa(p, "S\ta\tAC\nS\tb\tGT\nL\ta\t+\tb\t+\t0M\n")
    assert recs == [] and g.consensus(p)[0] == b"ACGT"
    # :563-581 (-i graph.gfa -r1)
    out = mp.run(p.copy(result=1), [Sequence(name="new", seq=b"ACGT")], incremental="S\ta\tACGT\nP\told\ta+\t*\n")
    assert out == ">old \nACGT\n>new \nACGT\n"
    # :604-610
    with pytest.raises(mp.PoaError, match="revisits"):
        mp.read_gfa(p, "S\ta\tA\nP\tcycle\ta+,a+\t*\n")
    with pytest.raises(mp.PoaError, match="cycle"):
        mp.read_gfa(p, "S\ta\tA\nS\tb\tC\nL\ta\t+\tb\t+\t0M\nL\tb\t+\ta\t+\t0M\n")


@pytest.mark.parametrize("seed", [11, 12])
def test_imported_and_extended_graphs_match_oracle(mp, oracle, seed):
    # a graph of prior reads written as GFA, read back, then extended with new
    # reads: the whole graph (edges in order, weights, ranks, paths) and the
    # MSA / GFA bytes equal the oracle's
    p = Params()
    rng = np.random.default_rng(seed)
    reads = rc.synthetic_reads(rng, 400, 18, 0.04, 0.01, 0.01)
    prior, new = reads[:12], reads[12:]
    names = [Sequence(name=f"r{i}", seq=s) for i, s in enumerate(prior)]
    text = oracle.align_sequences(p, prior).gfa(p, names)
    g, recs = mp.read_gfa(p, text)
    o, orecs = oracle.read_gfa(p, text)
    assert [(r.name, r.seq) for r in recs] == orecs
    assert g.dump() == o.dump(5)
    allrecs = recs + [Sequence(name=f"n{i}", seq=s) for i, s in enumerate(new)]
    mp.extend_graph(p.copy(progressive=False), g, allrecs, len(recs))
    oracle.extend_graph(p, o, [r.seq for r in allrecs], len(orecs))
    assert g.dump() == o.dump(5)
    assert g.msa(p, allrecs) == o.msa(p, allrecs)
    assert g.gfa(p, allrecs) == o.gfa(p, allrecs)
