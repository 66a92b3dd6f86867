"""Pins the CPU oracle's DP with the reference's own property tests.

Restates src/align.rs:1426-1871 and tests/avx512.rs:115-143 with the same case
streams (same LCG seeds), so the oracle is checked on exactly the reference's
cases: independent pairwise optimum, zero-gap / ambiguous scoring, band
behaviour, prefix-scan equivalence, i32 == i64 tracebacks on branched DAGs
and at band/lane edges, the score guard, and MSA/GFA workflow invariants.
"""
import pytest

import refcases as rc
from minipoa_b200.params import Params, Sequence

KERNELS = [0, 1, 2]  # serial i32 (auto), forced i64, AVX2 i32 (auto)


def linear(orc, params, reference: bytes):
    """align.rs:1352-1358"""
    g = orc.OracleGraph(params)
    g.add_path(params, 0, g.align(params, reference))
    g.toposort(False)
    return g


def path_score(params, g, path, reflen):
    d = g.dump(len(params.alphabet))
    return rc.alignment_score(params, d["rank_of"], d["base"], path, reflen)


@pytest.mark.parametrize("kernel", KERNELS)
def test_affine_alignment_matches_independent_pairwise_optimum(oracle, kernel):
    # align.rs:1426-1455
    params = Params(f=0)
    for ref, q in rc.pairwise_cases():
        g = linear(oracle, params, ref)
        path = g.align(params, q, kernel)
        assert len(path) == len(q) + 1
        assert path_score(params, g, path, len(ref)) == rc.pairwise_optimum(params, ref, q), (ref, q)


@pytest.mark.parametrize("kernel", KERNELS)
def test_affine_alignment_handles_zero_gaps_and_ambiguous_bases(oracle, kernel):
    # align.rs:1456-1492
    for params, cases in rc.zero_gap_cases():
        for ref, q in cases:
            g = linear(oracle, params, ref)
            path = g.align(params, q, kernel)
            assert len(path) == len(q) + 1
            assert path_score(params, g, path, len(ref)) == rc.pairwise_optimum(params, ref, q), (ref, q)


def test_static_and_adaptive_bands_preserve_simple_indels(oracle):
    # align.rs:1493-1524
    params = Params(b=2, f=40)
    reference = b"ACGTACGATAGCTACGATCGATGCTAGCTAGCTAGCATCGATCG"
    query = b"ACGTACGATAGCTACGATCGATTTTGCTAGCTAGCTAGCATCGATCG"
    g = linear(oracle, params, reference)
    full = params.copy(f=0)
    optimum = rc.pairwise_optimum(params, reference, query)
    for adaptive in (False, True):
        params.adaptive = adaptive
        path = g.align(params, query)
        assert len(path) == len(query) + 1
        assert path_score(params, g, path, len(reference)) == optimum
    assert path_score(params, g, g.align(full, query), len(reference)) == optimum


def test_avx2_prefix_scan_matches_serial_affine_transitions(oracle):
    # align.rs:1568-1601 (the 8-lane scan of the AVX2 CPU baseline)
    if not oracle.avx2_available():
        pytest.skip("no AVX2 on this host")
    for md, carry, opening, extension in rc.prefix_cases():
        assert oracle.avx2_prefix(md, carry, opening, extension) == rc.serial_prefix(md, carry, opening,
                                                                                      extension)


def _res(fn):
    try:
        return ("ok", fn())
    except Exception as e:  # the Result, errors included, must agree
        return ("err", str(e))


@pytest.mark.parametrize("fast_kernel", [3, 2])
def test_simd_matches_i64_traceback_on_branched_graphs_and_bands(oracle, fast_kernel):
    # align.rs:1603-1669 (560 i32 vs i64 comparisons)
    compared = 0
    for case, params, template, reads in rc.branched_cases():
        g = linear(oracle, params, template)
        for rid, query in enumerate(reads, start=1):
            for f, adaptive, band in rc.BRANCHED_BANDS:
                params.f = f
                params.adaptive = adaptive
                fast = _res(lambda: g.poa(params, 0, 1, query, adaptive, band, fast_kernel, retry=False))
                scalar = _res(lambda: g.poa(params, 0, 1, query, adaptive, band, 4, retry=False))
                assert fast == scalar, (case, rid, f, adaptive, band)
                compared += 1
            params.f = 0
            path = g.poa(params, 0, 1, query, False, 100, 4, retry=False)
            g.add_path(params, rid, path)
            g.toposort(False)
    assert compared == 560


def test_score_guard_dispatches_normal_work_to_simd_and_extreme_work_to_i64(oracle):
    # align.rs:1671-1692
    params = Params()
    g = linear(oracle, params, b"ACGTACGTACGT")
    assert g.i32_scores_safe(params, 0, 1, 12)
    extreme = params.copy(matrix=[2 ** 31 - 1] * 25)
    assert not g.i32_scores_safe(extreme, 0, 1, 12)
    auto = _res(lambda: g.poa(extreme, 0, 1, b"ACGTACCTACGT", False, 100, 0, retry=False))
    i64 = _res(lambda: g.poa(extreme, 0, 1, b"ACGTACCTACGT", False, 100, 4, retry=False))
    assert auto == i64


def test_simd_arena_rejects_reversed_anchors(oracle):
    # align.rs:1694-1706 (the error half; arena reuse is an internal detail)
    params = Params()
    g = linear(oracle, params, b"ACGTACGTACGTACGT")
    g.poa(params, 0, 1, b"ACGTACCTACGTACGT", False, 100, 3, retry=False)
    with pytest.raises(oracle.OracleError, match="topologically ordered"):
        g.poa(params, 1, 0, b"A", False, 100, 3, retry=False)


@pytest.mark.parametrize("fast_kernel", [3, 2])
def test_tracebacks_match_scalar_across_vector_and_band_edges(oracle, fast_kernel):
    # align.rs:1802-1871 (1080 cases: band widths 0/1/7/8/15 at lane edges)
    template = rc.edge_template()
    cases = 0
    for length in rc.EDGE_LENGTHS:
        params = rc.edge_params(length)
        reference = template[:length]
        g = linear(oracle, params, reference)
        alternate = rc.edge_alternate(reference)
        alt_path = g.poa(params, 0, 1, alternate, False, 100, 4, retry=False)
        g.add_path(params, 1, alt_path)
        g.toposort(False)
        for query in rc.edge_queries(reference, alternate):
            for f, adaptive, band in rc.EDGE_BANDS:
                params.f = f
                params.adaptive = adaptive
                fast = _res(lambda: g.poa(params, 0, 1, query, adaptive, band, fast_kernel, retry=False))
                scalar = _res(lambda: g.poa(params, 0, 1, query, adaptive, band, 4, retry=False))
                assert fast == scalar, (length, len(query), f, adaptive, band)
                cases += 1
    assert cases == 1080


@pytest.mark.parametrize("kernel", KERNELS)
def test_lane_boundary_workflows_preserve_every_read(oracle, kernel):
    # tests/avx512.rs:115-143
    for length in rc.LANE_LENGTHS:
        reads = rc.lane_reads(length)
        names = [f"read{i}" for i in range(len(reads))]
        recs = [Sequence(name=n, seq=s) for n, s in zip(names, reads)]
        for adaptive in (False, True):
            params = Params(b=1, f=40, adaptive=adaptive)
            g = oracle.align_sequences(params, reads, kernel)
            rc.validate_msa(g.msa(params, recs), names, reads)
            rc.validate_gfa(g.gfa(params, recs), names, reads)


def test_kernels_agree_on_synthetic_read_sets(oracle):
    """The three oracle kernels give identical graphs on seeded synthetic sets
    (static and adaptive bands), the property the GPU parity tests rely on."""
    import numpy as np

    rng = np.random.default_rng(4242)
    for adaptive in (False, True):
        params = Params(adaptive=adaptive)
        reads = rc.synthetic_reads(rng, 300, 8, 0.05, 0.02, 0.02)
        dumps = [oracle.align_sequences(params, reads, k).dump(5) for k in KERNELS]
        assert dumps[0] == dumps[1] == dumps[2]
