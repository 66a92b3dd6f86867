"""Seed windows (-S) on the host: the reference's own checks of
src/minimizer.rs (tests at src/minimizer.rs:580-785) against this library's
C ABI. Minimizer selection is the library's own (the reference takes it from
the simd-minimizers crate), so the checks that need that crate's exact
choice are replaced by properties every minimizer scheme has; the k-mer
values, run splitting, repeat filter, chaining and window partition are
checked as the reference checks them."""
import numpy as np

import minipoa_b200 as mp
from minipoa_b200 import Anchor, Minimizer
from minipoa_b200.params import Params


def random_dna(n):
    # the reference's xorshift generator (src/minimizer.rs:583-593)
    x = 42
    out = bytearray()
    for _ in range(n):
        x ^= (x << 13) & 0xFFFFFFFFFFFFFFFF
        x ^= x >> 7
        x ^= (x << 17) & 0xFFFFFFFFFFFFFFFF
        out.append(b"ACGT"[x & 3])
    return bytes(out)


def test_ambiguous_runs_do_not_create_spanning_seeds():
    seeds = mp.sketch(b"acgtACGTNNNNacguACGU", 4, 3)
    assert seeds
    assert all(s.end < 8 or s.end >= 15 for s in seeds)
    assert mp.sketch(b"acgu", 4, 10) == mp.sketch(b"ACGT", 4, 10)
    assert mp.sketch(b"NNNN", 3, 3) == []
    assert mp.sketch(b"AC", 3, 3) == []
    assert mp.sketch(b"ACGT", 0, 2) == []
    assert mp.sketch(b"ACGT", 3, 32768) == []


def test_exact_kmer_values_match():
    dna = random_dna(1024)
    dna = dna + dna
    code = {ord("A"): 0, ord("C"): 1, ord("T"): 2, ord("G"): 3}
    for k in (1, 3, 19, 31):
        seeds = mp.sketch(dna, k, 1)
        assert len(seeds) == len(dna) - k + 1
        seen = {}
        for s in seeds:
            kmer = dna[s.end + 1 - s.span: s.end + 1]
            exact = 0
            for i, b in enumerate(kmer):
                exact |= code[b] << (2 * i)
            assert s.value == exact
            assert seen.setdefault(s.value, kmer) == kmer


def test_sketch_covers_every_window_once():
    # properties of any minimizer scheme: one chosen k-mer per window of w
    # consecutive k-mers, positions increasing, each reported once
    dna = random_dna(4097)
    for k, w in ((5, 3), (19, 10), (31, 255)):
        seeds = mp.sketch(dna, k, w)
        starts = [s.end + 1 - k for s in seeds]
        assert starts == sorted(set(starts))
        nk = len(dna) - k + 1
        for i in range(0, nk - w + 1, 97):
            assert any(i <= p < i + w for p in starts)


def test_repeat_filter_removes_homopolymer_matches():
    p = Params(k=5, w=3, tr_dist=100)
    dna = b"A" * 100
    assert mp.collect_anchors(p, dna, dna) == []
    unfiltered = Params(k=5, w=3, tr_dist=0, max_occ=1)
    assert mp.collect_anchors(unfiltered, dna, dna) == []


def test_repeat_intervals_extend_clip_and_merge():
    mm = [Minimizer(1, 9, 5), Minimizer(1, 19, 5), Minimizer(2, 80, 5), Minimizer(2, 90, 5)]
    assert mp.repeat_intervals(mm, 100, 5) == []
    assert mp.repeat_intervals(mm, 100, 100) == [(0, 100)]


def test_chain_and_windows_are_monotone():
    dna = random_dna(5000)
    p = Params(k=19, w=10)
    anchors, tail = mp.anchor_windows(p, dna, dna)
    assert anchors and not tail
    assert all(a.target_end == a.query_end and not a.adaptive_before for a in anchors)
    for x, y in zip(anchors, anchors[1:]):
        assert x.target_end + y.span <= y.target_end


def test_windows_split_cumulative_drift():
    chain = [Anchor(t, q, 19) for t, q in ((100, 100), (200, 200), (300, 220), (400, 230), (600, 600))]
    windows, _ = mp.partition_windows(chain, 800, 800, 100, 500)
    assert any(a.adaptive_before for a in windows)
    for x, y in zip(windows, windows[1:]):
        assert y.target_end >= x.target_end + y.span
        assert y.query_end >= x.query_end + y.span


def test_no_local_chain_without_minimum_score():
    anchors = [Anchor(100 + i * 20, 100 + i * 20, 19) for i in range(3)]
    assert mp.chain(anchors, 19) == []


def test_protein_alphabet_has_no_anchors():
    # collect_anchors returns nothing for alphabets above 5 letters
    aa = b"ACDEFGHIKLMNPQRSTVWYN"
    m = [2 if i == j else -1 for i in range(len(aa)) for j in range(len(aa))]
    p = Params(alphabet=aa, matrix=m, k=5, w=3)
    assert mp.collect_anchors(p, aa * 20, aa * 20) == []
    dna = Params(k=5, w=3, tr_dist=0)
    assert mp.collect_anchors(dna, random_dna(300), random_dna(300))


def test_seeded_windows_of_a_mutated_read_are_ordered():
    rng = np.random.default_rng(1002)
    from minipoa_b200 import workloads

    reads = workloads.read_set(rng, 3000, 2, 0.03, 0.01, 0.01, indel_mean=1.5)
    p = Params(seeding=True)
    anchors, _ = mp.anchor_windows(p, reads[1], reads[0])
    assert anchors
    prev_t = prev_q = -1
    for a in anchors:
        assert a.target_end - a.span + 1 > prev_t and a.query_end - a.span + 1 > prev_q
        prev_t, prev_q = a.target_end, a.query_end


def _guide_order_restated(params, seqs):
    """src/minimizer.rs:505-578 over this library's sketches, in Python: the
    independent check of the similarity arithmetic and the greedy order."""
    n = len(seqs)
    if not params.progressive or n < 2 or len(params.alphabet) > 5:
        return list(range(n))
    groups = {}
    for rid, s in enumerate(seqs):
        for m in mp.sketch(s, params.k, params.w):
            counts = groups.setdefault(m.value, {})
            counts[rid] = counts.get(rid, 0) + 1
    if not groups:
        return list(range(n))
    total = [0] * n
    shared = [0] * (n * n)
    for value in sorted(groups):
        counts = groups[value]
        if len(counts) > n * params.mm_filter_ratio:
            continue
        keys = sorted(counts)
        for ia, a in enumerate(keys):
            total[a] += counts[a]
            for b in keys[:ia]:
                m = min(counts[a], counts[b])
                shared[a * n + b] += m
                shared[b * n + a] += m
    max_len = float(max(1, max(len(s) for s in seqs)))
    sim = [0.0] * (n * n)
    best = (-1.0, 0, 1)
    for i in range(n):
        for j in range(n):
            if i == j:
                continue
            common = shared[i * n + j]
            union = total[i] + total[j] - common
            jac = 0.0 if union == 0 else common / union * (0.51 * len(seqs[i]) / max_len + 0.49 * len(seqs[j]) / max_len)
            sim[i * n + j] = jac
            if jac > best[0]:
                best = (jac, i, j)
    order = [best[1], best[2]]
    used = [False] * n
    used[best[1]] = used[best[2]] = True
    sums = [sim[best[1] * n + v] + sim[best[2] * n + v] for v in range(n)]
    while len(order) < n:
        nxt = max((v for v in range(n) if not used[v]), key=lambda v: (sums[v], -v))
        order.append(nxt)
        used[nxt] = True
        for v in range(n):
            if not used[v]:
                sums[v] += sim[nxt * n + v]
    return order


def test_guide_order_is_permutation_and_deterministic():
    # src/minimizer.rs:746-772
    seqs = [random_dna(600 + i) for i in range(12)]
    p = Params(progressive=True)
    order = mp.guide_order(p, seqs)
    assert order == mp.guide_order(p, seqs)
    assert sorted(order) == list(range(len(seqs)))
    assert mp.guide_order(p, [b"ACGT"] * 3) == [0, 1, 2]
    assert mp.guide_order(Params(), seqs) == list(range(len(seqs)))  # not progressive


def test_guide_order_arithmetic_matches_a_restatement():
    rng = np.random.default_rng(505)
    from minipoa_b200 import workloads

    p = Params(progressive=True)
    for trial in range(4):
        anc = int(rng.integers(300, 900))
        reads = workloads.read_set(rng, anc, int(rng.integers(4, 14)), 0.03 * trial, 0.01 * trial, 0.01 * trial)
        # unrelated reads too, so that some pairs share nothing
        reads += [random_dna(200 + 37 * trial)[::-1]]
        assert mp.guide_order(p, reads) == _guide_order_restated(p, reads)
    prot = Params(progressive=True, alphabet=b"ACDEFGHIKLMNPQRSTVWYX",
                  matrix=[1 if i == j else 0 for i in range(21) for j in range(21)])
    assert mp.guide_order(prot, [b"ACD", b"CDE", b"DEF"]) == [0, 1, 2]  # protein: input order
