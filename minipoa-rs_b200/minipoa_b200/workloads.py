"""Seeded synthetic read sets in the shapes of the benchmark workloads.

No public dataset is named for these workloads, so inputs are generated: a
uniform-random ACGT ancestor and reads derived from it with i.i.d. per-base
substitution / deletion and insertion-after events (numpy PCG64 streams).
"""
from __future__ import annotations

from typing import List

import numpy as np

_ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


def mutate(rng: np.random.Generator, anc: np.ndarray, sub: float, ins: float, dele: float,
           indel_mean: float = 1.0) -> bytes:
    """One read from ancestor codes `anc` (0..3). Per ancestor base: deletion
    with probability `dele` (runs of geometric length when indel_mean > 1),
    else substitution with probability `sub` / (1 - dele); after a kept base an
    insertion with probability `ins` (geometric length when indel_mean > 1)."""
    L = anc.shape[0]
    if L == 0:
        return b""
    u = rng.random(L)
    dmask = u < dele
    if indel_mean > 1.0 and dmask.any():
        starts = np.flatnonzero(dmask)
        lens = rng.geometric(1.0 / indel_mean, size=starts.shape[0])
        cover = np.zeros(L + 1, dtype=np.int64)
        np.add.at(cover, starts, 1)
        np.add.at(cover, np.minimum(starts + lens, L), -1)
        dmask = np.cumsum(cover[:L]) > 0
    smask = (~dmask) & (u >= dele) & (u < dele + sub)
    base = anc.copy()
    ns = int(smask.sum())
    if ns:
        base[smask] = (anc[smask] + rng.integers(1, 4, size=ns)) % 4
    keep = ~dmask
    imask = keep & (rng.random(L) < ins)
    if indel_mean > 1.0:
        ilen = np.where(imask, rng.geometric(1.0 / indel_mean, size=L), 0)
    else:
        ilen = imask.astype(np.int64)
    per = keep.astype(np.int64) + ilen
    total = int(per.sum())
    out = np.empty(total, dtype=np.uint8)
    off = np.cumsum(per) - per
    out[off[keep]] = base[keep]
    if ilen.any():
        src = np.repeat(off + keep.astype(np.int64), ilen)
        rep = np.arange(int(ilen.sum())) - np.repeat(np.cumsum(ilen) - ilen, ilen)
        out[src + rep] = rng.integers(0, 4, size=src.shape[0])
    return _ACGT[out].tobytes()


def read_set(rng: np.random.Generator, ancestor_len: int, depth: int, sub: float, ins: float, dele: float,
             indel_mean: float = 1.0) -> List[bytes]:
    anc = rng.integers(0, 4, size=ancestor_len)
    return [mutate(rng, anc, sub, ins, dele, indel_mean) for _ in range(depth)]


def unseeded_consensus_set(seed: int = 1001) -> List[bytes]:
    """1,000 bp ancestor, 20 reads, 1% substitution, 0.5% single-base
    insertion, 0.5% single-base deletion."""
    return read_set(np.random.default_rng(seed), 1000, 20, 0.01, 0.005, 0.005)


def batched_sets(n_sets: int = 4096, seed: int = 1003, lmin: int = 200, lmax: int = 5000, dmin: int = 10,
                 dmax: int = 60, emin: float = 0.02, emax: float = 0.15) -> List[List[bytes]]:
    """Independent read sets: ancestor length log-uniform in [lmin, lmax],
    depth uniform in {dmin..dmax}, error rate uniform in [emin, emax] split
    60/20/20 among substitution / insertion / deletion."""
    rng = np.random.default_rng(seed)
    sets = []
    for _ in range(n_sets):
        L = int(np.exp(rng.uniform(np.log(lmin), np.log(lmax))))
        d = int(rng.integers(dmin, dmax + 1))
        e = float(rng.uniform(emin, emax))
        sets.append(read_set(rng, L, d, 0.6 * e, 0.2 * e, 0.2 * e))
    return sets


def seeded_window_set(seed: int = 1002) -> List[bytes]:
    """16,500 bp ancestor, 100 reads at ~5% error (3% substitution, 1%
    insertion, 1% deletion, indel lengths geometric with mean 1.5)."""
    return read_set(np.random.default_rng(seed), 16500, 100, 0.03, 0.01, 0.01, indel_mean=1.5)


PROTEIN_ALPHABET = b"ACDEFGHIKLMNPQRSTVWYX"


def protein_matrix(seed: int = 1004) -> List[int]:
    """Symmetric 20 x 20 integer matrix (diagonal uniform in 4..11,
    off-diagonal uniform in -4..2) plus a last (X) row and column of 0 with
    X-X = 5, in the layout of a matrix file over PROTEIN_ALPHABET."""
    rng = np.random.default_rng(seed)
    k = len(PROTEIN_ALPHABET)
    m = [0] * (k * k)
    for i in range(k - 1):
        for j in range(i, k - 1):
            v = int(rng.integers(4, 12)) if i == j else int(rng.integers(-4, 3))
            m[i * k + j] = m[j * k + i] = v
    m[k * k - 1] = 5
    return m


def protein_families(n_families: int = 1000, depth: int = 30, seed: int = 1004) -> List[List[bytes]]:
    """Protein families: a uniform random ancestor of length uniform in
    300..800 over 20 amino acids and `depth` members at 20% divergence (15%
    substitution, 2.5% deletion, 2.5% insertion per ancestor residue)."""
    rng = np.random.default_rng(seed + 1)
    fams = []
    for _ in range(n_families):
        L = int(rng.integers(300, 801))
        anc = rng.integers(0, 20, size=L)
        fam = []
        for _ in range(depth):
            u = rng.random(L)
            keep = u >= 0.025
            sub = (rng.random(L) < 0.15) & keep
            res = np.where(sub, rng.integers(0, 20, size=L), anc)[keep]
            ins = rng.random(res.shape[0]) < 0.025
            if ins.any():
                pos = np.flatnonzero(ins)
                res = np.insert(res, pos + 1, rng.integers(0, 20, size=pos.shape[0]))
            fam.append(bytes(PROTEIN_ALPHABET[int(x)] for x in res))
        fams.append(fam)
    return fams

