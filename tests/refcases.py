"""Case generators and checkers restated from the reference's own tests.

Each helper cites the minipoa-rs test it restates. The LCG streams use the
same multipliers, increments and seeds, so the generated cases are the
reference's own cases.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

from minipoa_b200.params import Params

MASK64 = (1 << 64) - 1
NEG = -(1 << 50)
NEG32 = -(1 << 29)
MATCH, DELETE, INSERT = 1, 2, 4


def lcg(seed: int, inc: int = 1) -> Callable[[], int]:
    """rng = rng * 6364136223846793005 + inc (wrapping); returns rng >> 32."""
    state = [seed]

    def nxt() -> int:
        state[0] = (state[0] * 6364136223846793005 + inc) & MASK64
        return state[0] >> 32

    return nxt


def lcg_i31(seed: int) -> Callable[[], int]:
    """align.rs:1570-1574: ((state >> 32) as i32) & 0x7fffffff."""
    r = lcg(seed)

    def nxt() -> int:
        v = r() & 0xFFFFFFFF
        return v & 0x7FFFFFFF

    return nxt


def pairwise_optimum(params: Params, reference: bytes, query: bytes) -> int:
    """align.rs:1359-1390: independent global affine optimum."""
    width = len(query) + 1
    size = (len(reference) + 1) * width
    best = [NEG] * size
    deletion = [NEG] * size
    insertion = [NEG] * size
    best[0] = 0
    e = params.gap_ext
    o = params.gap_open + e
    for i in range(len(reference) + 1):
        for j in range(len(query) + 1):
            pos = i * width + j
            if i > 0:
                deletion[pos] = max(best[pos - width] + o, deletion[pos - width] + e)
            if j > 0:
                insertion[pos] = max(best[pos - 1] + o, insertion[pos - 1] + e)
            if i > 0 and j > 0:
                diagonal = best[pos - width - 1] + params.score(params.encode(reference[i - 1]),
                                                                params.encode(query[j - 1]))
            else:
                diagonal = best[pos]
            best[pos] = max(diagonal, deletion[pos], insertion[pos])
    return best[-1]


def alignment_score(params: Params, node_rank: List[int], node_base: List[int], path, reference_len: int) -> int:
    """align.rs:1391-1425: score of a returned path over a linear graph."""
    score = 0
    previous = 0
    last = [0]

    def add_gap(op):
        nonlocal score
        score += params.gap_ext
        if last[0] != op:
            score += params.gap_open
        last[0] = op

    for node, base, aligned in path[1:]:
        target = node if node is not None else aligned
        if target is not None:
            rank = node_rank[target]
            for _ in range(previous + 1, rank):
                add_gap(DELETE)
            score += params.score(node_base[target], base)
            last[0] = MATCH
            previous = rank
        else:
            add_gap(INSERT)
    for _ in range(previous, reference_len):
        add_gap(DELETE)
    return score


def pairwise_cases() -> List[Tuple[bytes, bytes]]:
    """align.rs:1427-1444: 500 cases, seed 1923827, increment 1442695040888963407."""
    random = lcg(1923827, 1442695040888963407)
    out = []
    for _ in range(500):
        n = 1 + random() % 22
        ref = bytes(b"ACGT"[random() % 4] for _ in range(n))
        n = random() % 23
        q = bytes(b"ACGT"[random() % 4] for _ in range(n))
        out.append((ref, q))
    return out


ZERO_GAP_SCORINGS = [(2, -4, -4, -2), (5, -1, 0, -1), (0, -2, -2, 0), (3, 0, 0, 0)]


def zero_gap_cases():
    """align.rs:1457-1486: 4 scoring sets x 150 cases, seed 912873."""
    random = lcg(912873)
    out = []
    for matching, mismatch, opening, extension in ZERO_GAP_SCORINGS:
        params = Params(f=0, gap_open=opening, gap_ext=extension)
        for a in range(4):
            for b in range(4):
                params.matrix[a * 5 + b] = matching if a == b else mismatch
        params.matrix[24] = matching
        cases = []
        for _ in range(150):
            n = 1 + random() % 20
            ref = bytes(b"ACGTN"[random() % 5] for _ in range(n))
            n = random() % 21
            q = bytes(b"ACGTN"[random() % 5] for _ in range(n))
            cases.append((ref, q))
        out.append((params, cases))
    return out


def prefix_cases():
    """align.rs:1569-1588: 5 gap sets x 500 eight-lane scans, seed 8917321."""
    random = lcg_i31(8917321)
    out = []
    for opening, extension in [(0, 0), (0, -2), (-4, 0), (-6, -2), (-117, -12)]:
        for case in range(500):
            md = []
            for _ in range(8):
                md.append(NEG32 if random() % 11 == 0 else random() % 201 - 100)
            carry = NEG32 if case % 9 == 0 else random() % 201 - 100
            out.append((md, carry, opening, extension))
    return out


def serial_prefix(md, carry, opening, extension):
    value = carry
    out = []
    for x in md:
        value = max(value + extension, x + opening)
        out.append(value)
    return out


def branched_cases():
    """align.rs:1604-1647: 35 templates x 4 reads (seed 7512129). Yields
    (case, params-before-bands, template, reads)."""
    random = lcg(7512129)
    out = []
    for case in range(35):
        params = Params()
        if case % 4 == 1:
            params.gap_open, params.gap_ext = 0, -1
        elif case % 4 == 2:
            params.gap_ext = 0
        elif case % 4 == 3:
            params.gap_open, params.gap_ext = 0, 0
        if case % 5 == 0:
            params.matrix[24] = 0
        n = 40 + random() % 80
        template = bytes(b"ACGTN"[random() % 5] for _ in range(n))
        reads = []
        for rid in range(1, 5):
            q = bytearray()
            for base in template:
                if random() % 20 == 0:
                    continue
                if random() % 12 == 0:
                    q.append(b"ACGTN"[random() % 5])
                else:
                    q.append(base)
                if random() % 20 == 0:
                    q.append(b"ACGT"[random() % 4])
            reads.append(bytes(q))
        out.append((case, params, template, reads))
    return out


BRANCHED_BANDS = [(0, False, 0), (40, False, 2), (40, True, 3), (40, False, 100)]

EDGE_LENGTHS = [1, 6, 7, 8, 9, 14, 15, 16, 17, 22, 23, 24, 25, 30, 31, 32, 33, 47, 48, 49, 63, 64, 65, 79, 80, 81,
                95]
EDGE_BANDS = [(0, False, 0), (40, False, 0), (40, False, 1), (40, False, 7), (40, False, 8), (40, False, 15),
              (40, True, 1), (40, True, 8)]


def edge_template() -> bytes:
    """align.rs:1805-1811: 95 bases, seed 1923801."""
    random = lcg(1923801)
    return bytes(b"ACGTN"[random() % 5] for _ in range(95))


def edge_queries(reference: bytes, alternate: bytes):
    """align.rs:1834-1847."""
    n = len(reference)
    insertion = reference[: n // 2] + b"ACGTACGTA" + reference[n // 2:]
    deletion = bytes(b for i, b in enumerate(reference) if i % 13 != 7)
    return [b"", reference, alternate, insertion, deletion]


def edge_params(length: int) -> Params:
    p = Params()
    if length % 3 == 0:
        p.gap_open = 0
    if length % 5 == 0:
        p.gap_ext = 0
    return p


def edge_alternate(reference: bytes) -> bytes:
    alt = bytearray(reference)
    if len(reference) > 8:
        alt[7] = ord("C") if alt[7] == ord("A") else ord("A")
    return bytes(alt)


LANE_LENGTHS = [1, 7, 8, 9, 15, 16, 17, 23, 24, 25, 31, 32, 33, 47, 48, 49, 63, 64, 65, 79]


def lane_dna(length: int) -> bytes:
    """tests/avx512.rs:5-13."""
    random = lcg(0x5A71B301)
    return bytes(b"ACGT"[random() % 4] for _ in range(length))


def lane_reads(length: int) -> List[bytes]:
    """tests/avx512.rs:117-130."""
    reference = lane_dna(length)
    split = length // 2
    insertion = reference[:split] + b"TGCATGCA" + reference[split:]
    deletion = bytes(b for i, b in enumerate(reference) if i % 5 != 2)
    return [reference, insertion, deletion, b""]


def validate_msa(output: str, names: List[str], seqs: List[bytes]):
    """tests/avx512.rs:27-53."""
    rows = {}
    lines = output.splitlines()
    it = iter(lines)
    for header in it:
        assert header.startswith(">")
        name = header[1:].split()[0]
        rows[name] = next(it)
    assert len(rows) == len(names)
    assert len({len(r) for r in rows.values()}) <= 1
    for name, seq in zip(names, seqs):
        assert rows[name].replace("-", "").encode() == seq


def validate_gfa(output: str, names: List[str], seqs: List[bytes]):
    """tests/avx512.rs:55-91."""
    nodes, links, paths = {}, set(), {}
    for line in output.splitlines():
        fields = line.split("\t")
        if fields[0] == "S":
            nodes[fields[1]] = fields[2]
        elif fields[0] == "L":
            links.add((fields[1], fields[3]))
        elif fields[0] == "P":
            paths[fields[1]] = [] if fields[2] == "*" else [x[:-1] for x in fields[2].split(",")]
    assert len(paths) == len(names)
    for name, seq in zip(names, seqs):
        path = paths[name]
        assert "".join(nodes[i] for i in path).encode() == seq
        assert all((a, b) in links for a, b in zip(path, path[1:]))


def synthetic_reads(rng, ancestor_len: int, depth: int, sub: float, ins: float, dele: float,
                    indel_mean: float = 1.0) -> List[bytes]:
    """Seeded synthetic read set: a uniform ACGT ancestor and `depth` reads with
    i.i.d. per-base substitution / insertion / deletion (indel lengths
    geometric with the given mean; 1.0 means single-base)."""
    import numpy as np

    anc = rng.integers(0, 4, size=ancestor_len)
    alphabet = np.frombuffer(b"ACGT", dtype=np.uint8)
    reads = []
    p_geo = 1.0 / indel_mean
    for _ in range(depth):
        out = []
        u = rng.random(ancestor_len)
        i = 0
        while i < ancestor_len:
            x = u[i]
            if x < dele:
                i += int(rng.geometric(p_geo)) if indel_mean > 1.0 else 1
                continue
            if x < dele + sub:
                out.append((anc[i] + int(rng.integers(1, 4))) % 4)
            else:
                out.append(anc[i])
            if rng.random() < ins:
                k = int(rng.geometric(p_geo)) if indel_mean > 1.0 else 1
                out.extend(int(v) for v in rng.integers(0, 4, size=k))
            i += 1
        reads.append(bytes(alphabet[np.array(out, dtype=np.int64)]) if out else b"")
    return reads
