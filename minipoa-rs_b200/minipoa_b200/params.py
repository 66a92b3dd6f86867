"""Alignment parameters, sequences and alignment items.

Mirrors the reference library types: ``Params`` (minipoa-rs src/lib.rs:47-107,
encode/decode/score at lib.rs:109-138), ``Sequence`` (lib.rs:39-45) and
``AlignedBase`` (lib.rs:140-145). The command-line score-matrix rebuild rule
(src/cli.rs:166-199) is ``Params.from_cli_scores``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional


def default_matrix() -> List[int]:
    """The library default 5x5 DNA matrix (lib.rs:75-81): match 2, mismatch -4,
    N row/column 0 except N-N = 2."""
    m = [0] * 25
    for i in range(4):
        for j in range(4):
            m[i * 5 + j] = 2 if i == j else -4
    m[24] = 2
    return m


class CParams(ctypes.Structure):
    """C layout shared by ``poa_params`` (include/minipoa_b200.h)."""

    _fields_ = [
        ("match_score", ctypes.c_int32),
        ("mismatch", ctypes.c_int32),
        ("gap_open", ctypes.c_int32),
        ("gap_ext", ctypes.c_int32),
        ("b", ctypes.c_uint64),
        ("f", ctypes.c_uint64),
        ("adaptive", ctypes.c_int32),
        ("seeding", ctypes.c_int32),
        ("k", ctypes.c_uint64),
        ("w", ctypes.c_uint64),
        ("progressive", ctypes.c_int32),
        ("result", ctypes.c_int32),
        ("threads", ctypes.c_uint64),
        ("win_band", ctypes.c_uint64),
        ("win_max", ctypes.c_uint64),
        ("mm_filter_ratio", ctypes.c_double),
        ("max_occ", ctypes.c_uint64),
        ("tr_dist", ctypes.c_uint64),
        ("verbose", ctypes.c_int32),
        ("is_rna", ctypes.c_int32),
        ("alphabet_len", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("alphabet", ctypes.POINTER(ctypes.c_uint8)),
        ("matrix", ctypes.POINTER(ctypes.c_int32)),
    ]


@dataclass
class Params:
    match_score: int = 2
    mismatch: int = -4
    gap_open: int = -4
    gap_ext: int = -2
    b: int = 100
    f: int = 40
    adaptive: bool = False
    seeding: bool = False
    k: int = 19
    w: int = 10
    progressive: bool = False
    threads: int = 1
    win_band: int = 500
    win_max: int = 10000
    mm_filter_ratio: float = 0.25
    max_occ: int = 0
    tr_dist: int = 1000
    result: int = 0
    verbose: int = 0
    alphabet: bytes = b"ACGTN"
    matrix: List[int] = field(default_factory=default_matrix)
    is_rna: bool = False

    # lib.rs:110-126
    def encode(self, base) -> int:
        if isinstance(base, str):
            base = ord(base)
        if 97 <= base <= 122:
            base -= 32
        if len(self.alphabet) <= 5 and base == ord("U"):
            base = ord("T")
        i = self.alphabet.find(bytes([base]))
        if i >= 0:
            return i
        i = self.alphabet.find(b"N")
        return i if i >= 0 else len(self.alphabet) - 1

    # lib.rs:127-134
    def decode(self, base: int) -> int:
        c = self.alphabet[base]
        if self.is_rna and len(self.alphabet) <= 5 and c == ord("T"):
            return ord("U")
        return c

    # lib.rs:135-137
    def score(self, a: int, b: int) -> int:
        return self.matrix[a * len(self.alphabet) + b]

    def copy(self, **changes) -> "Params":
        d = dict(self.__dict__)
        d["matrix"] = list(self.matrix)
        d.update(changes)
        return Params(**d)

    @classmethod
    def from_cli_scores(cls, match: int = 2, mismatch: int = -4, gap_open: int = -4, gap_ext: int = -2,
                        **rest) -> "Params":
        """Score flags as the command line normalises them (cli.rs:166-199):
        match positive, penalties negative, and the matrix rebuilt with the
        last (N) row and column 0 except N-N = match."""
        p = cls(match_score=abs(match), mismatch=-abs(mismatch), gap_open=-abs(gap_open),
                gap_ext=-abs(gap_ext), **rest)
        m = len(p.alphabet)
        p.matrix = [0] * (m * m)
        for i in range(m):
            for j in range(m):
                if i == j:
                    v = p.match_score
                elif i == m - 1 or j == m - 1:
                    v = 0
                else:
                    v = p.mismatch
                p.matrix[i * m + j] = v
        return p

    def to_c(self):
        """Returns (CParams, keepalive) for a C call."""
        alpha = (ctypes.c_uint8 * max(1, len(self.alphabet)))(*self.alphabet)
        mat = (ctypes.c_int32 * max(1, len(self.matrix)))(*self.matrix)
        c = CParams(
            match_score=self.match_score, mismatch=self.mismatch, gap_open=self.gap_open,
            gap_ext=self.gap_ext, b=self.b, f=self.f, adaptive=int(bool(self.adaptive)),
            seeding=int(bool(self.seeding)), k=self.k, w=self.w,
            progressive=int(bool(self.progressive)), result=self.result, threads=self.threads,
            win_band=self.win_band, win_max=self.win_max, mm_filter_ratio=self.mm_filter_ratio,
            max_occ=self.max_occ, tr_dist=self.tr_dist, verbose=self.verbose,
            is_rna=int(bool(self.is_rna)), alphabet_len=len(self.alphabet), reserved=0,
            alphabet=ctypes.cast(alpha, ctypes.POINTER(ctypes.c_uint8)),
            matrix=ctypes.cast(mat, ctypes.POINTER(ctypes.c_int32)),
        )
        return c, (alpha, mat)


@dataclass
class Sequence:
    name: str = ""
    comment: str = ""
    seq: bytes = b""
    qual: bytes = b""


@dataclass(frozen=True)
class AlignedBase:
    node: Optional[int]
    base: int
    aligned: Optional[int]
