"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over oracle/liboracle.so, the CPU restatement of minipoa-rs's
partial-order-alignment path (src/align.rs, src/graph.rs, src/lib.rs). Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module; the shipped library never does.

Parity pinning: the reference crate cannot be built (src/io.rs is missing and
no Rust toolchain is present), so the restatement is pinned by the reference's
own known-answer and property tests, restated in tests/test_oracle_*.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence as Seq

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

AUTO_SERIAL, FORCE_I64, AUTO_AVX2, I32_ONLY, I64_ONLY = 0, 1, 2, 3, 4


class _CParams(ctypes.Structure):
    _fields_ = [
        ("match_score", ctypes.c_int32), ("mismatch", ctypes.c_int32), ("gap_open", ctypes.c_int32),
        ("gap_ext", ctypes.c_int32), ("b", ctypes.c_uint64), ("f", ctypes.c_uint64),
        ("adaptive", ctypes.c_int32), ("seeding", ctypes.c_int32), ("k", ctypes.c_uint64),
        ("w", ctypes.c_uint64), ("progressive", ctypes.c_int32), ("result", ctypes.c_int32),
        ("threads", ctypes.c_uint64), ("win_band", ctypes.c_uint64), ("win_max", ctypes.c_uint64),
        ("mm_filter_ratio", ctypes.c_double), ("max_occ", ctypes.c_uint64), ("tr_dist", ctypes.c_uint64),
        ("verbose", ctypes.c_int32), ("is_rna", ctypes.c_int32), ("alphabet_len", ctypes.c_int32),
        ("reserved", ctypes.c_int32), ("alphabet", ctypes.POINTER(ctypes.c_uint8)),
        ("matrix", ctypes.POINTER(ctypes.c_int32)),
    ]


class _Item(ctypes.Structure):
    _fields_ = [("node", ctypes.c_int64), ("base", ctypes.c_int64), ("aligned", ctypes.c_int64)]


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        vp, i64, u64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64
        cp = P(_CParams)
        L.orc_graph_new.argtypes = [cp]
        L.orc_graph_new.restype = vp
        L.orc_graph_free.argtypes = [vp]
        L.orc_graph_clone.argtypes = [vp]
        L.orc_graph_clone.restype = vp
        L.orc_free.argtypes = [vp]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_align_sequences.argtypes = [cp, i64, P(P(ctypes.c_uint8)), P(i64), ctypes.c_int, P(vp)]
        L.orc_extend_graph.argtypes = [cp, vp, i64, P(P(ctypes.c_uint8)), P(i64), i64, ctypes.c_int]
        L.orc_align_sequences_in_order.argtypes = [cp, i64, P(P(ctypes.c_uint8)), P(i64), P(i64), ctypes.c_int,
                                                   P(vp)]
        L.orc_align.argtypes = [cp, vp, P(ctypes.c_uint8), i64, ctypes.c_int, P(P(_Item)), P(i64)]
        L.orc_poa.argtypes = [cp, vp, i64, i64, P(ctypes.c_uint8), i64, ctypes.c_int, u64, ctypes.c_int,
                              ctypes.c_int, P(P(_Item)), P(i64)]
        L.orc_i32_scores_safe.argtypes = [cp, vp, i64, i64, i64]
        L.orc_add_path.argtypes = [cp, vp, i64, P(_Item), i64]
        L.orc_toposort.argtypes = [vp, ctypes.c_int]
        L.orc_add_node.argtypes = [vp, i64]
        L.orc_add_node.restype = i64
        L.orc_add_edge.argtypes = [vp, i64, i64]
        L.orc_consensus.argtypes = [cp, vp, P(P(ctypes.c_uint8)), P(P(i64)), P(P(i64)), P(i64)]
        L.orc_msa.argtypes = [cp, vp, i64, P(ctypes.c_char_p), P(ctypes.c_char_p), P(ctypes.c_char_p), P(i64)]
        L.orc_gfa.argtypes = [cp, vp, i64, P(ctypes.c_char_p), P(ctypes.c_char_p), P(i64)]
        L.orc_params_validate.argtypes = [cp]
        L.orc_encode.argtypes = [cp, ctypes.c_uint8]
        L.orc_encode.restype = i64
        L.orc_graph_nodes.argtypes = [vp]
        L.orc_graph_nodes.restype = i64
        L.orc_graph_paths.argtypes = [vp]
        L.orc_graph_paths.restype = i64
        L.orc_graph_node_fields.argtypes = [vp, P(i64)]
        L.orc_graph_edge_total.argtypes = [vp]
        L.orc_graph_edge_total.restype = i64
        L.orc_graph_edges.argtypes = [vp, P(i64), P(i64), P(i64), P(i64)]
        L.orc_graph_rank.argtypes = [vp, P(i64)]
        L.orc_graph_rank_len.argtypes = [vp]
        L.orc_graph_rank_len.restype = i64
        L.orc_graph_aligned.argtypes = [vp, P(i64)]
        L.orc_graph_path_total.argtypes = [vp]
        L.orc_graph_path_total.restype = i64
        L.orc_graph_path_data.argtypes = [vp, P(i64), P(i64), P(i64)]
        L.orc_cells.restype = u64
        L.orc_batch_run.argtypes = [cp, i64, P(i64), P(P(ctypes.c_uint8)), P(i64), ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, P(u64), P(u64)]
        L.orc_avx2_prefix.argtypes = [P(ctypes.c_int32), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                      P(ctypes.c_int32)]
        L.orc_read_gfa.argtypes = [cp, ctypes.c_char_p, i64, P(vp), P(ctypes.c_void_p), P(i64)]
        L.orc_fnv1a.argtypes = [ctypes.c_char_p, i64]
        L.orc_fnv1a.restype = u64
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _params(p):
    alpha = (ctypes.c_uint8 * max(1, len(p.alphabet)))(*p.alphabet)
    mat = (ctypes.c_int32 * max(1, len(p.matrix)))(*p.matrix)
    c = _CParams(
        match_score=p.match_score, mismatch=p.mismatch, gap_open=p.gap_open, gap_ext=p.gap_ext, b=p.b, f=p.f,
        adaptive=int(bool(p.adaptive)), seeding=int(bool(p.seeding)), k=p.k, w=p.w,
        progressive=int(bool(p.progressive)), result=p.result, threads=p.threads, win_band=p.win_band,
        win_max=p.win_max, mm_filter_ratio=p.mm_filter_ratio, max_occ=p.max_occ, tr_dist=p.tr_dist,
        verbose=p.verbose, is_rna=int(bool(p.is_rna)), alphabet_len=len(p.alphabet), reserved=0,
        alphabet=ctypes.cast(alpha, ctypes.POINTER(ctypes.c_uint8)),
        matrix=ctypes.cast(mat, ctypes.POINTER(ctypes.c_int32)))
    return c, (alpha, mat)


def _check(rc):
    if rc != 0:
        raise OracleError(lib().orc_last_error().decode())


def _seqs(seqs: Seq[bytes]):
    bufs = [(ctypes.c_uint8 * max(1, len(s))).from_buffer_copy(bytes(s) if len(s) else b"\0") for s in seqs]
    arr = (ctypes.POINTER(ctypes.c_uint8) * max(1, len(seqs)))(
        *[ctypes.cast(b, ctypes.POINTER(ctypes.c_uint8)) for b in bufs])
    lens = (ctypes.c_int64 * max(1, len(seqs)))(*[len(s) for s in seqs])
    return arr, lens, bufs


def _items(ptr, n):
    out = []
    for i in range(n):
        it = ptr[i]
        out.append((None if it.node < 0 else it.node, it.base, None if it.aligned < 0 else it.aligned))
    lib().orc_free(ptr)
    return out


def _query(q: bytes):
    q = bytes(q)
    return (ctypes.c_uint8 * max(1, len(q))).from_buffer_copy(q if q else b"\0"), len(q)


class OracleGraph:
    """graph.rs Graph held by the oracle."""

    def __init__(self, params=None, handle=None):
        if handle is None:
            c, keep = _params(params)
            handle = lib().orc_graph_new(ctypes.byref(c))
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_graph_free(self.h)
            self.h = None

    def clone(self) -> "OracleGraph":
        return OracleGraph(handle=lib().orc_graph_clone(self.h))

    def align(self, params, query: bytes, kernel=AUTO_SERIAL):
        c, keep = _params(params)
        qb, n = _query(query)
        out = ctypes.POINTER(_Item)()
        ln = ctypes.c_int64()
        _check(lib().orc_align(ctypes.byref(c), self.h, qb, n, kernel, ctypes.byref(out), ctypes.byref(ln)))
        return _items(out, ln.value)

    def poa(self, params, beg_id, end_id, query: bytes, adaptive: bool, band_b: int, kernel=AUTO_SERIAL,
            retry=True):
        c, keep = _params(params)
        qb, n = _query(query)
        out = ctypes.POINTER(_Item)()
        ln = ctypes.c_int64()
        _check(lib().orc_poa(ctypes.byref(c), self.h, beg_id, end_id, qb, n, int(adaptive), band_b, kernel,
                             int(retry), ctypes.byref(out), ctypes.byref(ln)))
        return _items(out, ln.value)

    def i32_scores_safe(self, params, beg_id, end_id, qlen) -> bool:
        c, keep = _params(params)
        return bool(lib().orc_i32_scores_safe(ctypes.byref(c), self.h, beg_id, end_id, qlen))

    def add_path(self, params, seq_id: int, items):
        c, keep = _params(params)
        arr = (_Item * max(1, len(items)))()
        for i, (node, base, aligned) in enumerate(items):
            arr[i].node = -1 if node is None else node
            arr[i].base = base
            arr[i].aligned = -1 if aligned is None else aligned
        _check(lib().orc_add_path(ctypes.byref(c), self.h, seq_id, arr, len(items)))

    def add_node(self, base: int) -> int:
        return lib().orc_add_node(self.h, base)

    def add_edge(self, a: int, b: int):
        lib().orc_add_edge(self.h, a, b)

    def toposort(self, grouped=False):
        _check(lib().orc_toposort(self.h, int(grouped)))

    def consensus(self, params):
        c, keep = _params(params)
        s = ctypes.POINTER(ctypes.c_uint8)()
        ids = ctypes.POINTER(ctypes.c_int64)()
        cov = ctypes.POINTER(ctypes.c_int64)()
        n = ctypes.c_int64()
        _check(lib().orc_consensus(ctypes.byref(c), self.h, ctypes.byref(s), ctypes.byref(ids), ctypes.byref(cov),
                                   ctypes.byref(n)))
        seq = bytes(s[: n.value])
        idl = [ids[i] for i in range(n.value)]
        cvl = [cov[i] for i in range(n.value)]
        for p in (s, ids, cov):
            lib().orc_free(p)
        return seq, idl, cvl

    def msa(self, params, sequences) -> str:
        c, keep = _params(params)
        names = (ctypes.c_char_p * max(1, len(sequences)))(*[s.name.encode() for s in sequences])
        comments = (ctypes.c_char_p * max(1, len(sequences)))(*[s.comment.encode() for s in sequences])
        out = ctypes.c_char_p()
        n = ctypes.c_int64()
        _check(lib().orc_msa(ctypes.byref(c), self.h, len(sequences), names, comments, ctypes.byref(out),
                             ctypes.byref(n)))
        s = ctypes.string_at(out, n.value).decode()
        lib().orc_free(ctypes.cast(out, ctypes.c_void_p))
        return s

    def gfa(self, params, sequences) -> str:
        c, keep = _params(params)
        names = (ctypes.c_char_p * max(1, len(sequences)))(*[s.name.encode() for s in sequences])
        out = ctypes.c_char_p()
        n = ctypes.c_int64()
        _check(lib().orc_gfa(ctypes.byref(c), self.h, len(sequences), names, ctypes.byref(out), ctypes.byref(n)))
        s = ctypes.string_at(out, n.value).decode()
        lib().orc_free(ctypes.cast(out, ctypes.c_void_p))
        return s

    # -- inspection ---------------------------------------------------------
    def n_nodes(self) -> int:
        return lib().orc_graph_nodes(self.h)

    def dump(self, alphabet_size: int) -> dict:
        """All graph state as plain lists (nodes, edges in insertion order,
        ranks, column groups, paths) for exact comparison."""
        L = lib()
        n = L.orc_graph_nodes(self.h)
        f = (ctypes.c_int64 * (4 * n))()
        L.orc_graph_node_fields(self.h, f)
        e = L.orc_graph_edge_total(self.h)
        ic = (ctypes.c_int64 * n)()
        oc = (ctypes.c_int64 * n)()
        ip = (ctypes.c_int64 * max(1, 2 * e))()
        op = (ctypes.c_int64 * max(1, 2 * e))()
        L.orc_graph_edges(self.h, ic, oc, ip, op)
        nr = L.orc_graph_rank_len(self.h)
        rk = (ctypes.c_int64 * max(1, nr))()
        L.orc_graph_rank(self.h, rk)
        al = (ctypes.c_int64 * (n * alphabet_size))()
        L.orc_graph_aligned(self.h, al)
        npaths = L.orc_graph_paths(self.h)
        pt = L.orc_graph_path_total(self.h)
        sid = (ctypes.c_int64 * max(1, npaths))()
        pl = (ctypes.c_int64 * max(1, npaths))()
        ids = (ctypes.c_int64 * max(1, pt))()
        L.orc_graph_path_data(self.h, sid, pl, ids)
        incoming, outgoing = [], []
        a = b = 0
        for i in range(n):
            incoming.append([(ip[a + 2 * k], ip[a + 2 * k + 1]) for k in range(ic[i])])
            a += 2 * ic[i]
            outgoing.append([(op[b + 2 * k], op[b + 2 * k + 1]) for k in range(oc[i])])
            b += 2 * oc[i]
        paths = []
        c = 0
        for i in range(npaths):
            paths.append((sid[i], list(ids[c:c + pl[i]])))
            c += pl[i]
        return {
            "base": [f[4 * i] for i in range(n)],
            "parent": [f[4 * i + 1] for i in range(n)],
            "rank_of": [f[4 * i + 2] for i in range(n)],
            "coverage": [f[4 * i + 3] for i in range(n)],
            "incoming": incoming,
            "outgoing": outgoing,
            "rank": list(rk[:nr]),
            "aligned": [list(al[i * alphabet_size:(i + 1) * alphabet_size]) for i in range(n)],
            "paths": paths,
        }


def align_sequences(params, seqs: Seq[bytes], kernel=AUTO_SERIAL) -> OracleGraph:
    """lib.rs:177"""
    c, keep = _params(params)
    arr, lens, bufs = _seqs(seqs)
    out = ctypes.c_void_p()
    _check(lib().orc_align_sequences(ctypes.byref(c), len(seqs), arr, lens, kernel, ctypes.byref(out)))
    return OracleGraph(handle=out.value)


def align_sequences_in_order(params, seqs: Seq[bytes], order: Seq[int], kernel=AUTO_SERIAL) -> OracleGraph:
    """lib.rs:177 with progressive (-p): the reads added in `order` (the
    guide order, src/minimizer.rs:505-578, computed from the same sketches
    as the GPU path's)."""
    c, keep = _params(params)
    arr, lens, bufs = _seqs(seqs)
    od = (ctypes.c_int64 * max(1, len(order)))(*order)
    out = ctypes.c_void_p()
    _check(lib().orc_align_sequences_in_order(ctypes.byref(c), len(seqs), arr, lens, od, kernel,
                                              ctypes.byref(out)))
    return OracleGraph(handle=out.value)


def extend_graph(params, graph: OracleGraph, seqs: Seq[bytes], existing: int, kernel=AUTO_SERIAL):
    """lib.rs:184"""
    c, keep = _params(params)
    arr, lens, bufs = _seqs(seqs)
    _check(lib().orc_extend_graph(ctypes.byref(c), graph.h, len(seqs), arr, lens, existing, kernel))


def validate(params) -> Optional[str]:
    c, keep = _params(params)
    rc = lib().orc_params_validate(ctypes.byref(c))
    return None if rc == 0 else lib().orc_last_error().decode()


def reset_cells():
    lib().orc_reset_cells()


def cells() -> int:
    return lib().orc_cells()


def batch_run(params, sets: List[List[bytes]], kernel=AUTO_AVX2, threads=1, out_format=-1):
    """Independent read sets on `threads` host threads. Returns (cells, hashes)."""
    c, keep = _params(params)
    flat = [s for st in sets for s in st]
    off = [0]
    for st in sets:
        off.append(off[-1] + len(st))
    arr, lens, bufs = _seqs(flat)
    offs = (ctypes.c_int64 * len(off))(*off)
    hashes = (ctypes.c_uint64 * max(1, len(sets)))()
    cells_out = ctypes.c_uint64()
    _check(lib().orc_batch_run(ctypes.byref(c), len(sets), offs, arr, lens, kernel, threads, out_format, hashes,
                               ctypes.byref(cells_out)))
    return cells_out.value, list(hashes[: len(sets)])


def avx2_prefix(md: List[int], carry: int, open_: int, ext: int) -> List[int]:
    a = (ctypes.c_int32 * 8)(*md)
    o = (ctypes.c_int32 * 8)()
    lib().orc_avx2_prefix(a, carry, open_, ext, o)
    return list(o)


def avx2_available() -> bool:
    return bool(lib().orc_avx2_available())


def fnv1a(data) -> int:
    """FNV-1a of a text or byte string, the hash batch_run reports per set."""
    b = data.encode() if isinstance(data, str) else bytes(data)
    return lib().orc_fnv1a(b, len(b))


def read_gfa(params, text):
    """GFA text -> (OracleGraph, [(name, sequence)]) (io::read_gfa as restated
    in poa_oracle.cpp from the reference's tests)."""
    c, keep = _params(params)
    b = text.encode() if isinstance(text, str) else bytes(text)
    h = ctypes.c_void_p()
    recs = ctypes.c_void_p()
    n = ctypes.c_int64()
    _check(lib().orc_read_gfa(ctypes.byref(c), b, len(b), ctypes.byref(h), ctypes.byref(recs), ctypes.byref(n)))
    raw = ctypes.string_at(recs, n.value).decode()
    lib().orc_free(recs)
    records = [tuple(line.split("\t", 1)) for line in raw.splitlines()]
    return OracleGraph(params, handle=h.value), [(nm, sq.encode()) for nm, sq in records]
