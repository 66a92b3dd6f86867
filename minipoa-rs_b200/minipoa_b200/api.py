"""Host API mirroring the minipoa-rs library (src/lib.rs, src/align.rs,
src/graph.rs) on top of the C ABI. The DP, traceback, fusion and toposort run
on the B200; this module only marshals arguments and results.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional, Sequence as Seq, Tuple

import numpy as np

from . import _lib
from .params import AlignedBase, Params, Sequence


class PoaError(RuntimeError):
    """A failed call; `code` is the POA_ERR_* status, str() the message."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def dp_backend() -> str:
    """lib.rs:15"""
    return _lib.load().poa_dp_backend().decode()


def int_peak(device: int = 0) -> Tuple[float, float, float]:
    """Measured integer-pipe throughput of `device` in operations per second:
    (plain add, plain max, fused add-max counted as two operations)."""
    out = (ctypes.c_double * 3)()
    rc = _lib.load().poa_probe_int_peak(device, out)
    if rc != 0:
        raise PoaError(rc, "integer throughput probe failed")
    return out[0], out[1], out[2]


def _bytes(x) -> bytes:
    return x.encode() if isinstance(x, str) else bytes(x)


def _seq_arrays(seqs: Seq[bytes]):
    """The C ABI's (pointer array, length array) for `seqs`: the sequences
    joined into one buffer, each pointer its start in it (one copy of the
    bytes, no per-sequence objects). The third value keeps the buffers alive
    while the pointers are in use."""
    seqs = [s if isinstance(s, bytes) else _bytes(s) for s in seqs]
    n = len(seqs)
    lens = np.fromiter((len(s) for s in seqs), dtype=np.int64, count=n)
    if n == 0:
        lens = np.zeros(1, dtype=np.int64)
    joined = b"".join(seqs + [b"\0"])  # (one copy: the terminator joins the list)
    base = np.frombuffer(joined, dtype=np.uint8)
    starts = np.zeros(max(1, n), dtype=np.uint64)
    if n > 1:
        np.cumsum(lens[:-1], out=starts[1:].view(np.int64))
    ptrs = starts + np.uint64(base.ctypes.data)
    arr = ptrs.ctypes.data_as(ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)))
    lens_p = lens.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    return arr, lens_p, (joined, base, ptrs, lens)


class Context:
    """One CUDA device with a stream, a DP arena and a memory budget."""

    def __init__(self, device: int = 0, mem_budget: int = 0):
        self.L = _lib.load()
        h = ctypes.c_void_p()
        rc = self.L.poa_ctx_create(device, mem_budget, ctypes.byref(h))
        if rc != 0:
            raise PoaError(rc, self.L.poa_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.poa_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int):
        if rc != 0:
            raise PoaError(rc, self.L.poa_last_error(self.h).decode())

    def tune_windows(self, one_launch_per_window: bool) -> None:
        """Seeded reads: align a read's seed windows in one launch (False,
        default) or one launch per window (True)."""
        self.check(self.L.poa_ctx_tune_windows(self.h, int(bool(one_launch_per_window))))

    def window_stats(self) -> Tuple[int, int, int]:
        """(windows aligned, launches for them, whole-graph fallbacks) of the
        seeded reads run on this context so far."""
        w, la, fb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.check(self.L.poa_ctx_window_stats(self.h, ctypes.byref(w), ctypes.byref(la), ctypes.byref(fb)))
        return w.value, la.value, fb.value

    def validate(self, params: Params) -> Optional[str]:
        c, keep = params.to_c()
        rc = self.L.poa_params_validate(self.h, ctypes.byref(c))
        return None if rc == 0 else self.L.poa_last_error(self.h).decode()


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context()
    return _default_ctx


def _items_to_list(ptr, n) -> List[AlignedBase]:
    out = []
    for k in range(n):
        it = ptr[k]
        out.append(AlignedBase(None if it.node < 0 else it.node, it.base, None if it.aligned < 0 else it.aligned))
    return out


class Graph:
    """graph.rs Graph, resident in device memory."""

    def __init__(self, params: Optional[Params] = None, ctx: Optional[Context] = None, handle=None):
        self.ctx = ctx or default_context()
        self.L = self.ctx.L
        if handle is None:
            c, keep = (params or Params()).to_c()
            h = ctypes.c_void_p()
            self.ctx.check(self.L.poa_graph_new(self.ctx.h, ctypes.byref(c), ctypes.byref(h)))
            handle = h
        self.h = handle

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.poa_graph_free(self.h)
                self.h = None
        except Exception:
            pass

    # graph.rs:82
    def add_path(self, seq_id: int, path: Seq) -> None:
        arr = (_lib.AlignedBaseC * max(1, len(path)))()
        for k, it in enumerate(path):
            node, base, aligned = (it.node, it.base, it.aligned) if isinstance(it, AlignedBase) else it
            arr[k].node = -1 if node is None else node
            arr[k].base = base
            arr[k].aligned = -1 if aligned is None else aligned
        self.ctx.check(self.L.poa_graph_add_path(self.ctx.h, self.h, seq_id, arr, len(path)))

    # graph.rs:42
    def add_node(self, base: int) -> int:
        out = ctypes.c_int64()
        self.ctx.check(self.L.poa_graph_add_node(self.ctx.h, self.h, base, ctypes.byref(out)))
        return out.value

    # graph.rs:62
    def add_edge(self, a: int, b: int) -> None:
        self.ctx.check(self.L.poa_graph_add_edge(self.ctx.h, self.h, a, b))

    # graph.rs:125
    def toposort(self, grouped: bool = False) -> None:
        self.ctx.check(self.L.poa_graph_toposort(self.ctx.h, self.h, int(grouped)))

    # graph.rs:181
    def consensus(self, params: Params) -> Tuple[bytes, List[int], List[int]]:
        c, keep = params.to_c()
        s = ctypes.POINTER(ctypes.c_uint8)()
        ids = ctypes.POINTER(ctypes.c_int64)()
        cov = ctypes.POINTER(ctypes.c_int64)()
        n = ctypes.c_int64()
        self.ctx.check(self.L.poa_graph_consensus(self.ctx.h, ctypes.byref(c), self.h, ctypes.byref(s),
                                                  ctypes.byref(ids), ctypes.byref(cov), ctypes.byref(n)))
        try:
            return bytes(s[: n.value]), [ids[i] for i in range(n.value)], [cov[i] for i in range(n.value)]
        finally:
            for p in (s, ids, cov):
                self.L.poa_free(ctypes.cast(p, ctypes.c_void_p))

    def _text(self, fn, *args) -> str:
        out = ctypes.c_char_p()
        n = ctypes.c_int64()
        self.ctx.check(fn(*args, ctypes.byref(out), ctypes.byref(n)))
        try:
            return ctypes.string_at(out, n.value).decode()
        finally:
            self.L.poa_free(ctypes.cast(out, ctypes.c_void_p))

    # graph.rs:239
    def msa(self, params: Params, sequences: Seq[Sequence]) -> str:
        c, keep = params.to_c()
        names = (ctypes.c_char_p * max(1, len(sequences)))(*[s.name.encode() for s in sequences])
        comments = (ctypes.c_char_p * max(1, len(sequences)))(*[s.comment.encode() for s in sequences])
        return self._text(self.L.poa_graph_msa, self.ctx.h, ctypes.byref(c), self.h, len(sequences), names,
                          comments)

    # graph.rs:281
    def gfa(self, params: Params, sequences: Seq[Sequence]) -> str:
        c, keep = params.to_c()
        names = (ctypes.c_char_p * max(1, len(sequences)))(*[s.name.encode() for s in sequences])
        return self._text(self.L.poa_graph_gfa, self.ctx.h, ctypes.byref(c), self.h, len(sequences), names)

    def sizes(self) -> _lib.GraphSizes:
        s = _lib.GraphSizes()
        self.ctx.check(self.L.poa_graph_sizes_get(self.ctx.h, self.h, ctypes.byref(s)))
        return s

    def n_nodes(self) -> int:
        return self.sizes().n_nodes

    def dump(self) -> dict:
        """Every public graph field (graph.rs:6-27) as plain lists, in the
        same shape as the oracle's dump."""
        s = self.sizes()
        n, e, npth, pit, sig = s.n_nodes, s.n_edges, s.n_paths, s.path_items, s.alphabet
        A = lambda k: (ctypes.c_int64 * max(1, k))()  # noqa: E731
        fields, rank, aligned = A(4 * n), A(n), A(n * sig)
        icnt, ocnt, ipairs, opairs = A(n), A(n), A(2 * e), A(2 * e)
        pseq, plen, pids = A(npth), A(npth), A(pit)
        self.ctx.check(self.L.poa_graph_export(self.ctx.h, self.h, fields, rank, aligned, icnt, ocnt, ipairs,
                                               opairs, pseq, plen, pids))
        incoming, outgoing = [], []
        a = b = 0
        for i in range(n):
            incoming.append([(ipairs[a + 2 * k], ipairs[a + 2 * k + 1]) for k in range(icnt[i])])
            a += 2 * icnt[i]
            outgoing.append([(opairs[b + 2 * k], opairs[b + 2 * k + 1]) for k in range(ocnt[i])])
            b += 2 * ocnt[i]
        paths, c = [], 0
        for i in range(npth):
            paths.append((pseq[i], list(pids[c:c + plen[i]])))
            c += plen[i]
        return {
            "base": [fields[4 * i] for i in range(n)],
            "parent": [fields[4 * i + 1] for i in range(n)],
            "rank_of": [fields[4 * i + 2] for i in range(n)],
            "coverage": [fields[4 * i + 3] for i in range(n)],
            "incoming": incoming,
            "outgoing": outgoing,
            "rank": list(rank[:s.n_rank]),
            "aligned": [list(aligned[i * sig:(i + 1) * sig]) for i in range(n)],
            "paths": paths,
        }


def _call_path(ctx, fn, *args) -> List[AlignedBase]:
    out = ctypes.POINTER(_lib.AlignedBaseC)()
    n = ctypes.c_int64()
    ctx.check(fn(*args, ctypes.byref(out), ctypes.byref(n)))
    try:
        return _items_to_list(out, n.value)
    finally:
        ctx.L.poa_free(ctypes.cast(out, ctypes.c_void_p))


def align(params: Params, graph: Graph, query: bytes) -> List[AlignedBase]:
    """align.rs:81"""
    c, keep = params.to_c()
    q = _bytes(query)
    qb = (ctypes.c_uint8 * max(1, len(q))).from_buffer_copy(q if q else b"\0")
    return _call_path(graph.ctx, graph.L.poa_align, graph.ctx.h, ctypes.byref(c), graph.h, qb, len(q))


def poa(params: Params, graph: Graph, beg_id: int, end_id: int, query: bytes, adaptive: bool, band_b: int,
        kernel: int = 0, retry: bool = True) -> List[AlignedBase]:
    """align.rs:192 (retry=True) / poa_inner and a forced kernel (retry=False,
    kernel 1 = i32, 2 = i64)."""
    c, keep = params.to_c()
    q = _bytes(query)
    qb = (ctypes.c_uint8 * max(1, len(q))).from_buffer_copy(q if q else b"\0")
    return _call_path(graph.ctx, graph.L.poa_poa, graph.ctx.h, ctypes.byref(c), graph.h, beg_id, end_id, qb,
                      len(q), int(adaptive), band_b, kernel, int(retry))


def align_sequences(params: Params, sequences: Seq, ctx: Optional[Context] = None) -> Graph:
    """lib.rs:177. `sequences` are Sequence records or raw bytes."""
    ctx = ctx or default_context()
    raw = [s.seq if isinstance(s, Sequence) else _bytes(s) for s in sequences]
    c, keep = params.to_c()
    arr, lens, bufs = _seq_arrays(raw)
    h = ctypes.c_void_p()
    ctx.check(ctx.L.poa_align_sequences(ctx.h, ctypes.byref(c), len(raw), arr, lens, ctypes.byref(h)))
    return Graph(ctx=ctx, handle=h)


def extend_graph(params: Params, graph: Graph, sequences: Seq, existing: int) -> None:
    """lib.rs:184"""
    raw = [s.seq if isinstance(s, Sequence) else _bytes(s) for s in sequences]
    c, keep = params.to_c()
    arr, lens, bufs = _seq_arrays(raw)
    graph.ctx.check(graph.L.poa_extend_graph(graph.ctx.h, ctypes.byref(c), graph.h, len(raw), arr, lens, existing))


def read_gfa(params: Params, text, ctx: Optional[Context] = None) -> Tuple["Graph", List[Sequence]]:
    """io::read_gfa (called at lib.rs:214-218): GFA text -> (graph resident on
    the device, the path records in file order)."""
    ctx = ctx or default_context()
    c, keep = params.to_c()
    b = text.encode() if isinstance(text, str) else bytes(text)
    h = ctypes.c_void_p()
    recs = ctypes.c_void_p()
    n = ctypes.c_int64()
    ctx.check(ctx.L.poa_graph_read_gfa(ctx.h, ctypes.byref(c), b, len(b), ctypes.byref(h), ctypes.byref(recs),
                                       ctypes.byref(n)))
    raw = ctypes.string_at(recs, n.value).decode()
    ctx.L.poa_free(recs)
    records = []
    for line in raw.splitlines():
        name, seq = line.split("\t", 1)
        records.append(Sequence(name=name, seq=seq.encode()))
    return Graph(ctx=ctx, handle=h), records


def run(params: Params, sequences: Seq[Sequence], ctx: Optional[Context] = None, incremental=None) -> str:
    """lib.rs:207-242 after input parsing: the optional initial GFA graph
    (`incremental`, GFA text; its path records come first and progressive
    ordering is off), RNA detection, the read loop and the selected output
    (params.result: 0 consensus, 1 MSA, 2 GFA)."""
    params = params.copy()
    if incremental is not None:
        g, records = read_gfa(params, incremental, ctx)
        sequences = records + list(sequences)
    if not sequences:
        raise PoaError(_lib.POA_ERR_INVALID, "input contains no sequences")
    params.is_rna = len(params.alphabet) <= 5 and any(b"U" in s.seq.upper() for s in sequences)
    if incremental is not None:
        extend_graph(params.copy(progressive=False), g, sequences, len(records))
    else:
        g = align_sequences(params, sequences, ctx)
    if params.result == 0:
        return ">consensus sequence\n" + g.consensus(params)[0].decode() + "\n"
    if params.result == 1:
        return g.msa(params, sequences)
    return g.gfa(params, sequences)


class Batch:
    """Independent read sets resident on the device; one run aligns them all
    (mode 0: persistent batched kernel, mode 1: one launch per read)."""

    def __init__(self, params: Params, sets: List[List[bytes]], ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.L = self.ctx.L
        self.params = params
        flat = [s if isinstance(s, bytes) else _bytes(s) for st in sets for s in st]
        off = [0]
        for st in sets:
            off.append(off[-1] + len(st))
        self.n_sets = len(sets)
        self.set_sizes = [len(st) for st in sets]
        c, keep = params.to_c()
        arr, lens, bufs = _seq_arrays(flat)
        offs = (ctypes.c_int64 * len(off))(*off)
        h = ctypes.c_void_p()
        self.ctx.check(self.L.poa_batch_create(self.ctx.h, ctypes.byref(c), len(sets), offs, arr, lens,
                                               ctypes.byref(h)))
        self.h = h

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.poa_batch_free(self.h)
                self.h = None
        except Exception:
            pass

    def autotune(self) -> _lib.BatchTuning:
        """Runs the batch under each candidate launch setting, applies and
        caches the fastest (results are identical under every setting)."""
        t = _lib.BatchTuning()
        self.ctx.check(self.L.poa_batch_autotune(self.ctx.h, self.h, ctypes.byref(t)))
        return t

    def tuning(self) -> _lib.BatchTuning:
        t = _lib.BatchTuning()
        self.ctx.check(self.L.poa_batch_tuning_get(self.ctx.h, self.h, ctypes.byref(t)))
        return t

    def tune(self, warps_per_sm: int = 0, arena_bytes_per_slot: int = 0):
        self.ctx.check(self.L.poa_batch_tune(self.ctx.h, self.h, warps_per_sm, arena_bytes_per_slot))

    def run(self, mode: int = 0) -> _lib.BatchStats:
        st = _lib.BatchStats()
        self.ctx.check(self.L.poa_batch_run(self.ctx.h, self.h, mode, ctypes.byref(st)))
        return st

    def status(self, s: int) -> Optional[str]:
        msg = ctypes.c_char_p()
        rc = self.L.poa_batch_status(self.ctx.h, self.h, s, ctypes.byref(msg))
        if rc == 0:
            return None
        text = msg.value.decode() if msg.value else self.L.poa_last_error(self.ctx.h).decode()
        if msg:
            self.L.poa_free(ctypes.cast(msg, ctypes.c_void_p))
        return text

    def output(self, s: int, result: int, sequences: Optional[Seq[Sequence]] = None) -> str:
        out = ctypes.c_char_p()
        n = ctypes.c_int64()
        names = comments = None
        if sequences is not None:
            names = (ctypes.c_char_p * max(1, len(sequences)))(*[x.name.encode() for x in sequences])
            comments = (ctypes.c_char_p * max(1, len(sequences)))(*[x.comment.encode() for x in sequences])
        self.ctx.check(self.L.poa_batch_output(self.ctx.h, self.h, s, result, names, comments, ctypes.byref(out),
                                               ctypes.byref(n)))
        try:
            return ctypes.string_at(out, n.value).decode()
        finally:
            self.L.poa_free(ctypes.cast(out, ctypes.c_void_p))

    def output_all(self, result: int) -> bytes:
        out = ctypes.c_char_p()
        n = ctypes.c_int64()
        self.ctx.check(self.L.poa_batch_output_all(self.ctx.h, self.h, result, ctypes.byref(out), ctypes.byref(n)))
        try:
            return ctypes.string_at(out, n.value)
        finally:
            self.L.poa_free(ctypes.cast(out, ctypes.c_void_p))

    def transfer_bytes(self):
        h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
        self.ctx.check(self.L.poa_batch_transfer_bytes(self.ctx.h, self.h, ctypes.byref(h2d), ctypes.byref(d2h)))
        return h2d.value, d2h.value

    def graph(self, s: int) -> Graph:
        h = ctypes.c_void_p()
        self.ctx.check(self.L.poa_batch_graph(self.ctx.h, self.h, s, ctypes.byref(h)))
        return Graph(ctx=self.ctx, handle=h)


class Server:
    """Serving loop over the C ABI (poa_server_*): jobs (read sets) are
    submitted at any time and run with continuous batching on the device;
    each finished job's graph stays resident until released. Safe to use
    from several threads (submit on one, wait on others)."""

    def __init__(self, params: Params, ctx: Optional[Context] = None, pool_bytes: int = 0, idle_ms: int = 0):
        self.ctx = ctx or default_context()
        self.L = self.ctx.L
        self.params = params
        self._c, self._keep = params.to_c()
        h = ctypes.c_void_p()
        self.ctx.check(self.L.poa_server_create(self.ctx.h, ctypes.byref(self._c), pool_bytes, idle_ms,
                                                ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.poa_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, reads: Seq[bytes], gfa=None) -> int:
        """Queues a job: its reads, optionally extending an initial graph given
        as GFA text (the -i workflow; the reads' sequence ids follow the GFA's
        path records)."""
        arr, lens, _bufs = _seq_arrays([_bytes(r) for r in reads])
        job = ctypes.c_int64()
        if gfa is None:
            self.ctx.check(self.L.poa_server_submit(self.ctx.h, self.h, len(reads), arr, lens, ctypes.byref(job)))
        else:
            g = gfa.encode() if isinstance(gfa, str) else bytes(gfa)
            self.ctx.check(self.L.poa_server_submit_gfa(self.ctx.h, self.h, g, len(g), len(reads), arr, lens,
                                                        ctypes.byref(job)))
        return job.value

    def wait(self, job: int, timeout_ms: float = -1.0) -> int:
        st = ctypes.c_int32()
        self.ctx.check(self.L.poa_server_wait(self.ctx.h, self.h, job, float(timeout_ms), ctypes.byref(st)))
        return st.value

    def info(self, job: int) -> _lib.ServerJobInfo:
        out = _lib.ServerJobInfo()
        self.ctx.check(self.L.poa_server_job_info(self.ctx.h, self.h, job, ctypes.byref(out)))
        return out

    def output(self, job: int, result: int, sequences: Optional[Seq[Sequence]] = None) -> str:
        out = ctypes.c_char_p()
        n = ctypes.c_int64()
        names = comments = None
        if sequences is not None:
            names = (ctypes.c_char_p * max(1, len(sequences)))(*[x.name.encode() for x in sequences])
            comments = (ctypes.c_char_p * max(1, len(sequences)))(*[x.comment.encode() for x in sequences])
        self.ctx.check(self.L.poa_server_output(self.ctx.h, self.h, job, result, names, comments, ctypes.byref(out),
                                                ctypes.byref(n)))
        try:
            return ctypes.string_at(out, n.value).decode()
        finally:
            self.L.poa_free(ctypes.cast(out, ctypes.c_void_p))

    def release(self, job: int) -> None:
        self.ctx.check(self.L.poa_server_release(self.ctx.h, self.h, job))

    def tune(self, arena_scale: float) -> None:
        self.ctx.check(self.L.poa_server_tune(self.ctx.h, self.h, float(arena_scale)))

    def stats(self) -> _lib.ServerStats:
        out = _lib.ServerStats()
        self.ctx.check(self.L.poa_server_stats_get(self.ctx.h, self.h, ctypes.byref(out)))
        return out


# ---- seed windows (src/minimizer.rs), host only ----------------------------

@dataclasses.dataclass(frozen=True)
class Minimizer:
    value: int
    end: int
    span: int


@dataclasses.dataclass(frozen=True)
class Anchor:
    target_end: int
    query_end: int
    span: int
    adaptive_before: bool = False


def _u8(data: bytes):
    buf = ctypes.create_string_buffer(bytes(data) or b"\0", max(1, len(data)))
    return ctypes.cast(buf, ctypes.POINTER(ctypes.c_uint8)), buf


def _take(L, ptr, n, conv):
    try:
        return [conv(ptr[k]) for k in range(n)]
    finally:
        L.poa_free(ctypes.cast(ptr, ctypes.c_void_p))


def _anchor(a) -> Anchor:
    return Anchor(a.target_end, a.query_end, a.span, bool(a.adaptive_before))


def _anchors_c(anchors: Seq[Anchor]):
    arr = (_lib.AnchorC * max(1, len(anchors)))()
    for k, a in enumerate(anchors):
        arr[k] = _lib.AnchorC(a.target_end, a.query_end, a.span, int(a.adaptive_before), 0)
    return arr


def _check(rc: int):
    if rc != 0:
        raise PoaError(rc, "invalid arguments")


def sketch(seq: bytes, k: int, w: int) -> List[Minimizer]:
    """minimizer::sketch (src/minimizer.rs:39-75)."""
    L = _lib.load()
    p, _keep = _u8(seq)
    out, n = ctypes.POINTER(_lib.MinimizerC)(), ctypes.c_int64()
    _check(L.poa_seed_sketch(p, len(seq), k, w, ctypes.byref(out), ctypes.byref(n)))
    return _take(L, out, n.value, lambda m: Minimizer(m.value, m.end, m.span))


def repeat_intervals(mm: Seq[Minimizer], length: int, max_dist: int) -> List[Tuple[int, int]]:
    """minimizer::repeat_intervals (src/minimizer.rs:79-110)."""
    L = _lib.load()
    arr = (_lib.MinimizerC * max(1, len(mm)))(*[_lib.MinimizerC(m.value, m.end, m.span) for m in mm])
    out, n = ctypes.POINTER(ctypes.c_int64)(), ctypes.c_int64()
    _check(L.poa_seed_repeat_intervals(arr, len(mm), length, max_dist, ctypes.byref(out), ctypes.byref(n)))
    flat = _take(L, out, 2 * n.value, int)
    return [(flat[2 * i], flat[2 * i + 1]) for i in range(n.value)]


def collect_anchors(params: Params, query: bytes, target: bytes) -> List[Anchor]:
    """minimizer::collect_anchors (src/minimizer.rs:128-172)."""
    L = _lib.load()
    c, _k = params.to_c()
    q, _kq = _u8(query)
    t, _kt = _u8(target)
    out, n = ctypes.POINTER(_lib.AnchorC)(), ctypes.c_int64()
    _check(L.poa_seed_collect_anchors(ctypes.byref(c), q, len(query), t, len(target), ctypes.byref(out),
                                      ctypes.byref(n)))
    return _take(L, out, n.value, _anchor)


def chain(anchors: Seq[Anchor], k: int) -> List[Anchor]:
    """minimizer::chain (src/minimizer.rs:199-366)."""
    L = _lib.load()
    out, n = ctypes.POINTER(_lib.AnchorC)(), ctypes.c_int64()
    _check(L.poa_seed_chain(_anchors_c(anchors), len(anchors), k, ctypes.byref(out), ctypes.byref(n)))
    return _take(L, out, n.value, _anchor)


def partition_windows(chain_: Seq[Anchor], tlen: int, qlen: int, max_drift: int,
                      max_win: int) -> Tuple[List[Anchor], bool]:
    """minimizer::partition_windows (src/minimizer.rs:371-457)."""
    L = _lib.load()
    out, n, tail = ctypes.POINTER(_lib.AnchorC)(), ctypes.c_int64(), ctypes.c_int32()
    _check(L.poa_seed_partition_windows(_anchors_c(chain_), len(chain_), tlen, qlen, max_drift, max_win,
                                        ctypes.byref(out), ctypes.byref(n), ctypes.byref(tail)))
    return _take(L, out, n.value, _anchor), bool(tail.value)


def anchor_windows(params: Params, query: bytes, consensus: bytes) -> Tuple[List[Anchor], bool]:
    """minimizer::anchor_windows (src/minimizer.rs:466-479)."""
    L = _lib.load()
    c, _k = params.to_c()
    q, _kq = _u8(query)
    t, _kt = _u8(consensus)
    out, n, tail = ctypes.POINTER(_lib.AnchorC)(), ctypes.c_int64(), ctypes.c_int32()
    _check(L.poa_seed_anchor_windows(ctypes.byref(c), q, len(query), t, len(consensus), ctypes.byref(out),
                                     ctypes.byref(n), ctypes.byref(tail)))
    return _take(L, out, n.value, _anchor), bool(tail.value)


def guide_order(params: Params, reads: Seq[bytes]) -> List[int]:
    """minimizer::guide_order (src/minimizer.rs:505-578): the order in which
    progressive alignment (params.progressive, -p) adds the reads."""
    L = _lib.load()
    c, _k = params.to_c()
    arr, lens, _bufs = _seq_arrays(reads)
    out = ctypes.POINTER(ctypes.c_int64)()
    _check(L.poa_seed_guide_order(ctypes.byref(c), len(reads), arr, lens, ctypes.byref(out)))
    return _take(L, out, len(reads), int)
