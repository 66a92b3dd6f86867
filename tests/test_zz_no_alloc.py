"""poa_align_noalloc: the alignment entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc when they align -- a serving
loop whose device memory belongs to another allocator, a strict memory
budget, or a thread that must not trigger the device-wide synchronisation of
cudaMalloc/cudaFree. Its scratch is one fixed library-owned array, so these
checks compare it, through the C ABI, with poa_align on two calls in a row
(the second call must not see the first call's leftovers), and check that an
oversized request is refused with a clear error instead of running.

The file sorts last so a run that stops at the first failure has already run
every other test. It passes alone in a fresh process and after the others.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    import minipoa_b200 as mp
    from minipoa_b200 import _lib

    ctx = mp.default_context()
    return mp, _lib, ctx, torch


def _noalloc(mp, _lib, ctx, torch, params, graph, query: bytes):
    """Calls poa_align_noalloc with caller-owned device buffers (the test
    allocates them; the entry point does not)."""
    q = torch.tensor(list(query) or [0], dtype=torch.uint8, device="cuda")
    cap = len(query) + 1
    out = torch.full((cap * 3,), -7, dtype=torch.int64, device="cuda")
    n = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    c, keep = params.to_c()
    rc = ctx.L.poa_align_noalloc(ctx.h, ctypes.byref(c), graph.h, ctypes.c_void_p(q.data_ptr()), len(query),
                                 ctypes.c_void_p(out.data_ptr()), cap, ctypes.c_void_p(n.data_ptr()))
    torch.cuda.synchronize()
    if rc != 0:
        raise mp.PoaError(rc, ctx.L.poa_last_error(ctx.h).decode())
    k = int(n.item())
    vals = out[: 3 * k].cpu().tolist()
    return [(None if vals[3 * i] < 0 else vals[3 * i], vals[3 * i + 1],
             None if vals[3 * i + 2] < 0 else vals[3 * i + 2]) for i in range(k)]


def _tup(path):
    return [(a.node, a.base, a.aligned) for a in path]


def test_noalloc_matches_align_on_two_calls_in_a_row(env):
    mp, _lib, ctx, torch = env
    from minipoa_b200 import workloads

    rng = np.random.default_rng(2024)
    reads = workloads.read_set(rng, 800, 8, 0.03, 0.01, 0.01)
    for adaptive in (False, True):
        params = mp.Params(adaptive=adaptive)
        g = mp.align_sequences(params, reads[:6])
        # two different queries back to back: exact integer parity with poa_align
        for q in (reads[6], reads[7]):
            want = _tup(mp.align(params, g, q))
            got = _noalloc(mp, _lib, ctx, torch, params, g, q)
            assert got == want
        # and the same query again after a different one
        assert _noalloc(mp, _lib, ctx, torch, params, g, reads[6]) == _tup(mp.align(params, g, reads[6]))


def test_noalloc_rejects_requests_beyond_its_scratch(env):
    mp, _lib, ctx, torch = env
    params = mp.Params(f=0)
    g = mp.align_sequences(params, [b"ACGT" * 500])
    with pytest.raises(mp.PoaError, match="no-allocation scratch") as e:
        _noalloc(mp, _lib, ctx, torch, params, g, b"ACGT" * 200000)
    assert e.value.code == _lib.POA_ERR_ALLOC
    # the graph stays usable afterwards
    q = b"ACGTACGAACGT" * 20
    assert _noalloc(mp, _lib, ctx, torch, params, g, q) == _tup(mp.align(params, g, q))


def test_noalloc_rejects_a_graph_of_another_context(env):
    # a graph lives on its own context's stream; aligning it through another
    # context would read its descriptor before the launch finished
    mp, _lib, ctx, torch = env
    params = mp.Params()
    other = mp.Context(0)
    g = mp.align_sequences(params, [b"ACGTACGT", b"ACGAACGT"], ctx=other)
    with pytest.raises(mp.PoaError, match="another context") as e:
        _noalloc(mp, _lib, ctx, torch, params, g, b"ACGTACGT")
    assert e.value.code == _lib.POA_ERR_INVALID
    del g
    other.close()
