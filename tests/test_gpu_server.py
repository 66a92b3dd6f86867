"""The serving loop (poa_server_*, continuous batching) through the C ABI:
a job's result is the same alone and in a mix of concurrently admitted
jobs, equals the batched kernel's and the oracle's, survives arena growth
(parking) and several submitting threads, and a job larger than the pool is
refused with a message."""
import threading

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


def _jobs(seed, n, lmin, lmax, dmin, dmax):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(np.exp(rng.uniform(np.log(lmin), np.log(lmax))))
        d = int(rng.integers(dmin, dmax + 1))
        e = rng.uniform(0.02, 0.15)
        out.append(rc.synthetic_reads(rng, L, d, 0.6 * e, 0.2 * e, 0.2 * e))
    return out


def _outputs(server, job, reads):
    recs = [Sequence(name=f"read{i}", seq=x) for i, x in enumerate(reads)]
    return [server.output(job, r, recs) for r in (0, 1, 2)]


def test_server_results_same_alone_and_in_the_mix(mp, oracle):
    params = Params()
    jobs = _jobs(2025, 30, 150, 1500, 3, 12)
    server = mp.Server(params)
    x = jobs[15]
    jx = server.submit(x)
    assert server.wait(jx) == mp._lib.POA_SERVER_DONE
    alone = _outputs(server, jx, x)
    server.release(jx)
    ids = [server.submit(r) for r in jobs]
    states = [server.wait(i) for i in ids]
    assert all(s == mp._lib.POA_SERVER_DONE for s in states)
    assert _outputs(server, ids[15], x) == alone
    # every job equals the batched kernel's bytes; a few also the oracle's
    batch = mp.Batch(params, jobs)
    batch.run(0)
    for s, i in enumerate(ids):
        assert server.output(i, 0) == batch.output(s, 0)
        assert server.output(i, 2) == batch.output(s, 2)
        info = server.info(i)
        assert info.cells > 0 and info.latency_ms > 0
    for s in (0, 7, 15):
        o = oracle.align_sequences(params, jobs[s])
        assert server.output(ids[s], 0) == ">consensus sequence\n" + o.consensus(params)[0].decode() + "\n"
    st = server.stats()
    assert st.done_jobs == 31 and st.waves >= 2
    for i in ids:
        server.release(i)
    server.close()


def test_server_parks_jobs_and_grows_their_arena(mp):
    params = Params()
    jobs = _jobs(77, 10, 300, 900, 8, 14)
    server = mp.Server(params)
    server.tune(0.02)  # far too little arena: every job parks and comes back
    ids = [server.submit(r) for r in jobs]
    assert all(server.wait(i) == mp._lib.POA_SERVER_DONE for i in ids)
    batch = mp.Batch(params, jobs)
    batch.run(0)
    for s, i in enumerate(ids):
        assert server.output(i, 2) == batch.output(s, 2)
    assert server.stats().waves > 1
    server.close()


def test_server_threads_submit_and_wait_concurrently(mp):
    params = Params()
    jobs = _jobs(31, 24, 150, 800, 3, 8)
    server = mp.Server(params)
    results, errors = {}, []

    def worker(k):
        try:
            for s in range(k, len(jobs), 4):
                j = server.submit(jobs[s])
                server.wait(j)
                results[s] = server.output(j, 0)
                server.release(j)
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    th = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert errors == []
    batch = mp.Batch(params, jobs)
    batch.run(0)
    assert [results[s] for s in range(len(jobs))] == [batch.output(s, 0) for s in range(len(jobs))]
    server.close()


def test_server_refuses_a_job_larger_than_its_pool(mp):
    params = Params()
    ctx = mp.Context(0)
    server = mp.Server(params, ctx=ctx, pool_bytes=64 << 20)
    big = [b"ACGT" * 50000] * 4
    j = server.submit(big)
    assert server.wait(j) == mp._lib.POA_SERVER_FAILED
    with pytest.raises(mp.PoaError, match="more device memory than the server pool"):
        server.info(j)
    small = server.submit([b"ACGTACGT", b"ACGAACGT"])
    assert server.wait(small) == mp._lib.POA_SERVER_DONE
    server.close()


def test_server_extends_gfa_graphs_like_the_oracle(mp, oracle):
    # serving jobs that bring an initial graph (GFA of prior reads) and new
    # reads, mixed with plain jobs: each result equals the oracle's read_gfa +
    # extend_graph (the -i workflow, src/lib.rs:214-231)
    params = Params()
    rng = np.random.default_rng(606)
    server = mp.Server(params)
    cases = []
    for k in range(6):
        reads = rc.synthetic_reads(rng, int(rng.integers(200, 700)), int(rng.integers(12, 30)), 0.05, 0.015, 0.015)
        n_prior = int(rng.integers(4, 10))
        prior, new = reads[:n_prior], reads[n_prior:]
        names = [Sequence(name=f"p{i}", seq=s) for i, s in enumerate(prior)]
        gfa = oracle.align_sequences(params, prior).gfa(params, names)
        cases.append((gfa, names, new))
    plain = _jobs(9, 6, 150, 600, 3, 8)
    ids = []
    for k in range(6):
        ids.append(server.submit(cases[k][2], gfa=cases[k][0]))
        server.submit(plain[k])
    for k, (gfa, names, new) in enumerate(cases):
        assert server.wait(ids[k]) == mp._lib.POA_SERVER_DONE
        o, orecs = oracle.read_gfa(params, gfa)
        allrecs = names + [Sequence(name=f"n{i}", seq=s) for i, s in enumerate(new)]
        oracle.extend_graph(params, o, [r.seq for r in allrecs], len(orecs))
        assert server.output(ids[k], 1, allrecs) == o.msa(params, allrecs)
        assert server.output(ids[k], 2, allrecs) == o.gfa(params, allrecs)
        assert server.output(ids[k], 0) == ">consensus sequence\n" + o.consensus(params)[0].decode() + "\n"
    with pytest.raises(mp.PoaError, match="revisits"):
        server.submit([b"ACGT"], gfa="S\ta\tA\nP\tc\ta+,a+\t*\n")
    server.close()
