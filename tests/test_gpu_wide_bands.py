"""Bands wider than one striped tile (512 columns) on the GPU against the
oracle. The windowed entry point (poa, src/align.rs:192-211, and poa_inner,
src/align.rs:531-545) computes rows of up to 2048 columns as 512-column
segments chained by their insertion state, and wider rows by the generic row;
paths (and errors) must equal the oracle's for static and adaptive bands on
both sides of every segment boundary, with the full matrix (f = 0) too.
Seeded windows, whose static band is 500 on each side, run the same code.
"""
import numpy as np
import pytest

from minipoa_b200.params import Params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mp():
    import minipoa_b200 as m

    m.default_context()
    return m


def tup(path):
    return [(a.node, a.base, a.aligned) if hasattr(a, "node") else tuple(a) for a in path]


def res(fn):
    try:
        return ("ok", tup(fn()))
    except Exception as e:
        return ("err", str(e))


@pytest.mark.parametrize("anc_len", [1100, 2600])
def test_wide_bands_match_oracle(mp, oracle, anc_len):
    from minipoa_b200 import workloads

    rng = np.random.default_rng(4242 + anc_len)
    reads = workloads.read_set(rng, anc_len, 6, 0.04, 0.02, 0.02, indel_mean=1.5)
    params = Params()
    g = mp.align_sequences(params, reads[:5])
    o = oracle.align_sequences(params, reads[:5])
    assert g.dump() == o.dump(5)
    q = reads[5]
    n = 0
    for f, adaptive, band in [(0, False, 0), (40, False, 200), (40, False, 250), (40, False, 300),
                              (40, False, 700), (40, False, 1000), (40, False, 1500),
                              (40, True, 300), (40, True, 700), (40, True, 1100)]:
        params.f = f
        params.adaptive = adaptive
        got = res(lambda: mp.poa(params, g, 0, 1, q, adaptive, band, kernel=1, retry=False))
        want = res(lambda: o.poa(params, 0, 1, q, adaptive, band, 3, retry=False))
        assert got == want, (anc_len, f, adaptive, band)
        got = res(lambda: mp.poa(params, g, 0, 1, q, adaptive, band, kernel=0, retry=True))
        want = res(lambda: o.poa(params, 0, 1, q, adaptive, band))
        assert got == want, (anc_len, f, adaptive, band, "retry")
        n += 1
    assert n == 10


def test_wide_window_band_read_loop_matches_oracle(mp, oracle):
    # whole reads through windows of the seeded path with a window band that
    # keeps every row in the segmented form
    from minipoa_b200 import workloads

    rng = np.random.default_rng(77)
    reads = workloads.read_set(rng, 4000, 5, 0.03, 0.01, 0.01, indel_mean=1.5)
    for win_band in (300, 900):
        params = Params(seeding=True, result=1, win_band=win_band)
        g = mp.align_sequences(params, reads)
        # the same windows on the oracle side (shared host windows)
        from test_gpu_seeded import oracle_seeded

        o = oracle_seeded(mp, oracle, params, reads)
        assert g.dump() == o.dump(5), win_band
