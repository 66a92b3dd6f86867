"""The batched kernel's autotuner and its CUDA-graph replay, through the C
ABI: every candidate launch setting gives the same bytes, the chosen setting
is cached per size bucket and applied to the next batch of that bucket, and
repeated runs replay the captured first pass."""
import os

import numpy as np
import pytest

import refcases as rc
from minipoa_b200.params import Params

pytestmark = pytest.mark.gpu


def test_autotune_caches_a_setting_and_keeps_the_bytes(tmp_path, monkeypatch):
    import minipoa_b200 as mp

    monkeypatch.setenv("MINIPOA_B200_TUNE_CACHE", str(tmp_path / "tune.tsv"))
    rng = np.random.default_rng(99)
    sets = [rc.synthetic_reads(rng, int(rng.integers(100, 900)), int(rng.integers(3, 9)), 0.05, 0.02, 0.02)
            for _ in range(200)]
    params = Params()
    b = mp.Batch(params, sets)
    b.run(0)
    want = b.output_all(2)
    t = b.autotune()
    assert t.trials == 9 and t.warps_per_sm in (4, 5, 6, 7, 8) and t.giant_factor in (1.0, 1.5)
    assert t.giant_alone in (0, 1)
    assert b.output_all(2) == want
    b.run(0)
    assert b.output_all(2) == want
    assert b.tuning().trials >= 2  # runs replayed from the captured graph
    lines = open(tmp_path / "tune.tsv").read().splitlines()
    assert len(lines) == 1 and lines[0].split("\t")[1] == str(t.warps_per_sm)
    b2 = mp.Batch(params, sets)  # same size bucket: the cached setting applies
    tt = b2.tuning()
    assert tt.warps_per_sm == t.warps_per_sm and tt.giant_factor == t.giant_factor
    assert tt.giant_alone == t.giant_alone
    b2.run(0)
    assert b2.output_all(2) == want
    os.unlink(tmp_path / "tune.tsv")
