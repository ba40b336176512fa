"""The autotuner (clsparse_b200.autotune): table logic on CPU; on the GPU a
sweep whose every candidate shape is parity-checked, and the batched
lanes-per-row tuning."""
from __future__ import annotations

import numpy as np
import pytest

from clsparse_b200 import autotune, matgen


def test_features_and_lookup(tmp_path):
    rp_a, _, _ = matgen.poisson2d(64)
    rp_b, _, _ = matgen.irregular(20_000, n_dense=5, dense_len=8_000, seed=2)
    fa, fb = autotune.features(rp_a), autotune.features(rp_b)
    assert fa["rows"] == 4096 and abs(fa["mean_row"] - np.diff(rp_a.astype(np.int64)).mean()) < 1e-12
    t = autotune.TuningTable(device="test")
    assert t.lookup_shape(fa) == autotune.SHAPES_DEFAULT
    t.add_spmv(fa, (512, 1, 1, 128), 10.0, 12.0, "stencil")
    t.add_spmv(fb, (2048, 8, 4, 256), 20.0, 25.0, "irregular")
    assert t.lookup_shape(fa) == (512, 1, 1, 128)
    assert t.lookup_shape(fb) == (2048, 8, 4, 256)
    t.batched = [{"n_min": 500, "n_max": 2000, "lanes": 2}, {"n_min": 2000, "n_max": 50001, "lanes": 4}]
    np.testing.assert_array_equal(t.lanes_for([600, 1999, 2000, 40000, 100]), [2, 2, 4, 4, 0])
    p = tmp_path / "t.json"
    t.save(p)
    u = autotune.TuningTable.load(p)
    assert u.lookup_shape(fb) == (2048, 8, 4, 256) and u.batched == t.batched and u.device == "test"


def test_candidates_are_valid_shapes():
    for blk, mult, rfv, nt in autotune.CANDIDATES:
        assert blk in (512, 1024, 2048) and nt in (128, 256) and blk // 4 // nt >= 1
        assert mult >= 1 and rfv >= 1


@pytest.mark.gpu
def test_tune_spmv_checks_every_candidate(ctrl):
    rp, col, val = matgen.irregular(60_000, n_dense=4, dense_len=20_000, seed=5)
    cands = [(512, 1, 1, 128), (1024, 3, 4, 256), (2048, 8, 1, 128)]
    shape, us, dus, sweep = autotune.tune_spmv(ctrl, rp, col, val, candidates=cands, reps=5)
    assert [s for s, _ in sweep] == cands
    assert us <= dus and all(t > 0 for _, t in sweep)
    assert shape in cands or shape == autotune.SHAPES_DEFAULT


@pytest.mark.gpu
def test_tune_batched_lanes(ctrl):
    out = autotune.tune_batched_lanes(ctrl, classes=((200, 400), (400, 900)), per_class=8, lanes=(1, 4))
    assert [c["lanes"] for c in out] and all(c["lanes"] in (1, 4) for c in out)
