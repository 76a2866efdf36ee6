"""The learned scheduler's host side: the class tables, the numpy restatement of the inference
arithmetic, and (on the committed traces) the gain of the committed weights over the fixed
heuristic on batches held out of training."""
import os

import numpy as np
import pytest

from dyng_b200 import scheduler as S


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=10000).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 10000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.0078125, 1.01171875, 3.0e38],
                                 np.float32)]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(S.bf16_round(x), want)


def test_class_tables():
    assert len(S.all_settings()) == 96
    assert S.width_for(2, 1000) == 1000
    assert S.width_for(3, 1000) == 4000
    assert S.width_for(0, 1000) == 62 and S.width_for(1, 1000) == 250
    assert S.width_for(0, 3) == 1  # never below 1
    assert S.width_for(7, 1 << 39) == 1 << 40  # clamped
    assert S.grid_for(2, 592) == 0 and S.grid_for(1, 592) == 296 and S.grid_for(0, 592) == 148
    sc = S.schedule_for((5, 3, 1), 100, 600)
    assert (sc.delta, sc.invalidation, sc.small_frontier, sc.grid_blocks) == (6400, 1, -1, 300)
    assert S.schedule_for(S.DEFAULT_CLASSES, 100, 600).delta == 100


def test_reference_forward_is_the_mlp():
    rng = np.random.default_rng(1)
    params = (rng.normal(size=5967) * 0.2).astype(np.float32)
    x = rng.normal(size=(50, 12)).astype(np.float32)
    mean = np.zeros(12, np.float32)
    scale = np.ones(12, np.float32)
    got = S.reference_forward(params, mean, scale, x)
    p = S.unflatten(params.astype(np.float64))
    h = np.maximum(x @ p["w1"].T + p["b1"], 0)
    h = np.maximum(h @ p["w2"].T + p["b2"], 0)
    lo = h @ p["w3"].T + p["b3"]
    # bf16 weights and activations: within a few bf16 ulps of the float64 network
    assert np.allclose(got, lo, rtol=0.05, atol=0.05 * np.abs(lo).max())
    cls = S.classes_of(got)
    assert cls.shape == (50, 3)
    assert (cls[:, 0] < 8).all() and (cls[:, 1] < 4).all() and (cls[:, 2] < 3).all()


TRACES = os.path.join(S.DATA_DIR, "scheduler_traces.npz")


@pytest.mark.skipif(not os.path.exists(TRACES), reason="no recorded traces")
def test_committed_weights_beat_the_heuristic_on_heldout_traces():
    with np.load(TRACES) as z:
        traces = {k: z[k] for k in z.files}
    times = traces["times"]
    assert times.shape[1] == 96 and (times > 0).all()
    with np.load(S.PRETRAINED) as z:
        p, m, s = z["params"], z["feature_mean"], z["feature_scale"]
        lo, hi = (z["feature_lo"], z["feature_hi"]) if "feature_lo" in z.files else (None, None)
    pred = S.within_range(S.classes_of(S.reference_forward(p, m, s, traces["features"])),
                          traces["features"], lo, hi)
    hold = S.holdout_mask(traces)
    report = S.evaluate(pred, traces, hold)
    assert report["batches"] >= 30
    # the learned schedules are never slower in total than the fixed heuristic on unseen batches
    assert report["learned_ms"] <= report["default_ms"]


def test_outside_the_trained_range_the_plain_schedule_runs():
    x = np.zeros((3, 12), np.float32)
    x[1, 5] = 30.0   # a graph far larger than any in training
    x[2, 0] = -5.0
    lo, hi = S.feature_range(np.zeros((4, 12)) + np.arange(4)[:, None])
    got = S.within_range([[6, 1, 2]] * 3, x, lo, hi)
    assert got.tolist() == [[6, 1, 2], list(S.DEFAULT_CLASSES), list(S.DEFAULT_CLASSES)]
    assert S.within_range([[6, 1, 2]], x[:1], None, None).tolist() == [[6, 1, 2]]


def test_merging_trace_sets_renumbers_workloads():
    def part(names, rows):
        return {"workload": np.arange(rows) % len(names), "size": np.ones(rows),
                "features": np.zeros((rows, 12)), "times": np.ones((rows, 96)),
                "settings": np.asarray(S.all_settings(), np.int32),
                "workload_names": np.asarray(names)}
    m = S.merge_traces([part(["a", "b"], 4), part(["c"], 2)])
    assert m["workload"].tolist() == [0, 1, 0, 1, 2, 2]
    assert m["workload_names"].tolist() == ["a", "b", "c"] and m["times"].shape == (6, 96)
