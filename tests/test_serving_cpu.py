"""The serving load generator's host-side accounting (dyng_b200/serving.py), on the CPU: the wait
a request spends behind its own graph's earlier requests, the per-decade latency split with and
without that wait, the summary line, and the Zipf target weights."""
import numpy as np

from dyng_b200 import serving as S


def _record(graph, changes, total_ms, submitted_s, service_ms=1.0, group=1, lane=0):
    """One per-request record in the field order of serving.RECORD."""
    r = {"graph": graph, "changes": changes, "total_ms": total_ms, "queued_ms": 0.1,
         "group_size": group, "service_ms": service_ms, "begin_ms": 0.05, "round_ms": 0.5,
         "copy_ms": 0.02, "submitted_s": submitted_s, "lane": lane}
    return tuple(r[k] for k in S.RECORD)


def test_graph_waits_follow_each_graphs_submission_order():
    # graph 0: submitted at 0 ms (5 ms in all) and at 1 ms (8 ms in all); the second could not
    # start before the first finished at 5 ms, so it waited 4 ms.  Graph 1 waits for nothing.
    # Records arrive in completion order, not submission order.
    done = [_record(1, 100, 2.0, 0.002), _record(0, 100, 5.0, 0.000),
            _record(0, 100, 8.0, 0.001)]
    waits = S.graph_waits(done)
    assert waits == [0.0, 0.0, 4.0]


def test_graph_waits_chain_over_several_requests():
    # three requests of one graph 1 ms apart, each 3 ms end to end: the finishes are at 3, 4 and
    # 5 ms, so the waits are 0, 3 - 1 = 2 and 4 - 2 = 2 ms
    done = [_record(0, 500, 3.0, 0.000), _record(0, 500, 3.0, 0.001),
            _record(0, 500, 3.0, 0.002)]
    assert S.graph_waits(done) == [0.0, 2.0, 2.0]


def test_by_size_splits_decades_and_removes_the_graph_wait():
    done = [_record(0, 150, 1.0, 0.0), _record(1, 5_000, 2.0, 0.0),
            _record(2, 50_000, 3.0, 0.0), _record(3, 2_000_000, 9.0, 0.0),
            _record(3, 120_000, 12.0, 0.001)]
    out = S.by_size(done)
    assert set(out) == {"100+", "1000+", "10000+", "100000+"}
    assert out["100+"]["n"] == 1 and out["100+"]["p50_ms"] == 1.0
    big = out["100000+"]
    assert big["n"] == 2
    # the 120k request waited 9 - 1 = 8 ms for the 2M request of its graph
    assert big["graph_wait_p99_ms"] > 7.0
    assert np.isclose(big["own_p50_ms"], np.percentile([9.0, 4.0], 50))


def test_summarize_reports_the_mix():
    done = [_record(i % 4, 1_000 * (i + 1), float(i + 1), i * 0.001, group=1 + i % 2)
            for i in range(100)]
    s = S.summarize(done, wall=2.0, rate=50)
    lat = np.arange(1, 101, dtype=float)
    assert s["requests"] == 100 and s["rate"] == 50
    assert np.isclose(s["p50_ms"], np.percentile(lat, 50))
    assert np.isclose(s["p99_ms"], np.percentile(lat, 99))
    assert np.isclose(s["p99_over_p50"], s["p99_ms"] / s["p50_ms"])
    assert np.isclose(s["changed_edges_per_s"], sum(1_000 * (i + 1) for i in range(100)) / 2.0)
    assert np.isclose(s["mean_group"], 1.5)
    assert set(s["parts_p50_ms"]) == {k for k, _ in S.PARTS}


def test_zipf_weights():
    w = S.zipf_weights(8)
    assert np.isclose(w.sum(), 1.0)
    assert np.all(np.diff(w) < 0)
    assert np.isclose(w[0] / w[1], 2 ** 1.1)
