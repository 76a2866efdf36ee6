"""The benchmark's synthetic workloads (dyng_b200/generators.py) have the shapes they are quoted
with, on the CPU: R-MAT with edge factor 16 and weights in [1, 1000] (the numpy and torch paths
identical), batches of 75 % uniform insertions and 25 % deletions of which half are tree edges
and the rest live edges, and the grid's near-source churn (half deletions near the source, the
previous batch's near deletions inserted back)."""
import numpy as np
import pytest

from dyng_b200 import generators as G
from oracle import oracle as O


def test_rmat_shape():
    e = G.rmat(14, 16, w_max=1000, seed=1)
    n, m = e.num_vertices, e.src.size
    assert n == 1 << 14
    assert 12 * n < m <= 16 * n  # edge factor 16 less the dropped self-loops and duplicates
    assert e.weights.min() >= 1 and e.weights.max() <= 1000
    assert np.all(e.src != e.dst)
    assert e.src.min() >= 0 and e.dst.max() < n
    deg = np.bincount(e.src, minlength=n)
    assert deg.max() > 20 * deg.mean()  # R-MAT's skew: hubs far above the mean degree


def test_rmat_numpy_and_torch_paths_agree():
    pytest.importorskip("torch")
    a = G.rmat(12, 16, w_max=1000, seed=3)
    b = G.rmat(12, 16, w_max=1000, seed=3, device="cpu")
    assert np.array_equal(a.src, b.src) and np.array_equal(a.dst, b.dst)
    assert np.array_equal(a.weights, b.weights)


def test_batch_stream_mix():
    e = G.rmat(12, 16, w_max=1000, seed=2)
    rp, col, w = e.csr()
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    ot, _ = O.compute(og, 0, rule=1)
    stream = G.BatchStream(e, seed=7)
    base = set(zip(e.src.tolist(), e.dst.tolist()))
    for _ in range(3):
        b = stream.next(4000, 0.75, 0.5, parents=ot.parents)
        assert b.size == 4000 and b.insert_src.size == 3000 and b.delete_src.size == 1000
        assert b.insert_weights.min() >= 1 and b.insert_weights.max() <= 1000
        assert b.insert_src.max() < e.num_vertices and b.insert_dst.max() < e.num_vertices
        # the first half of the deletions are tree edges parent[v] -> v, distinct heads
        tree_s, tree_d = b.delete_src[:500], b.delete_dst[:500]
        assert np.array_equal(ot.parents[tree_d], tree_s)
        assert np.unique(tree_d).size == 500
        # the rest are edges of the base graph
        assert all(p in base for p in zip(b.delete_src[500:].tolist(),
                                          b.delete_dst[500:].tolist()))
        O.update(og, O.Batch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                             b.delete_dst), ot)


def test_uniform_deletions_come_from_live_edges_only():
    e = G.rmat(10, 8, w_max=100, seed=4)
    stream = G.BatchStream(e, seed=1)
    deleted = set()
    for _ in range(5):
        b = stream.next(600, 0.0, 0.0)  # deletions only, uniform over the live base edges
        pairs = set(zip(b.delete_src.tolist(), b.delete_dst.tolist()))
        assert not (pairs & deleted)
        deleted |= pairs


def test_near_source_churn():
    side = 64
    source = (side // 2) * side + side // 2
    e = G.grid(side, seed=1)
    churn = G.NearSourceChurn(G.BatchStream(e, seed=7), side, source, hops=8)
    stream = churn.stream
    b1 = churn.next(400)
    assert b1.insert_src.size == 200 and b1.delete_src.size == 200
    # the first deletions are near edges (at most a quarter of those alive), listed for return
    near_picked = churn.back.copy()
    k = near_picked.size
    assert 0 < k <= 200
    assert np.array_equal(b1.delete_src[:k], stream.src[near_picked])
    cx, cy = source % side, source // side
    src = stream.src[near_picked].astype(np.int64)
    assert np.all(np.abs(src % side - cx) + np.abs(src // side - cy) <= 8)
    b2 = churn.next(400)
    # the previous batch's near deletions are inserted back first
    assert np.array_equal(b2.insert_src[:k], stream.src[near_picked])
    assert np.array_equal(b2.insert_dst[:k], stream.dst[near_picked])
    assert b2.insert_weights.min() >= 1 and b2.insert_weights.max() <= 10000
