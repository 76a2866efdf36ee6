"""Failures made on the host, and what the library leaves behind (no GPU fault is made).

  - a grid barrier that never completes (a phantom block that never arrives, with a short
    test-only time limit): every block leaves the kernel and the call reports INTERNAL; in the
    batch applier before any change (graph and tree unchanged), in the sssp kernel after the
    batch was applied (the tree poisoned); the context keeps working either way;
  - a long loop run by one block while the others wait at a grid barrier outlives that limit
    without a timeout: the waiting blocks restart their limit whenever the working block shows
    progress;
  - a device without cooperative launch (sssp_cuda_test.cpp:106-150): calls that ask for the fused
    engine are refused before anything changes, automatic ones run the operators engine;
  - every device allocation of an update failed in turn (the sweep of the reference's
    tests/support/failing_allocator.hpp:18-143): the call reports OUT_OF_MEMORY and leaves the
    graph and the tree either unchanged or, after the batch was applied, the tree poisoned; the
    next calls give the oracle's results;
  - steady-state updates allocate nothing (sssp_cuda_test.cpp:657-700): once a stream of
    same-size batches has warmed the workspace, an update makes no device allocation unless the
    graph's own storage grows.
"""
import numpy as np
import pytest

import dyng_b200 as D
from dyng_b200.graph import device_allocations, fail_device_allocation
from oracle import oracle as O
from tests.helpers import random_batch, random_graph

pytestmark = pytest.mark.gpu


def _batch(b, k=1):
    return D.EdgeBatch.from_arrays(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"],
                                   b["del_dst"], num_weights=k)


def _obatch(b, k=1):
    return O.Batch(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"], b["del_dst"], k)


def _case(seed=3, n=3000):
    rng = np.random.default_rng(seed)
    n, s, d, w = random_graph(rng, "sparse", n)
    return rng, n, s, d, w


def test_a_barrier_of_the_applier_that_never_completes_changes_nothing():
    # the batch applier's first grid barrier comes before any change: its timeout leaves the
    # graph and the tree as they were (strong guarantee), and the same update then succeeds
    rng, n, s, d, w = _case()
    res = D.Resources(0)
    g = D.Graph.from_edges(s, d, w, n, resources=res)
    og = O.Graph.from_edges(n, s, d, w, 1)
    t = D.sssp.compute(g, 0)
    ot, _ = O.compute(og, 0, rule=1)
    d0, p0, m0 = t.distances, t.parents, g.num_edges()
    b = random_batch(rng, n, s, d, 400, tree_parents=ot.parents)
    res.set_test_hooks(barrier_timeout_ns=2_000_000, barrier_extra_arrivals=1, barrier_kernel=1)
    try:
        with pytest.raises(D.InternalError, match="timed out before the batch was applied"):
            D.sssp.update(g, _batch(b), t)
    finally:
        res.set_test_hooks()
    assert g.version() == 0 and g.num_edges() == m0 and not t.poisoned
    np.testing.assert_array_equal(t.distances, d0)
    np.testing.assert_array_equal(t.parents, p0)
    D.sssp.update(g, _batch(b), t)
    O.update(og, _obatch(b), ot)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)


def test_a_barrier_of_the_sssp_kernel_that_never_completes_times_out_and_poisons():
    rng, n, s, d, w = _case()
    res = D.Resources(0)
    g = D.Graph.from_edges(s, d, w, n, resources=res)
    og = O.Graph.from_edges(n, s, d, w, 1)
    t = D.sssp.compute(g, 0)
    ot, _ = O.compute(og, 0, rule=1)
    b = random_batch(rng, n, s, d, 400, tree_parents=ot.parents)
    res.set_test_hooks(barrier_timeout_ns=2_000_000, barrier_extra_arrivals=1, barrier_kernel=2)
    try:
        with pytest.raises(D.InternalError, match="timed out"):
            D.sssp.update(g, _batch(b), t)
        assert g.version() == 1  # the batch was applied before the sssp kernel ran
        with pytest.raises(D.StaleResultError):
            t.distances
        with pytest.raises(D.InternalError, match="timed out"):
            D.sssp.compute(g, 0)
    finally:
        res.set_test_hooks()
    # the context is usable again: a fresh tree of the applied graph equals the oracle's
    O.update(og, _obatch(b), ot)
    fresh = D.sssp.compute(g, 0)
    np.testing.assert_array_equal(fresh.distances, ot.distances)
    np.testing.assert_array_equal(fresh.parents, ot.parents)


def test_progress_keeps_a_long_single_block_loop_alive():
    # a path of 2^18 vertices: the near-far loop runs ~262k dependent steps on block 0 alone,
    # far longer than the 20 ms limit the other blocks wait with at their grid barrier
    n = 1 << 18
    src = np.arange(n - 1, dtype=np.int32)
    w = np.full(n - 1, 3, np.int32)
    res = D.Resources(0)
    g = D.Graph.from_edges(src, src + 1, w, n, resources=res)
    res.set_test_hooks(barrier_timeout_ns=20_000_000)
    try:
        t, st = D.sssp.compute(g, 0, stats=True)
    finally:
        res.set_test_hooks()
    assert st.sssp_ms > 40.0, st.sssp_ms  # the loop outlived the limit twice over
    np.testing.assert_array_equal(t.distances, 3 * np.arange(n, dtype=np.int64))


def test_without_cooperative_launch_the_fused_engine_is_refused():
    # cuda_engine="fused" on a device without cooperative launch is refused before anything
    # changes; "automatic" then runs the operators engine
    rng, n, s, d, w = _case(5)
    res = D.Resources(0)
    g = D.Graph.from_edges(s, d, w, n, resources=res)
    fused = D.sssp.Options(cuda_engine="fused")
    t = D.sssp.compute(g, 0, fused)
    d0, p0 = t.distances, t.parents
    b = random_batch(rng, n, s, d, 300, tree_parents=p0)
    m0 = g.num_edges()  # duplicate pairs of the random edge list were merged
    res.set_test_hooks(no_cooperative_launch=True)
    try:
        with pytest.raises(D.NotSupportedError, match="cooperative launch"):
            D.sssp.compute(g, 0, fused)
        with pytest.raises(D.NotSupportedError, match="cooperative launch"):
            D.sssp.update(g, _batch(b), t)
        assert g.version() == 0 and g.num_edges() == m0  # refused before the batch was applied
        np.testing.assert_array_equal(t.distances, d0)
        np.testing.assert_array_equal(t.parents, p0)
        t.set_options(D.sssp.Options())
        og = O.Graph.from_edges(n, s, d, w, 1)
        ot, _ = O.compute(og, 0, rule=1)
        st = D.sssp.update(g, _batch(b), t)
        assert st.engine_used == "operators"
    finally:
        res.set_test_hooks()
    O.update(og, _obatch(b), ot)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)


def test_each_failed_allocation_of_an_update_leaves_a_consistent_state():
    rng, n, s, d, w = _case(11, 2000)
    # a batch far larger than the slack rows (the arenas and the edge index grow) on a fresh
    # context (the workspace is sized by this call)
    b = random_batch(rng, n, s, d, 40_000)
    og = O.Graph.from_edges(n, s, d, w, 1)
    ot, _ = O.compute(og, 0, rule=1)
    d0, p0 = ot.distances, ot.parents
    O.update(og, _obatch(b), ot)

    def fresh():
        res = D.Resources(0)
        g = D.Graph.from_edges(s, d, w, n, resources=res)
        return res, g, D.sssp.compute(g, 0)

    res, g, t = fresh()
    m0 = g.num_edges()  # duplicate pairs of the random edge list were merged
    a0 = device_allocations()
    D.sssp.update(g, _batch(b), t)
    count = device_allocations() - a0
    assert count > 0
    np.testing.assert_array_equal(t.distances, ot.distances)
    failed = 0
    for k in range(1, count + 1):
        res, g, t = fresh()
        fail_device_allocation(k)
        try:
            D.sssp.update(g, _batch(b), t)
            raised = False
        except D.OutOfMemoryError:
            raised = True
        finally:
            fail_device_allocation(0)
        if not raised:  # an allocation skipped on this path: the update completed
            np.testing.assert_array_equal(t.distances, ot.distances, err_msg=f"alloc {k}")
            continue
        failed += 1
        if g.version() == 0:
            # before the commit: strong guarantee, graph and tree unchanged, the retry succeeds
            assert g.num_edges() == m0, k
            np.testing.assert_array_equal(t.distances, d0, err_msg=f"alloc {k}")
            np.testing.assert_array_equal(t.parents, p0, err_msg=f"alloc {k}")
            D.sssp.update(g, _batch(b), t)
            np.testing.assert_array_equal(t.distances, ot.distances, err_msg=f"alloc {k}")
            np.testing.assert_array_equal(t.parents, ot.parents, err_msg=f"alloc {k}")
        else:
            # after the commit: the tree is poisoned, the graph holds the batch
            assert g.version() == 1 and t.poisoned, k
            fresh_t = D.sssp.compute(g, 0)
            np.testing.assert_array_equal(fresh_t.distances, ot.distances, err_msg=f"alloc {k}")
        csr = g.to_csr()
        want = og.to_csr()
        np.testing.assert_array_equal(csr.col_ind, want["col"], err_msg=f"alloc {k}")
        np.testing.assert_array_equal(csr.weights.reshape(-1), want["w"].reshape(-1))
    assert failed >= count // 2, (failed, count)


def test_steady_state_updates_allocate_nothing():
    rng = np.random.default_rng(7)
    n, k = 2000, 3
    s = rng.integers(0, n, 8 * n).astype(np.int32)
    d = rng.integers(0, n, 8 * n).astype(np.int32)
    w = rng.integers(1, 100, 8 * n * k, endpoint=True).astype(np.int32)
    res = D.Resources(0)
    g = D.Graph.from_edges(s, d, w, n, D.GraphProperties.mosp_compatible(), num_weights=k,
                           resources=res)
    trees = [D.sssp.compute(g, 0, D.sssp.Options(objective=j)) for j in range(k)]
    quiet = 0
    for rnd in range(8):
        # deletions of existing edges and insertions of new pairs: the same sizes every batch
        csr = g.to_csr()
        rows = rng.integers(0, n, 100)
        has = csr.row_ptr[rows] < csr.row_ptr[rows + 1]
        du = rows[has].astype(np.int32)
        dv = csr.col_ind[csr.row_ptr[du]].astype(np.int32)
        iu = rng.integers(0, n, 100).astype(np.int32)
        iv = rng.integers(0, n, 100).astype(np.int32)
        iw = rng.integers(1, 100, 100 * k, endpoint=True).astype(np.int32)
        st0 = g.storage()
        a0 = device_allocations()
        D.sssp.update_each(g, D.EdgeBatch.from_arrays(iu, iv, iw, du, dv, num_weights=k), trees)
        made = device_allocations() - a0
        st1 = g.storage()
        grew = any(st1[key] != st0[key] for key in ("index_builds", "arena_growths", "compactions"))
        if rnd >= 2 and not grew:
            assert made == 0, (rnd, made)
            quiet += 1
    assert quiet >= 3
