"""The packing modes of the persistent kernel and long dependency chains, against the oracle.

  - cpp/tests/algorithms/sssp/sssp_cuda_test.cpp:555-620 (LargeWeightsUseTheDistanceOnlyFallback):
    on a 320 x 320 grid with weights 2 * 10^9 (every vertex has two tight in-neighbours) and with
    random weights up to 2^31 - 1, (n - 1) * max weight does not fit beside 17 parent bits, so the
    kernel keeps distances only and recovers the lowest-id tight parent after the search;
  - sssp_cuda_test.cpp:494-553 (PackingBoundaryOf47DistanceBits): n = 2^17 - 1 leaves 47 bits for
    distances; on the path 0 -> 1 -> ... -> n-1 with W = 2^30 + 2^14, (n - 1) * W still packs,
    but a back edge n-1 -> 1 forms the candidate n * W, which must be dropped, not packed (the
    pull, the push loop and compute each meet it);
  - a 2^20-vertex path: a million dependent near-far steps, most of them run by one block while
    the others wait at a grid barrier (compute, and an update that re-roots half of the path).
"""
import numpy as np
import pytest

import dyng_b200 as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _batch(ins_src=(), ins_dst=(), ins_w=(), del_src=(), del_dst=(), k=1):
    return D.EdgeBatch.from_arrays(ins_src, ins_dst, ins_w, del_src, del_dst, num_weights=k)


def _obatch(ins_src=(), ins_dst=(), ins_w=(), del_src=(), del_dst=(), k=1):
    return O.Batch(ins_src, ins_dst, ins_w, del_src, del_dst, k)


def _same(t, ot, label=""):
    np.testing.assert_array_equal(t.distances, ot.distances, err_msg=label)
    np.testing.assert_array_equal(t.parents, ot.parents, err_msg=label)


@pytest.mark.parametrize("objective", [0, 1])
def test_large_weights_use_the_distance_only_mode(objective):
    side = 320
    n = side * side
    rng = np.random.default_rng(20260927)
    v = np.arange(n)
    x, y = v % side, v // side
    right, down = v[x + 1 < side], v[y + 1 < side]
    src = np.concatenate([right, right + 1, down, down + side]).astype(np.int32)
    dst = np.concatenate([right + 1, right, down + side, down]).astype(np.int32)
    w = np.stack([np.full(src.size, 2_000_000_000), rng.integers(1, 2**31 - 1, src.size,
                                                                 endpoint=True)], axis=1)
    w = w.astype(np.int32).ravel()  # insertion-major, two weights per edge
    props = D.GraphProperties.mosp_compatible()
    g = D.Graph.from_edges(src, dst, w, n, props, num_weights=2)
    og = O.Graph.from_edges(n, src, dst, w, 2, O.mosp_props())
    t, cst = D.sssp.compute(g, 0, D.sssp.Options(objective=objective), stats=True)
    ot, _ = O.compute(og, 0, objective=objective, rule=1)
    assert not cst.packed_parents
    _same(t, ot, "compute")
    for rnd in range(3):
        # 1000 deletions of tree edges, 1000 insertions (weights 2e9 and random), as the reference
        parents = ot.parents
        vv = rng.integers(1, n, 1000)
        vv = vv[parents[vv] >= 0]
        a = rng.integers(0, n, 1000)
        c = rng.integers(0, n, 1000)
        keep = a != c
        a, c = a[keep], c[keep]
        iw = np.stack([np.full(a.size, 2_000_000_000),
                       rng.integers(1, 2**31 - 1, a.size, endpoint=True)], axis=1)
        iw = iw.astype(np.int32).ravel()
        b = (a.astype(np.int32), c.astype(np.int32), iw, parents[vv].astype(np.int32),
             vv.astype(np.int32))
        st = D.sssp.update(g, _batch(*b, k=2), t)
        ost, _ = O.update(og, _obatch(*b, k=2), ot)
        assert not st.packed_parents and not ost["packed_parents"]
        _same(t, ot, f"round {rnd}")
        assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])
        assert st.invalidated > 0


@pytest.mark.parametrize("scenario", ["pull", "push", "from-scratch"])
def test_packing_boundary_of_47_distance_bits(scenario):
    n = (1 << 17) - 1
    w = (1 << 30) + (1 << 14)
    back = scenario != "pull"
    src = list(range(n - 1)) + ([n - 1] if back else [])
    dst = list(range(1, n)) + ([1] if back else [])
    wts = [w] * len(src)
    props = D.GraphProperties.mosp_compatible()
    g = D.Graph.from_edges(src, dst, wts, n, props)
    og = O.Graph.from_edges(n, src, dst, wts, 1, O.mosp_props())
    t, cst = D.sssp.compute(g, 0, stats=True)
    ot, _ = O.compute(og, 0, rule=1)
    assert cst.packed_parents  # (n - 1) * W = 2^47 - 2^15 fits beside 17 parent bits
    _same(t, ot, "compute")
    assert t.distances[n - 1] == (n - 1) * w
    if scenario == "from-scratch":
        return
    ins = (n - 1, 1, w) if scenario == "pull" else (n - 2, n - 1, w - 1)
    st = D.sssp.update(g, _batch([ins[0]], [ins[1]], [ins[2]]), t)
    ost, _ = O.update(og, _obatch([ins[0]], [ins[1]], [ins[2]]), ot)
    assert st.packed_parents
    _same(t, ot, scenario)
    assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])
    assert t.distances[1] == w  # the candidate n * W over the back edge was dropped


def test_a_path_of_a_million_vertices():
    n = 1 << 20
    rng = np.random.default_rng(5)
    src = np.arange(n - 1, dtype=np.int32)
    dst = src + 1
    w = rng.integers(1, 100, n - 1, endpoint=True).astype(np.int32)
    g = D.Graph.from_edges(src, dst, w, n)
    og = O.Graph.from_edges(n, src, dst, w, 1)
    t, cst = D.sssp.compute(g, 0, stats=True)
    ot, _ = O.compute(og, 0, rule=1)
    _same(t, ot, "compute")
    assert cst.iterations >= n - 1  # one dependent step per vertex
    # cut the path after vertex 1 and hang its second half off the source: half of it is
    # re-rooted, the first half becomes unreachable
    mid = n // 2
    b = ([0], [mid], [7], [1], [2])
    st = D.sssp.update(g, _batch(*b), t)
    ost, _ = O.update(og, _obatch(*b), ot)
    _same(t, ot, "update")
    assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])
    assert st.invalidated == n - 2
