"""Pins the CPU oracle against the reference's golden fixtures and hand cases (CPU only).

The oracle (oracle/sssp_oracle.c) is the checker of the CUDA path; these tests establish that it
reproduces the reference's bytes before anything is compared against it:
  - cpp/tests/algorithms/sssp/sssp_fixture_test.cpp:110-190: compute() == the initial trees,
    update() from the initial trees (imported without canonicalisation) == the updated trees,
    `invalidated` == the recorded counter, for all 34 cases and every objective;
  - cpp/tests/data/mosp_graph_io/*/applied: the applied CSR, its transpose and the
    weight-increase mask of apply_batch_host;
  - the README quickstart and hand cases of cpp/tests/algorithms/sssp/sssp_test.cpp:74-330;
  - cpp/tests/data/mosp_combined: mosp's finalize step (the combined graph of the K updated
    trees under the case's preferences, its tree and the path costs over every weight column)
    equals the combined files of all 8 cases (python/tests/test_cli.py:686-723 replays them);
  - hand cases of cpp/tests/algorithms/mosp/mosp_test.cpp:249-280.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import INF, combined_case, fixture_case


def _cases(z):
    return [str(c) for c in z["cases"]]


def test_fixture_count(fixtures):
    assert len(_cases(fixtures)) == 34


@pytest.mark.parametrize("rule", [0, 1])
def test_fixtures_compute_and_update(fixtures, rule):
    comparisons = 0
    for name in _cases(fixtures):
        c = fixture_case(fixtures, name)
        for k in range(c["k"]):
            g = O.Graph.from_csr(c["row_ptr"], c["col"], c["w"], c["k"], O.mosp_props())
            t, _ = O.compute(g, 0, objective=k, rule=rule)
            np.testing.assert_array_equal(t.distances, c["init_d"][k], err_msg=f"{name} k{k}")
            np.testing.assert_array_equal(t.parents, c["init_p"][k], err_msg=f"{name} k{k}")
            t = O.from_arrays(g, 0, c["init_d"][k], c["init_p"][k], canonicalize=False,
                              objective=k, rule=rule)
            st, _ = O.update(g, O.Batch(c["ins_src"], c["ins_dst"], c["ins_w"], c["del_src"],
                                        c["del_dst"], c["k"]), t)
            np.testing.assert_array_equal(t.distances, c["upd_d"][k], err_msg=f"{name} k{k}")
            np.testing.assert_array_equal(t.parents, c["upd_p"][k], err_msg=f"{name} k{k}")
            assert st["invalidated"] == c["invalidated"][k], name
            comparisons += 1
    assert comparisons > 34


def test_fixtures_applied_csr(fixtures):
    checked = 0
    for name in _cases(fixtures):
        c = fixture_case(fixtures, name)
        if "applied_row_ptr" not in c:
            continue
        g = O.Graph.from_csr(c["row_ptr"], c["col"], c["w"], c["k"], O.mosp_props())
        g.apply(O.Batch(c["ins_src"], c["ins_dst"], c["ins_w"], c["del_src"], c["del_dst"],
                        c["k"]))
        csr = g.to_csr()
        np.testing.assert_array_equal(csr["row_ptr"], c["applied_row_ptr"], err_msg=name)
        np.testing.assert_array_equal(csr["col"], c["applied_col"], err_msg=name)
        np.testing.assert_array_equal(csr["w"], c["applied_w"], err_msg=name)
        np.testing.assert_array_equal(csr["in_row_ptr"], c["applied_in_row_ptr"], err_msg=name)
        np.testing.assert_array_equal(csr["in_col"], c["applied_in_col"], err_msg=name)
        np.testing.assert_array_equal(csr["in_w"], c["applied_in_w"], err_msg=name)
        np.testing.assert_array_equal(g.delta()["weight_increased"], c["applied_increase"],
                                      err_msg=name)
        checked += 1
    assert checked == 27


def _g(n, edges, props=None, k=1):
    src = [e[0] for e in edges]
    dst = [e[1] for e in edges]
    w = [x for e in edges for x in e[2:]]
    return O.Graph.from_edges(n, src, dst, w, k, props or O.mosp_props())


def test_readme_quickstart():
    # README.md:73-97: 0 4 1 2 | invalidated 2
    g = _g(4, [(0, 1, 4), (0, 2, 1), (2, 1, 2), (1, 3, 1)], O.default_props())
    t, _ = O.compute(g, 0)
    assert t.distances.tolist() == [0, 3, 1, 4]
    st, _ = O.update(g, O.Batch([2], [3], [1], [2], [1]), t)
    assert t.distances.tolist() == [0, 4, 1, 2]
    assert st["invalidated"] == 2


def test_canonical_tree_and_tie_parent():
    # sssp_test.cpp:74-99
    g = _g(5, [(0, 1, 5), (0, 2, 1), (2, 3, 1), (1, 4, 2), (3, 4, 2)])
    t, _ = O.compute(g, 0)
    assert t.distances.tolist() == [0, 5, 1, 2, 4]
    assert t.parents.tolist() == [-1, 0, 0, 2, 3]
    st, sm = O.update(g, O.Batch([2], [1], [1]), t)
    assert t.distances.tolist() == [0, 2, 1, 2, 4]
    assert t.parents.tolist() == [-1, 2, 0, 2, 1]
    assert st["invalidated"] == 0 and st["affected"] == 2
    assert sm["inserted_edges"] == 1


def test_no_count_to_infinity():
    # sssp_test.cpp:101-112
    g = _g(4, [(0, 1, 1), (0, 3, 50), (1, 2, 1), (2, 1, 1), (3, 1, 50)])
    t, _ = O.compute(g, 0)
    st, _ = O.update(g, O.Batch(delete_src=[0], delete_dst=[1]), t)
    assert t.distances.tolist() == [0, 100, 101, 50]
    assert t.parents.tolist() == [-1, 3, 1, 0]
    assert st["invalidated"] == 2 and st["affected"] == 2


def test_delete_all_then_reinsert():
    # sssp_test.cpp:114-135
    g = _g(5, [(0, 1, 3), (1, 2, 4), (0, 3, 2), (3, 4, 7)])
    t, _ = O.compute(g, 0)
    st, _ = O.update(g, O.Batch(delete_src=[0, 1, 0, 3], delete_dst=[1, 2, 3, 4]), t)
    assert g.m == 0
    assert t.distances.tolist() == [0, INF, INF, INF, INF]
    assert t.parents.tolist() == [-1] * 5
    assert st["invalidated"] == 4 and st["affected"] == 4
    O.update(g, O.Batch([0, 4], [4, 2], [9, 1]), t)
    assert t.distances.tolist() == [0, INF, 10, INF, 9]
    assert t.parents.tolist() == [-1, -1, 4, -1, 0]


def test_weight_increase_on_tree_edge():
    # sssp_test.cpp:154-166
    g = _g(3, [(0, 1, 1), (1, 2, 1), (0, 2, 5)])
    t, _ = O.compute(g, 0)
    st, sm = O.update(g, O.Batch([0], [1], [10]), t)
    assert st["invalidated"] == 2 and sm["updated_edges"] == 1
    assert t.distances.tolist() == [0, 10, 5]
    assert t.parents.tolist() == [-1, 0, 0]


def test_parallel_edges_and_self_loops():
    # sssp_test.cpp:168-186
    g = _g(3, [(0, 1, 7), (0, 1, 3), (1, 1, 1), (1, 2, 1)])
    t, _ = O.compute(g, 0)
    assert t.distances.tolist() == [0, 3, 4]
    st, _ = O.update(g, O.Batch(delete_src=[0], delete_dst=[1]), t)
    assert st["invalidated"] == 2
    assert t.distances.tolist() == [0, 3, 4]
    O.update(g, O.Batch(delete_src=[0], delete_dst=[1]), t)
    assert t.distances.tolist() == [0, INF, INF]


def test_vertex_growth():
    # sssp_test.cpp:188-199
    g = _g(3, [(0, 1, 2), (1, 2, 2)], O.default_props())
    t, _ = O.compute(g, 0)
    st, sm = O.update(g, O.Batch([2, 5], [5, 3], [1, 4]), t)
    assert g.n == 6 and sm["num_vertices_after"] == 6
    assert t.distances.tolist() == [0, 2, 4, 9, INF, 5]
    assert t.parents.tolist() == [-1, 0, 1, 5, -1, 2]


def test_undirected():
    # sssp_test.cpp:201-212
    g = _g(4, [(0, 1, 1), (1, 2, 1), (2, 3, 1)], O.mosp_props(directed=0))
    t, _ = O.compute(g, 3)
    assert t.distances.tolist() == [3, 2, 1, 0]
    O.update(g, O.Batch([0], [3], [5], [1], [2]), t)
    assert t.distances.tolist() == [5, 6, 1, 0]
    assert t.parents.tolist() == [3, 0, 3, -1]


def test_multi_objective_column():
    # sssp_test.cpp:214-236
    g = _g(3, [(0, 1, 1, 10), (1, 2, 1, 10), (0, 2, 5, 1)], k=2)
    t1, _ = O.compute(g, 0, objective=1)
    assert t1.distances.tolist() == [0, 10, 1]
    st, _ = O.update(g, O.Batch([0], [2], [5, 30], num_weights=2), t1)
    assert st["invalidated"] == 1
    assert t1.distances.tolist() == [0, 10, 20]
    assert t1.parents.tolist() == [-1, 0, 1]


def test_non_canonical_tree_keeps_tie_parents():
    # sssp_test.cpp:313-333
    g = _g(5, [(0, 1, 1), (0, 2, 1), (1, 3, 1), (2, 3, 1), (0, 4, 5), (4, 3, 1)])
    t = O.from_arrays(g, 0, [0, 1, 1, 2, 5], [-1, 0, 0, 2, 0], canonicalize=False)
    st, _ = O.update(g, O.Batch([0], [4], [1]), t)
    assert t.distances.tolist() == [0, 1, 1, 2, 1]
    assert t.parents.tolist() == [-1, 0, 0, 2, 0]
    assert st["affected"] == 1


@pytest.mark.parametrize("side,dup", [(272, False), (64, True)])
def test_distance_only_mode(side, dup):
    # sssp_test.cpp:238-311: weights 2e9 so (n-1)*w does not fit next to the parent bits; the
    # parents are recovered with the lowest-id rule.  Scaled down for the second case.
    w = 2_000_000_000
    v = np.arange(side * side)
    x, y = v % side, v // side
    r = v[x + 1 < side]
    d = v[y + 1 < side]
    src = np.concatenate([r, d] + ([r + 1, d + side] if dup else []))
    dst = np.concatenate([r + 1, d + side] + ([r, d] if dup else []))
    g = O.Graph.from_edges(side * side, src, dst, np.full(src.size, w), 1, O.mosp_props())
    n = side * side
    if not O.packs_parents(n, w, 0):
        t, st = O.compute(g, 0)
        assert st["packed_parents"] == 0
        del_src = list(range(0, n - 1, 97))
        st, _ = O.update(g, O.Batch([0], [n - 1], [w], del_src, [s + 1 for s in del_src]), t)
        fresh, _ = O.compute(g, 0)
        np.testing.assert_array_equal(t.distances, fresh.distances)
        np.testing.assert_array_equal(t.parents, fresh.parents)


def test_invalid_batches_raise():
    g = _g(3, [(0, 1, 2), (1, 2, 2)], O.default_props())
    t, _ = O.compute(g, 0)
    with pytest.raises(O.OracleError):
        O.update(g, O.Batch([0], [1], [0]), t)  # weight below 1
    with pytest.raises(O.OracleError):
        O.update(g, O.Batch([-1], [1], [3]), t)  # negative id
    assert g.n == 3 and g.m == 2  # nothing changed


def test_packing_rules():
    # cuda.cu:225-234 vs sssp.cpp:153-165 (the packing window)
    n = 1 << 17
    bits = 18
    maxd = ((2**64 - 1) >> bits) - 1
    w = maxd // (n - 1)
    assert O.packs_parents(n, w, 1)
    assert not O.packs_parents(n, w, 0)
    assert O.default_delta(100, 10, 1000) == 32


def oracle_mosp_update(c):
    """The K trees of a combined case updated by its batch (each on its own copy of the graph:
    the batch is applied once per copy), the updated graph, and mosp's finalize step."""
    k, kg = c["k"], c["kg"]
    trees, g = [], None
    for j in range(k):
        g = O.Graph.from_csr(c["row_ptr"], c["col"], c["w"], kg, O.mosp_props())
        t = O.from_arrays(g, 0, c["init_d"][j], c["init_p"][j], canonicalize=False, objective=j,
                          rule=1)
        O.update(g, O.Batch(c["ins_src"], c["ins_dst"], c["ins_w"], c["del_src"], c["del_dst"],
                            kg), t)
        trees.append(t)
    return trees, g, O.mosp_finalize(g, 0, [t.parents for t in trees], c["pref"], kg)


def test_combined_fixtures(combined_fixtures):
    names = [str(x) for x in combined_fixtures["cases"]]
    assert len(names) == 8
    for name in names:
        c = combined_case(combined_fixtures, name)
        _, _, m = oracle_mosp_update(c)
        np.testing.assert_array_equal(m.distances, c["combined_d"], err_msg=name)
        np.testing.assert_array_equal(m.parents, c["combined_p"], err_msg=name)
        np.testing.assert_array_equal(m.costs, c["costs"], err_msg=name)


def test_mosp_default_preferences_weigh_an_edge_by_its_trees():
    # mosp_test.cpp:249-269: 0->1->3 is best for objective 0, 0->2->3 for objective 1
    g = O.Graph.from_edges(4, [0, 0, 1, 2], [1, 2, 3, 3], [1, 5, 5, 1, 1, 5, 5, 1], 2)
    parents = [O.compute(g, 0, objective=j, rule=1)[0].parents for j in range(2)]
    m = O.mosp_finalize(g, 0, parents)
    assert m.scale == 1 and m.distances.tolist() == [0, 1, 1, 3]
    assert m.parents.tolist() == [-1, 0, 0, 1] and m.costs[3].tolist() == [2, 10]
    m = O.mosp_finalize(g, 0, parents, [2, 1])
    assert m.scale == 2 and m.distances.tolist() == [0, 3, 3, 7]
    assert m.parents.tolist() == [-1, 0, 0, 2] and m.costs[3].tolist() == [10, 2]


def test_mosp_unreachable_vertices_have_no_parent_and_infinite_costs():
    # mosp_test.cpp:271-279
    g = O.Graph.from_edges(4, [0, 2], [1, 3], [1, 1, 1, 1], 2)
    parents = [O.compute(g, 0, objective=j, rule=1)[0].parents for j in range(2)]
    m = O.mosp_finalize(g, 0, parents)
    assert m.distances.tolist() == [0, 1, INF, INF] and m.parents.tolist() == [-1, 0, -1, -1]
    assert m.costs[2].tolist() == [INF, INF] and m.costs[0].tolist() == [0, 0]


THESIS_EDGES = [(0, 1, 2, 1, 5), (0, 2, 4, 1, 1), (1, 3, 2, 4, 2), (2, 1, 10, 15, 2),
                (2, 3, 5, 16, 3), (3, 4, 1, 1, 1), (4, 1, 4, 3, 2), (4, 5, 1, 2, 2),
                (4, 6, 5, 6, 2), (5, 6, 1, 1, 1)]


def test_mosp_thesis_worked_example():
    # mosp_test.cpp:155-211: compute, the thesis' batch, then the MOSP path to u7 and its costs
    # under two preference vectors
    for pref, path, cost in (([4, 1, 4], [6, 5, 1, 0], [15, 3, 20]),
                             ([4, 4, 1], [6, 4, 3, 2, 0], [15, 24, 7])):
        trees = []
        for j in range(3):
            g = O.Graph.from_edges(7, [e[0] for e in THESIS_EDGES], [e[1] for e in THESIS_EDGES],
                                   [x for e in THESIS_EDGES for x in e[2:]], 3, O.mosp_props())
            t, _ = O.compute(g, 0, objective=j, rule=1)
            O.update(g, O.Batch([3, 1], [5, 5], [10, 2, 12, 12, 1, 14], [1, 4], [3, 1], 3), t)
            trees.append(t)
        assert [t.parents.tolist() for t in trees] == [
            [-1, 0, 0, 2, 3, 4, 5], [-1, 0, 0, 2, 3, 1, 5], [-1, 2, 0, 2, 3, 4, 4]]
        m = O.mosp_finalize(g, 0, [t.parents for t in trees], pref)
        walk = [6]
        while m.parents[walk[-1]] >= 0:
            walk.append(int(m.parents[walk[-1]]))
        assert m.scale == 4 and walk == path and m.costs[6].tolist() == cost


def test_parallel_apply_equals_sequential():
    # the CPU-baseline timing runs the oracle's CSR assembly and transposition on several
    # threads: graphs (out and in rows, weights) and repaired trees equal the sequential run
    from dyng_b200 import generators as G
    e = G.rmat(12, 16, w_max=100, seed=4)
    rp, col, w = e.csr()
    out = {}
    try:
        for threads in (1, 4):
            O.set_threads(threads)
            g = O.Graph.from_csr(rp, col, w, 1, O.default_props())
            t, _ = O.compute(g, 0, rule=1)
            stream = G.BatchStream(e, seed=5)
            for _ in range(3):
                b = stream.next(3000, 0.75, 0.5, parents=t.parents)
                O.update(g, O.Batch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                    b.delete_dst), t)
            out[threads] = (g.to_csr(), t.distances.copy(), t.parents.copy())
    finally:
        O.set_threads(1)
    a, b = out[1], out[4]
    for key in a[0]:
        np.testing.assert_array_equal(a[0][key], b[0][key], err_msg=key)
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])


@pytest.mark.parametrize("case", ["sparse", "multigraph-k2", "undirected", "growth", "no-tree-edges"])
def test_threaded_repair_equals_sequential(case):
    # the CPU baseline runs the oracle's repair on several threads (openmp.cpp:223-583): the
    # trees and the deterministic counters (invalidated, affected) equal the sequential engine's
    # after every batch of a chain
    from tests.helpers import random_batch, random_graph
    rng = np.random.default_rng({"sparse": 1, "multigraph-k2": 2, "undirected": 3, "growth": 4,
                                 "no-tree-edges": 5}[case])
    n, src, dst, w = random_graph(rng, "sparse", 2000, multi=case == "multigraph-k2")
    k = 2 if case == "multigraph-k2" else 1
    objective = k - 1
    if k == 2:
        w = np.stack([w, rng.integers(1, 9, w.size)], axis=1).reshape(-1)
    props = {"multigraph-k2": O.mosp_props(), "undirected": O.mosp_props(directed=0)}.get(
        case, O.default_props())
    batches = []
    parents = None
    runs = {}
    try:
        for threads in (1, 8):
            O.set_threads(threads)
            g = O.Graph.from_edges(n, src, dst, w, k, props)
            t, _ = O.compute(g, 0, objective=objective, rule=1)
            seen = []
            for step in range(4):
                if threads == 1:
                    if case == "no-tree-edges":
                        b = {"ins_src": rng.integers(0, n, 50).astype(np.int32),
                             "ins_dst": rng.integers(0, n, 50).astype(np.int32),
                             "ins_w": rng.integers(1, 9, 50).astype(np.int32),
                             "del_src": np.zeros(0, np.int32), "del_dst": np.zeros(0, np.int32)}
                    else:
                        b = random_batch(rng, g.n, src, dst, 400, tree_parents=t.parents,
                                         grow=40 if case == "growth" else 0)
                    b["ins_w"] = np.repeat(b["ins_w"], k) if k > 1 else b["ins_w"]
                    batches.append(b)
                b = batches[step]
                st, sm = O.update(g, O.Batch(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"],
                                             b["del_dst"], k), t)
                seen.append((st["invalidated"], st["affected"], sm["num_vertices_after"],
                             t.distances.copy(), t.parents.copy()))
            runs[threads] = seen
    finally:
        O.set_threads(1)
    for step, (a, b) in enumerate(zip(runs[1], runs[8])):
        assert a[:3] == b[:3], (case, step)
        np.testing.assert_array_equal(a[3], b[3], err_msg=f"{case} step {step}")
        np.testing.assert_array_equal(a[4], b[4], err_msg=f"{case} step {step}")
    assert any(s[0] > 0 for s in runs[1]) or case == "no-tree-edges"
