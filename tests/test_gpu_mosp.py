"""dyng_b200.mosp on the device against the reference's goldens and the oracle (bit-exact).

  - cpp/tests/data/mosp_combined (8 cases; python/tests/test_cli.py:686-723 replays them): the
    K initial trees adopted, the batch applied once, then the combined distances, the MOSP tree
    and the path costs over every weight column equal the golden files;
  - cpp/tests/algorithms/mosp/mosp_test.cpp:155-280: the thesis' worked example under two
    preference vectors, default preferences, unreachable vertices;
  - mosp_test.cpp:213-247 and mosp_random_test.cpp: K = 1..4, with and without preferences,
    simple graphs (edge index) and MOSP-compatible multigraphs (row scans), chains of batches
    with vertex growth, each step equal to the oracle's finalize step on the oracle's trees,
    `affected` equal to the vertices whose combined distance or parent changed;
  - mosp_test.cpp:281-430: the options are checked; path costs can be switched off and on.
"""
import numpy as np
import pytest

import dyng_b200 as D
from dyng_b200 import mosp
from oracle import oracle as O
from tests.helpers import INF, combined_case, random_batch

pytestmark = pytest.mark.gpu


def _batch(ins_src=(), ins_dst=(), ins_w=(), del_src=(), del_dst=(), k=1):
    return D.EdgeBatch.from_arrays(ins_src, ins_dst, ins_w, del_src, del_dst, num_weights=k)


def test_combined_fixtures(combined_fixtures):
    names = [str(x) for x in combined_fixtures["cases"]]
    for name in names:
        c = combined_case(combined_fixtures, name)
        k, kg = c["k"], c["kg"]
        g = D.Graph.from_csr(c["row_ptr"], c["col"], c["w"], D.GraphProperties.mosp_compatible(),
                             num_weights=kg)
        r = mosp.Result.from_arrays(g, 0, c["init_d"], c["init_p"], canonicalize=False,
                                    num_objectives=k, preferences=c["pref"])
        st = mosp.update(g, _batch(c["ins_src"], c["ins_dst"], c["ins_w"], c["del_src"],
                                   c["del_dst"], kg), r)
        np.testing.assert_array_equal(r.combined_distances, c["combined_d"], err_msg=name)
        np.testing.assert_array_equal(r.combined_parents, c["combined_p"], err_msg=name)
        np.testing.assert_array_equal(r.path_costs_over(kg), c["costs"], err_msg=name)
        np.testing.assert_array_equal(r.path_costs, c["costs"][:, :k], err_msg=name)
        assert st.preference_scale == r.preference_scale and len(st.objectives) == k
        assert r.graph_version == g.version() == 1
    assert len(names) == 8


def test_default_preferences_weigh_an_edge_by_its_trees():
    # mosp_test.cpp:249-269
    g = D.Graph.from_edges([0, 0, 1, 2], [1, 2, 3, 3], [1, 5, 5, 1, 1, 5, 5, 1], num_weights=2)
    r = mosp.compute(g, 0)
    assert r.preference_scale == 1 and r.combined_distances.tolist() == [0, 1, 1, 3]
    assert r.combined_parents.tolist() == [-1, 0, 0, 1] and r.path_costs[3].tolist() == [2, 10]
    q = mosp.compute(g, 0, preferences=[2, 1])
    assert q.preference_scale == 2 and q.combined_distances.tolist() == [0, 3, 3, 7]
    assert q.combined_parents.tolist() == [-1, 0, 0, 2] and q.path_costs[3].tolist() == [10, 2]


def test_unreachable_vertices_have_no_parent_and_infinite_costs():
    # mosp_test.cpp:271-279
    g = D.Graph.from_edges([0, 2], [1, 3], [1, 1, 1, 1], num_vertices=4, num_weights=2)
    r = mosp.compute(g, 0)
    assert r.combined_distances.tolist() == [0, 1, INF, INF]
    assert r.combined_parents.tolist() == [-1, 0, -1, -1]
    assert r.path_costs[2].tolist() == [INF, INF] and r.path_costs[0].tolist() == [0, 0]


THESIS = [(0, 1, 2, 1, 5), (0, 2, 4, 1, 1), (1, 3, 2, 4, 2), (2, 1, 10, 15, 2), (2, 3, 5, 16, 3),
          (3, 4, 1, 1, 1), (4, 1, 4, 3, 2), (4, 5, 1, 2, 2), (4, 6, 5, 6, 2), (5, 6, 1, 1, 1)]


def test_the_thesis_worked_example():
    # mosp_test.cpp:155-211
    for pref, path, cost in (([4, 1, 4], [6, 5, 1, 0], [15, 3, 20]),
                             ([4, 4, 1], [6, 4, 3, 2, 0], [15, 24, 7])):
        g = D.Graph.from_edges([e[0] for e in THESIS], [e[1] for e in THESIS],
                               [x for e in THESIS for x in e[2:]], num_vertices=7,
                               properties=D.GraphProperties.mosp_compatible(), num_weights=3)
        r = mosp.compute(g, 0, preferences=pref)
        assert r.preference_scale == 4
        st = mosp.update(g, _batch([3, 1], [5, 5], [10, 2, 12, 12, 1, 14], [1, 4], [3, 1], 3), r)
        assert [r.parents(k).tolist() for k in range(3)] == [
            [-1, 0, 0, 2, 3, 4, 5], [-1, 0, 0, 2, 3, 1, 5], [-1, 2, 0, 2, 3, 4, 4]]
        par = r.combined_parents
        walk = [6]
        while par[walk[-1]] >= 0:
            walk.append(int(par[walk[-1]]))
        assert walk == path and r.path_costs[6].tolist() == cost
        assert st.preference_scale == 4 and len(st.objectives) == 3
        fresh = mosp.compute(g, 0, preferences=pref)
        np.testing.assert_array_equal(fresh.combined_distances, r.combined_distances)
        np.testing.assert_array_equal(fresh.combined_parents, r.combined_parents)
        np.testing.assert_array_equal(fresh.path_costs, r.path_costs)


def _oracle_mosp(og, source, trees, pref):
    return O.mosp_finalize(og, source, [t.parents for t in trees], pref)


def _check(r, m, what):
    np.testing.assert_array_equal(r.combined_distances, m.distances, err_msg=what)
    np.testing.assert_array_equal(r.combined_parents, m.parents, err_msg=what)
    np.testing.assert_array_equal(r.path_costs, m.costs, err_msg=what)


@pytest.mark.parametrize("multi", [False, True])
@pytest.mark.parametrize("K", [1, 2, 3, 4])
def test_random_chains_equal_the_oracle(K, multi):
    rng = np.random.default_rng(100 * K + multi)
    n, m = 400, 1600
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    if not multi:
        pairs = np.unique(src.astype(np.int64) * n + dst)
        src, dst = (pairs // n).astype(np.int32), (pairs % n).astype(np.int32)
    w = rng.integers(1, 8, src.size * K)  # few distinct weights: many ties
    props = D.GraphProperties.mosp_compatible() if multi else D.GraphProperties()
    oprops = O.mosp_props() if multi else O.default_props()
    for pref in ([], [k + 1 for k in range(K)]):
        g = D.Graph.from_edges(src, dst, w, num_vertices=n, properties=props, num_weights=K)
        og = [O.Graph.from_edges(n, src, dst, w, K, oprops) for _ in range(K)]
        r = mosp.compute(g, 3, preferences=pref)
        trees = [O.compute(og[j], 3, objective=j, rule=1)[0] for j in range(K)]
        before = _oracle_mosp(og[0], 3, trees, pref)
        _check(r, before, f"K={K} compute")
        for step in range(3):
            b = random_batch(rng, n, src, dst, 120, weights="tiny", grow=4 if step == 1 else 0)
            iw = rng.integers(1, 8, len(b["ins_src"]) * K)
            st = mosp.update(g, _batch(b["ins_src"], b["ins_dst"], iw, b["del_src"], b["del_dst"],
                                       K), r)
            for j in range(K):
                O.update(og[j], O.Batch(b["ins_src"], b["ins_dst"], iw, b["del_src"],
                                        b["del_dst"], K), trees[j])
            after = _oracle_mosp(og[0], 3, trees, pref)
            _check(r, after, f"K={K} step {step}")
            for j in range(K):
                np.testing.assert_array_equal(r.distances(j), trees[j].distances)
                np.testing.assert_array_equal(r.parents(j), trees[j].parents)
            n_old = before.distances.size
            old_d = np.full(after.distances.size, INF, np.int64)
            old_p = np.full(after.distances.size, -1, np.int32)
            old_d[:n_old], old_p[:n_old] = before.distances, before.parents
            assert st.affected == int(np.sum((old_d != after.distances) |
                                             (old_p != after.parents)))
            assert st.combined_edges == after.combined_edges
            before = after


def test_options_are_checked():
    # mosp_test.cpp:281-336
    g = D.Graph.from_edges([0, 1], [1, 2], [1, 1, 1, 1], num_weights=2)
    for kw in ({"preferences": [0, 1]}, {"preferences": [1]}, {"preferences": [1, 2, 3]},
               {"preferences": [1 << 20, 3]}, {"num_objectives": 3}, {"delta": -1}):
        with pytest.raises(D.InvalidArgumentError):
            mosp.compute(g, 0, **kw)
    with pytest.raises(D.InvalidArgumentError):
        mosp.compute(g, 5)
    r = mosp.compute(g, 0, num_objectives=1)
    assert r.num_objectives == 1 and r.path_costs.shape == (3, 1)
    with pytest.raises(D.InvalidArgumentError):
        r.set_options(preferences=[3])
    with pytest.raises(D.InvalidArgumentError):
        r.tree(1)


def test_path_costs_can_be_switched_off_and_on():
    # mosp_test.cpp:398-430
    g = D.Graph.from_edges([0, 1], [1, 2], [1, 2, 3, 4], num_weights=2)
    r = mosp.compute(g, 0, compute_path_costs=False)
    with pytest.raises(D.InvalidArgumentError):
        r.path_costs
    r.set_options(compute_path_costs=True)
    with pytest.raises(D.InvalidArgumentError):
        r.path_costs  # takes effect at the next update
    mosp.update(g, _batch([0], [2], [9, 9], k=2), r)
    assert r.path_costs.tolist() == [[0, 0], [1, 2], [4, 6]]


def test_stale_results_are_refused():
    g = D.Graph.from_edges([0, 1], [1, 2], [1, 2, 3, 4], num_weights=2)
    r = mosp.compute(g, 0)
    D.sssp.update(g, _batch([0], [2], [5, 5], k=2), D.sssp.compute(g, 0))
    with pytest.raises(D.StaleResultError):
        mosp.update(g, _batch([0], [2], [1, 1], k=2), r)
