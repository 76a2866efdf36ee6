"""Parity of the CUDA path (through the C ABI) with the oracle and the reference's goldens.

Bit-exact int64 distances, int32 parents, `invalidated` and `affected` (integer work: no
tolerance).  The cases follow the reference's own tests:
  - cpp/tests/algorithms/sssp/sssp_fixture_test.cpp:110-190 (34 golden cases, every objective);
  - cpp/tests/data/mosp_graph_io/*/applied (the device applier's CSR, transpose and
    weight-increase mask);
  - cpp/tests/algorithms/sssp/sssp_test.cpp:74-333 (hand cases);
  - cpp/tests/algorithms/sssp/sssp_random_test.cpp:467-580 (random shapes, chains of batches,
    equal to the oracle and to compute() on the new graph).
"""
import zlib

import numpy as np
import pytest

import dyng_b200 as D
from dyng_b200 import generators as G
from oracle import oracle as O
from tests.helpers import INF, SHAPES, fixture_case, random_batch, random_graph

pytestmark = pytest.mark.gpu


def _batch(ins_src=(), ins_dst=(), ins_w=(), del_src=(), del_dst=(), k=1):
    return D.EdgeBatch.from_arrays(ins_src, ins_dst, ins_w, del_src, del_dst, num_weights=k)


def _obatch(ins_src=(), ins_dst=(), ins_w=(), del_src=(), del_dst=(), k=1):
    return O.Batch(ins_src, ins_dst, ins_w, del_src, del_dst, k)


def _cases(z):
    return [str(c) for c in z["cases"]]


def test_fixtures_compute_and_update(fixtures):
    done = 0
    for name in _cases(fixtures):
        c = fixture_case(fixtures, name)
        k = c["k"]
        for j in range(k):
            g = D.Graph.from_csr(c["row_ptr"], c["col"], c["w"], D.GraphProperties.mosp_compatible(),
                                 num_weights=k)
            r = D.sssp.compute(g, 0, D.sssp.Options(objective=j))
            np.testing.assert_array_equal(r.distances, c["init_d"][j], err_msg=f"{name} obj{j}")
            np.testing.assert_array_equal(r.parents, c["init_p"][j], err_msg=f"{name} obj{j}")
            t = D.sssp.Result.from_arrays(g, 0, c["init_d"][j], c["init_p"][j], canonicalize=False,
                                          options=D.sssp.Options(objective=j))
            st = D.sssp.update(g, _batch(c["ins_src"], c["ins_dst"], c["ins_w"], c["del_src"],
                                         c["del_dst"], k), t)
            np.testing.assert_array_equal(t.distances, c["upd_d"][j], err_msg=f"{name} obj{j}")
            np.testing.assert_array_equal(t.parents, c["upd_p"][j], err_msg=f"{name} obj{j}")
            assert st.invalidated == c["invalidated"][j], name
            assert t.graph_version == g.version() == 1
            done += 1
    assert done > 34


def test_fixtures_update_each_objective_on_one_graph(fixtures):
    # dyng::update_each (update.hpp:331): the K trees of a fixture on one graph, the batch applied
    # once; every tree equals the golden of its objective (the MOSP compat driver's use)
    done = 0
    for name in _cases(fixtures):
        c = fixture_case(fixtures, name)
        k = c["k"]
        if k < 2:
            continue
        g = D.Graph.from_csr(c["row_ptr"], c["col"], c["w"], D.GraphProperties.mosp_compatible(),
                             num_weights=k)
        trees = [D.sssp.Result.from_arrays(g, 0, c["init_d"][j], c["init_p"][j],
                                           canonicalize=False, options=D.sssp.Options(objective=j))
                 for j in range(k)]
        stats = D.sssp.update_each(g, _batch(c["ins_src"], c["ins_dst"], c["ins_w"], c["del_src"],
                                             c["del_dst"], k), trees)
        assert g.version() == 1 and len(stats) == k
        for j, (t, st) in enumerate(zip(trees, stats)):
            np.testing.assert_array_equal(t.distances, c["upd_d"][j], err_msg=f"{name} obj{j}")
            np.testing.assert_array_equal(t.parents, c["upd_p"][j], err_msg=f"{name} obj{j}")
            assert st.invalidated == c["invalidated"][j], (name, j)
            assert t.graph_version == 1
        done += 1
    assert done >= 10


def test_update_each_errors_keep_every_tree():
    # an error before the batch is applied (a weight below 1 in the second objective) changes
    # nothing; a tree listed twice is refused
    g = D.Graph.from_edges([0, 1], [1, 2], [[3, 4], [5, 6]], num_weights=2)
    t0 = D.sssp.compute(g, 0, D.sssp.Options(objective=0))
    t1 = D.sssp.compute(g, 0, D.sssp.Options(objective=1))
    with pytest.raises(D.InvalidArgumentError):
        D.sssp.update_each(g, _batch([0], [2], [1, 0], k=2), [t0, t1])
    assert g.version() == 0 and t0.distances.tolist() == [0, 3, 8]
    with pytest.raises(D.InvalidArgumentError):
        D.sssp.update_each(g, _batch([0], [2], [1, 1], k=2), [t0, t0])
    st = D.sssp.update_each(g, _batch([0], [2], [1, 1], k=2), [t0, t1])
    assert t0.distances.tolist() == [0, 3, 1] and t1.distances.tolist() == [0, 4, 1]
    assert [s.batch.inserted_edges for s in st] == [1, 1]


def test_fixtures_applied_csr(fixtures):
    checked = 0
    for name in _cases(fixtures):
        c = fixture_case(fixtures, name)
        if "applied_row_ptr" not in c:
            continue
        k = c["k"]
        g = D.Graph.from_csr(c["row_ptr"], c["col"], c["w"], D.GraphProperties.mosp_compatible(),
                             num_weights=k)
        _, mask = g.apply(_batch(c["ins_src"], c["ins_dst"], c["ins_w"], c["del_src"], c["del_dst"],
                                 k), classify=True)
        out = g.to_csr()
        np.testing.assert_array_equal(out.row_ptr, c["applied_row_ptr"], err_msg=name)
        np.testing.assert_array_equal(out.col_ind, c["applied_col"], err_msg=name)
        np.testing.assert_array_equal(out.weights, c["applied_w"], err_msg=name)
        tr = g.to_csr(transposed=True)
        np.testing.assert_array_equal(tr.row_ptr, c["applied_in_row_ptr"], err_msg=name)
        np.testing.assert_array_equal(tr.col_ind, c["applied_in_col"], err_msg=name)
        np.testing.assert_array_equal(tr.weights, c["applied_in_w"], err_msg=name)
        np.testing.assert_array_equal(mask, c["applied_increase"], err_msg=name)
        checked += 1
    assert checked == 27


def _pair(n, edges, props, k=1):
    src = [e[0] for e in edges]
    dst = [e[1] for e in edges]
    w = [x for e in edges for x in e[2:]]
    dp = D.GraphProperties.mosp_compatible() if props == "mosp" else D.GraphProperties(
        **(props or {}))
    op = O.mosp_props() if props == "mosp" else O.default_props(
        **{kk: int(v) for kk, v in (props or {}).items()})
    return (D.Graph.from_edges(src, dst, w, n, dp, num_weights=k),
            O.Graph.from_edges(n, src, dst, w, k, op))


def test_readme_quickstart():
    g, _ = _pair(4, [(0, 1, 4), (0, 2, 1), (2, 1, 2), (1, 3, 1)], None)
    t = D.sssp.compute(g, 0)
    assert t.distances.tolist() == [0, 3, 1, 4]
    st = D.sssp.update(g, _batch([2], [3], [1], [2], [1]), t)
    assert t.distances.tolist() == [0, 4, 1, 2] and st.invalidated == 2


def test_readme_quickstart_through_the_mirrored_python_api():
    # the reference's README quickstart (README.md:49-59), call for call
    g = D.Graph.from_edges([0, 0, 2, 1], [1, 2, 1, 3], [4, 1, 2, 1])
    tree = D.sssp.compute(g, source=0)
    assert tree.distances.tolist() == [0, 3, 1, 4]
    batch = D.EdgeBatch(insert=([2], [3], [1]), delete=([2], [1]))
    stats = D.sssp.update(g, batch, tree)
    assert (tree.distances.tolist(), stats.invalidated) == ([0, 4, 1, 2], 2)


def test_hand_cases():
    g, _ = _pair(5, [(0, 1, 5), (0, 2, 1), (2, 3, 1), (1, 4, 2), (3, 4, 2)], "mosp")
    t = D.sssp.compute(g, 0)
    assert t.parents.tolist() == [-1, 0, 0, 2, 3]
    st = D.sssp.update(g, _batch([2], [1], [1]), t)
    assert t.distances.tolist() == [0, 2, 1, 2, 4] and t.parents.tolist() == [-1, 2, 0, 2, 1]
    assert (st.invalidated, st.affected, st.batch.inserted_edges) == (0, 2, 1)
    # delete-all, then re-insert (sssp_test.cpp:114-135)
    g, _ = _pair(5, [(0, 1, 3), (1, 2, 4), (0, 3, 2), (3, 4, 7)], "mosp")
    t = D.sssp.compute(g, 0)
    st = D.sssp.update(g, _batch(del_src=[0, 1, 0, 3], del_dst=[1, 2, 3, 4]), t)
    assert g.num_edges() == 0 and t.distances.tolist() == [0] + [INF] * 4
    assert (st.invalidated, st.affected) == (4, 4)
    D.sssp.update(g, _batch([0, 4], [4, 2], [9, 1]), t)
    assert t.distances.tolist() == [0, INF, 10, INF, 9]
    assert t.parents.tolist() == [-1, -1, 4, -1, 0]
    # empty batch
    st = D.sssp.update(g, _batch(), t)
    assert (st.affected, st.invalidated, st.iterations) == (0, 0, 0)
    # vertex growth (sssp_test.cpp:188-199)
    g, _ = _pair(3, [(0, 1, 2), (1, 2, 2)], None)
    t = D.sssp.compute(g, 0)
    st = D.sssp.update(g, _batch([2, 5], [5, 3], [1, 4]), t)
    assert g.num_vertices() == 6 and st.batch.num_vertices_after == 6
    assert t.distances.tolist() == [0, 2, 4, 9, INF, 5]
    assert t.parents.tolist() == [-1, 0, 1, 5, -1, 2]
    # undirected (sssp_test.cpp:201-212)
    g, _ = _pair(4, [(0, 1, 1), (1, 2, 1), (2, 3, 1)], {"directed": False})
    t = D.sssp.compute(g, 3)
    assert t.distances.tolist() == [3, 2, 1, 0]
    D.sssp.update(g, _batch([0], [3], [5], [1], [2]), t)
    assert t.distances.tolist() == [5, 6, 1, 0] and t.parents.tolist() == [3, 0, 3, -1]
    # non-canonical input tree keeps its tie parents (sssp_test.cpp:313-333)
    g, _ = _pair(5, [(0, 1, 1), (0, 2, 1), (1, 3, 1), (2, 3, 1), (0, 4, 5), (4, 3, 1)], "mosp")
    t = D.sssp.Result.from_arrays(g, 0, [0, 1, 1, 2, 5], [-1, 0, 0, 2, 0], canonicalize=False)
    st = D.sssp.update(g, _batch([0], [4], [1]), t)
    assert t.parents.tolist() == [-1, 0, 0, 2, 0] and st.affected == 1


def test_errors_keep_state():
    g, _ = _pair(3, [(0, 1, 2), (1, 2, 2)], None)
    t = D.sssp.compute(g, 0)
    with pytest.raises(D.InvalidArgumentError):
        D.sssp.update(g, _batch([0], [1], [0]), t)  # weight below 1
    with pytest.raises(D.InvalidArgumentError):
        D.sssp.update(g, _batch([-1], [1], [3]), t)  # negative id
    assert g.version() == 0 and g.num_edges() == 2
    D.sssp.update(g, _batch([0], [2], [1]), t)
    other = D.sssp.compute(g, 0)
    D.sssp.update(g, _batch([1], [0], [1]), t)
    with pytest.raises(D.StaleResultError):
        D.sssp.update(g, _batch([1], [0], [1]), other)  # computed on an older version
    with pytest.raises(D.InvalidArgumentError):
        D.sssp.Result.from_arrays(g, 0, [0, 1, 1], [-1, 2, 1], canonicalize=False)  # a cycle


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("weights", ["tiny", "small", "huge"])
def test_random_chains(shape, weights):
    rng = np.random.default_rng(zlib.crc32(f"{shape}/{weights}".encode()))
    for trial in range(2):
        n = int(rng.integers(20, 400))
        n, src, dst, w = random_graph(rng, shape, n, weights)
        props = None if trial == 0 else "mosp"
        g, og = _pair(n, list(zip(src.tolist(), dst.tolist(), w.tolist())), props)
        source = int(rng.integers(0, n))
        t = D.sssp.compute(g, source)
        ot, _ = O.compute(og, source, rule=1)
        np.testing.assert_array_equal(t.distances, ot.distances)
        np.testing.assert_array_equal(t.parents, ot.parents)
        for step in range(4):
            b = random_batch(rng, og.n, src, dst, int(rng.integers(1, 3 * n)), weights,
                             tree_parents=ot.parents, grow=2 if step == 1 else 0)
            st = D.sssp.update(g, _batch(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"],
                                         b["del_dst"]), t)
            ost, osm = O.update(og, _obatch(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"],
                                            b["del_dst"]), ot)
            np.testing.assert_array_equal(t.distances, ot.distances, err_msg=f"step {step}")
            np.testing.assert_array_equal(t.parents, ot.parents, err_msg=f"step {step}")
            assert st.invalidated == ost["invalidated"]
            assert st.affected == ost["affected"]
            assert st.batch.inserted_edges == osm["inserted_edges"]
            assert st.batch.deleted_edges == osm["deleted_edges"]
            assert st.batch.updated_edges == osm["updated_edges"]
            assert st.batch.ignored_deletions == osm["ignored_deletions"]
            assert g.num_edges() == og.m and g.num_vertices() == og.n
            # equal to a from-scratch compute on the new graph (canonical trees)
            fresh = D.sssp.compute(g, source)
            np.testing.assert_array_equal(fresh.distances, t.distances)
            np.testing.assert_array_equal(fresh.parents, t.parents)
        csr = g.to_csr()
        ocsr = og.to_csr()
        np.testing.assert_array_equal(csr.row_ptr, ocsr["row_ptr"])
        np.testing.assert_array_equal(csr.col_ind, ocsr["col"])
        np.testing.assert_array_equal(csr.weights, ocsr["w"])


def test_rmat_scale16_batch():
    # the CPU configuration: R-MAT scale 16, ef 16, w in [1,100], 5k deletions + 5k insertions
    e = G.rmat(16, 16, w_max=100, seed=1)
    b = G.uniform_batch(e, 5000, 5000, seed=7, w_max=100)
    rp, col, w = e.csr()
    g = D.Graph.from_csr(rp, col, w)
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    t = D.sssp.compute(g, 0)
    ot, _ = O.compute(og, 0, rule=1)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)
    st = D.sssp.update(g, _batch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                 b.delete_dst), t)
    ost, _ = O.update(og, _obatch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                  b.delete_dst), ot)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)
    assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])
    # every finite distance fits in 31 bits at this size
    fin = t.distances[t.distances < INF // 2]
    assert fin.max() < 2**31


def test_large_frontiers_match_the_oracle():
    # frontiers of tens of thousands of rows (the edge-parallel expansion): a Bellman-Ford-like
    # width on R-MAT scale 17 for compute, and a 60k-change batch, against the oracle
    e = G.rmat(17, 16, w_max=1000, seed=4)
    rp, col, w = e.csr()
    g = D.Graph.from_csr(rp, col, w)
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    t, cst = D.sssp.compute(g, 0, D.sssp.Options(delta=1 << 40), stats=True)
    ot, _ = O.compute(og, 0, rule=1)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)
    assert max(light for light, _, _ in cst.trace) >= 8192
    b = G.BatchStream(e, seed=3).next(60000, 0.6, 0.5, parents=ot.parents)
    st = D.sssp.update(g, _batch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                 b.delete_dst), t, schedule=D.sssp.Schedule(delta=1 << 40))
    ost, _ = O.update(og, _obatch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                  b.delete_dst), ot)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)
    assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])
    assert max(light for light, _, _ in st.trace) >= 8192


def test_arena_growth_and_compaction_keep_results():
    # batches far larger than the slack rows: the arenas grow on the device (and, after heavy
    # churn, the graph is compacted); every step equals the oracle, and the exported CSR too
    rng = np.random.default_rng(21)
    n, s, d, w = random_graph(rng, "sparse", 2000)
    g = D.Graph.from_edges(s, d, w, num_vertices=n)
    og = O.Graph.from_edges(n, s, d, w, 1)
    t = D.sssp.compute(g, 0)
    ot, _ = O.compute(og, 0, rule=1)
    for step in range(6):
        b = random_batch(rng, n, s, d, 40000 if step % 2 == 0 else 30000, tree_parents=ot.parents)
        D.sssp.update(g, _batch(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"],
                                b["del_dst"]), t)
        O.update(og, _obatch(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"],
                             b["del_dst"]), ot)
        np.testing.assert_array_equal(t.distances, ot.distances, err_msg=f"step {step}")
        np.testing.assert_array_equal(t.parents, ot.parents, err_msg=f"step {step}")
    csr = g.to_csr()
    want = og.to_csr()
    np.testing.assert_array_equal(csr.row_ptr, want["row_ptr"])
    np.testing.assert_array_equal(csr.col_ind, want["col"])
    np.testing.assert_array_equal(csr.weights.reshape(-1), want["w"].reshape(-1))


@pytest.mark.parametrize("k", [1, 2])
def test_device_growth_and_compaction_keep_rows_and_results(k):
    # one batch far larger than the arena (it grows, on the device), then churn until the
    # abandoned slots pass half the edges and the next overflow compacts both sides on the
    # device; every step equals the oracle, and the exported CSR keeps the storage order
    rng = np.random.default_rng(40 + k)
    n, s, d, _ = random_graph(rng, "sparse", 2000)
    w = rng.integers(1, 60, (k, s.size)).reshape(-1)
    g = D.Graph.from_edges(s, d, w, num_vertices=n, num_weights=k)
    og = O.Graph.from_edges(n, s, d, w, k)
    obj = k - 1
    t = D.sssp.compute(g, 0, D.sssp.Options(objective=obj))
    ot, _ = O.compute(og, 0, objective=obj, rule=1)
    for step in range(24):
        size = 240000 if step == 0 else 20000
        b = random_batch(rng, n, s, d, size, tree_parents=ot.parents)
        ni = len(b["ins_src"])
        iw = rng.integers(1, 60, ni * k)
        D.sssp.update(g, _batch(b["ins_src"], b["ins_dst"], iw, b["del_src"], b["del_dst"], k), t)
        O.update(og, _obatch(b["ins_src"], b["ins_dst"], iw, b["del_src"], b["del_dst"], k), ot)
        np.testing.assert_array_equal(t.distances, ot.distances, err_msg=f"step {step}")
        np.testing.assert_array_equal(t.parents, ot.parents, err_msg=f"step {step}")
        st = g.storage()
        if step == 0:
            assert st["arena_growths"] >= 1 and st["compactions"] == 0, st
        if st["compactions"] >= 1:
            break
    assert st["compactions"] >= 1, st
    csr = g.to_csr()
    want = og.to_csr()
    np.testing.assert_array_equal(csr.row_ptr, want["row_ptr"])
    np.testing.assert_array_equal(csr.col_ind, want["col"])
    np.testing.assert_array_equal(csr.weights.reshape(-1), want["w"].reshape(-1))
    # the edge index was rebuilt over the moved slots: deleting and upserting through it works
    ed = og.to_csr()
    u = np.repeat(np.arange(n), np.diff(ed["row_ptr"]))[:50]
    v = ed["col"][:50]
    iw = rng.integers(1, 60, 50 * k)
    D.sssp.update(g, _batch(u, v, iw, u[::2], v[::2], k), t)
    O.update(og, _obatch(u, v, iw, u[::2], v[::2], k), ot)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)
    np.testing.assert_array_equal(g.to_csr().col_ind, og.to_csr()["col"])


def test_schedules_never_change_results():
    # sssp::options::delta and the schedule are tunables (sssp.hpp:78-94): every schedule gives
    # the same bytes as the oracle
    e = G.rmat(13, 8, w_max=1000, seed=11)
    rp, col, w = e.csr()
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    ot, _ = O.compute(og, 0, rule=1)
    schedules = [None, D.sssp.Schedule(delta=1), D.sssp.Schedule(delta=100000),
                 D.sssp.Schedule(grid_blocks=7), D.sssp.Schedule(small_frontier=-1),
                 D.sssp.Schedule(small_frontier=100000), D.sssp.Schedule(invalidation=1),
                 D.sssp.Schedule(heavy_degree=33), D.sssp.Schedule(heavy_degree=100000)]
    graphs = [(D.Graph.from_csr(rp, col, w), s) for s in schedules]
    trees = [D.sssp.compute(g, 0) for g, _ in graphs]
    stream = G.BatchStream(e, seed=3)
    for step in range(3):
        b = stream.next(600, 0.75, 0.5, parents=ot.parents)
        ost, _ = O.update(og, _obatch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                      b.delete_dst), ot)
        for (g, sched), t in zip(graphs, trees):
            st = D.sssp.update(g, _batch(b.insert_src, b.insert_dst, b.insert_weights,
                                         b.delete_src, b.delete_dst), t, schedule=sched)
            np.testing.assert_array_equal(t.distances, ot.distances, err_msg=str(sched))
            np.testing.assert_array_equal(t.parents, ot.parents, err_msg=str(sched))
            assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])


def test_unvalidated_cycle_is_reported_and_poisons():
    # sssp_cuda_test.cpp:982: a parent cycle in a tree imported without validation is found by
    # pointer jumping; the graph keeps the batch, the result is poisoned
    g, _ = _pair(4, [(0, 1, 1), (1, 2, 1), (2, 1, 1), (2, 3, 1)], None)
    t = D.sssp.Result.from_arrays(g, 0, [0, 1, 2, 3], [-1, 2, 1, 2], canonicalize=False,
                                  options=D.sssp.Options(validate_inputs=False))
    with pytest.raises(D.InvalidArgumentError):
        D.sssp.update(g, _batch(del_src=[2], del_dst=[3]), t)
    assert g.version() == 1
    with pytest.raises(D.StaleResultError):
        t.distances
