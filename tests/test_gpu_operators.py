"""The operators engine (cuda_engine="operators"): compute and update as ordinary kernel launches
with the near-far loop driven from the host, the engine that cuda_engine="automatic" runs on a
device without cooperative launch (sssp.cpp:195-226 of the reference; its operators.cu).  Its
results equal the oracle's (and the fused engine's) bit for bit:

  - the golden fixtures: compute, the update of imported non-canonical trees, update_each;
  - the random shapes of sssp_random_test.cpp with chains of batches, with pointer jumping and
    with the subtree walk, with graph growth;
  - the distance-only mode (large weights) and the 47-bit packing boundary;
  - a parent cycle in a tree imported without validation is reported and poisons the tree;
  - a device taken as one without cooperative launch (sssp_cuda_test.cpp:106-150): automatic runs
    the operators engine and the batch applier as one launch per step (graph.apply too), and the
    fused engine is refused before anything changes.
"""
import numpy as np
import pytest

import dyng_b200 as D
from oracle import oracle as O
from tests.helpers import SHAPES, fixture_case, random_batch, random_graph

pytestmark = pytest.mark.gpu

OPS = "operators"


def _batch(ins_src=(), ins_dst=(), ins_w=(), del_src=(), del_dst=(), k=1):
    return D.EdgeBatch.from_arrays(ins_src, ins_dst, ins_w, del_src, del_dst, num_weights=k)


def _obatch(ins_src=(), ins_dst=(), ins_w=(), del_src=(), del_dst=(), k=1):
    return O.Batch(ins_src, ins_dst, ins_w, del_src, del_dst, k)


def _db(b, k=1):
    return _batch(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"], b["del_dst"], k)


def _ob(b, k=1):
    return _obatch(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"], b["del_dst"], k)


def _same(t, ot, label=""):
    np.testing.assert_array_equal(t.distances, ot.distances, err_msg=label)
    np.testing.assert_array_equal(t.parents, ot.parents, err_msg=label)


def test_fixtures_compute_update_and_update_each(fixtures):
    done = 0
    for name in [str(c) for c in fixtures["cases"]]:
        c = fixture_case(fixtures, name)
        k = c["k"]
        props = D.GraphProperties.mosp_compatible()
        for j in range(k):
            opt = D.sssp.Options(objective=j, cuda_engine=OPS)
            g = D.Graph.from_csr(c["row_ptr"], c["col"], c["w"], props, num_weights=k)
            r, cst = D.sssp.compute(g, 0, opt, stats=True)
            assert cst.engine_used == OPS
            np.testing.assert_array_equal(r.distances, c["init_d"][j], err_msg=f"{name} obj{j}")
            np.testing.assert_array_equal(r.parents, c["init_p"][j], err_msg=f"{name} obj{j}")
            t = D.sssp.Result.from_arrays(g, 0, c["init_d"][j], c["init_p"][j],
                                          canonicalize=False, options=opt)
            st = D.sssp.update(g, _db(c, k), t)
            assert st.engine_used == OPS
            np.testing.assert_array_equal(t.distances, c["upd_d"][j], err_msg=f"{name} obj{j}")
            np.testing.assert_array_equal(t.parents, c["upd_p"][j], err_msg=f"{name} obj{j}")
            assert st.invalidated == c["invalidated"][j], name
            done += 1
        if k >= 2:
            g = D.Graph.from_csr(c["row_ptr"], c["col"], c["w"], props, num_weights=k)
            trees = [D.sssp.Result.from_arrays(g, 0, c["init_d"][j], c["init_p"][j],
                                               canonicalize=False,
                                               options=D.sssp.Options(objective=j, cuda_engine=OPS))
                     for j in range(k)]
            stats = D.sssp.update_each(g, _db(c, k), trees)
            for j, (t, st) in enumerate(zip(trees, stats)):
                assert st.engine_used == OPS
                np.testing.assert_array_equal(t.distances, c["upd_d"][j], err_msg=f"{name} {j}")
                np.testing.assert_array_equal(t.parents, c["upd_p"][j], err_msg=f"{name} {j}")
                assert st.invalidated == c["invalidated"][j], (name, j)
    assert done > 34


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("walk", [0, 1])
def test_random_shapes_chains_of_batches(shape, walk):
    rng = np.random.default_rng(1000 + SHAPES.index(shape) + 10 * walk)
    n, s, d, w = random_graph(rng, shape, 4000 if shape != "dense" else 300)
    g = D.Graph.from_edges(s, d, w, n)
    og = O.Graph.from_edges(n, s, d, w, 1)
    t = D.sssp.compute(g, 0, D.sssp.Options(cuda_engine=OPS))
    ot, _ = O.compute(og, 0, rule=1)
    _same(t, ot, "compute")
    sched = D.sssp.Schedule(invalidation=walk)
    for rnd in range(4):
        b = random_batch(rng, n, s, d, 600, tree_parents=ot.parents, grow=50 if rnd == 2 else 0)
        st = D.sssp.update(g, _db(b), t, schedule=sched)
        ost, _ = O.update(og, _ob(b), ot)
        assert st.engine_used == OPS
        _same(t, ot, f"{shape} round {rnd}")
        assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"]), rnd
        assert st.invalidation == walk
        assert g.num_vertices() == og.n


def test_engines_agree_on_an_rmat_stream():
    from dyng_b200 import generators as G
    e = G.rmat(14, 8, w_max=1000, seed=9)
    rp, col, w = e.csr()
    gf = D.Graph.from_csr(rp, col, w)
    go = D.Graph.from_csr(rp, col, w)
    tf = D.sssp.compute(gf, 0, D.sssp.Options(cuda_engine="fused"))
    to = D.sssp.compute(go, 0, D.sssp.Options(cuda_engine=OPS))
    _same(to, tf, "compute")
    stream = G.BatchStream(e, seed=4)
    for step in range(4):
        b = stream.next(2000, 0.75, 0.5, parents=tf.parents)
        args = (b.insert_src, b.insert_dst, b.insert_weights, b.delete_src, b.delete_dst)
        sf = D.sssp.update(gf, _batch(*args), tf)
        so = D.sssp.update(go, _batch(*args), to)
        assert (sf.engine_used, so.engine_used) == ("fused", OPS)
        _same(to, tf, f"step {step}")
        assert (so.invalidated, so.affected) == (sf.invalidated, sf.affected)
        np.testing.assert_array_equal(go.to_csr().col_ind, gf.to_csr().col_ind)


def test_large_weights_use_the_distance_only_mode():
    # sssp_cuda_test.cpp:555-620: (n - 1) * 2e9 on a 320 x 320 grid does not fit beside 17 bits
    side = 320
    n = side * side
    rng = np.random.default_rng(31)
    v = np.arange(n)
    x, y = v % side, v // side
    right, down = v[x + 1 < side], v[y + 1 < side]
    src = np.concatenate([right, right + 1, down, down + side]).astype(np.int32)
    dst = np.concatenate([right + 1, right, down + side, down]).astype(np.int32)
    w = np.full(src.size, 2_000_000_000, np.int32)
    g = D.Graph.from_edges(src, dst, w, n)
    og = O.Graph.from_edges(n, src, dst, w, 1)
    t, cst = D.sssp.compute(g, 0, D.sssp.Options(cuda_engine=OPS), stats=True)
    ot, _ = O.compute(og, 0, rule=1)
    assert not cst.packed_parents
    _same(t, ot, "compute")
    for rnd in range(3):
        vv = rng.integers(1, n, 300)
        vv = vv[ot.parents[vv] >= 0]
        a, c = rng.integers(0, n, 300), rng.integers(0, n, 300)
        keep = a != c
        b = (a[keep].astype(np.int32), c[keep].astype(np.int32),
             np.full(int(keep.sum()), 2_000_000_000, np.int32), ot.parents[vv].astype(np.int32),
             vv.astype(np.int32))
        st = D.sssp.update(g, _batch(*b), t)
        ost, _ = O.update(og, _obatch(*b), ot)
        assert not st.packed_parents
        _same(t, ot, f"round {rnd}")
        assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])


def test_packing_boundary_of_47_distance_bits():
    # the path 0 -> ... -> n-1 (n = 2^17 - 1, W = 2^30 + 2^14) plus the back edge n-1 -> 1: the
    # candidate n * W over the back edge must be dropped, not packed
    n = (1 << 17) - 1
    w = (1 << 30) + (1 << 14)
    src = list(range(n - 1)) + [n - 1]
    dst = list(range(1, n)) + [1]
    g = D.Graph.from_edges(src, dst, [w] * len(src), n, D.GraphProperties.mosp_compatible())
    og = O.Graph.from_edges(n, src, dst, [w] * len(src), 1, O.mosp_props())
    t, cst = D.sssp.compute(g, 0, D.sssp.Options(cuda_engine=OPS), stats=True)
    ot, _ = O.compute(og, 0, rule=1)
    assert cst.packed_parents
    _same(t, ot, "compute")
    b = ([n - 2], [n - 1], [w - 1])
    st = D.sssp.update(g, _batch(*b), t)
    ost, _ = O.update(og, _obatch(*b), ot)
    _same(t, ot, "update")
    assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])
    assert t.distances[1] == w


def test_unvalidated_cycle_is_reported_and_poisons():
    g = D.Graph.from_edges([0, 1, 2, 2], [1, 2, 1, 3], [1, 1, 1, 1], 4)
    t = D.sssp.Result.from_arrays(g, 0, [0, 1, 2, 3], [-1, 2, 1, 2], canonicalize=False,
                                  options=D.sssp.Options(validate_inputs=False, cuda_engine=OPS))
    with pytest.raises(D.InvalidArgumentError, match="parent cycle"):
        D.sssp.update(g, _batch(del_src=[2], del_dst=[3]), t)
    assert g.version() == 1
    with pytest.raises(D.StaleResultError):
        t.distances


def test_without_cooperative_launch_automatic_runs_the_operators_engine():
    rng = np.random.default_rng(17)
    n, s, d, w = random_graph(rng, "sparse", 3000)
    res = D.Resources(0)
    g = D.Graph.from_edges(s, d, w, n, resources=res)
    og = O.Graph.from_edges(n, s, d, w, 1)
    ot, _ = O.compute(og, 0, rule=1)
    res.set_test_hooks(no_cooperative_launch=True)
    try:
        with pytest.raises(D.NotSupportedError, match="cooperative launch"):
            D.sssp.compute(g, 0, D.sssp.Options(cuda_engine="fused"))
        t, cst = D.sssp.compute(g, 0, stats=True)
        assert cst.engine_used == OPS
        _same(t, ot, "compute")
        fused = D.sssp.compute(g, 0)  # automatic: the operators engine as well
        fused.set_options(D.sssp.Options(cuda_engine="fused"))
        b = random_batch(rng, n, s, d, 500, tree_parents=ot.parents)
        m0 = g.num_edges()
        with pytest.raises(D.NotSupportedError, match="cooperative launch"):
            D.sssp.update(g, _db(b), fused)
        assert g.version() == 0 and g.num_edges() == m0  # refused before the batch was applied
        for rnd in range(3):
            st = D.sssp.update(g, _db(b), t)
            ost, _ = O.update(og, _ob(b), ot)
            assert st.engine_used == OPS
            _same(t, ot, f"round {rnd}")
            assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"])
            b = random_batch(rng, n, s, d, 500, tree_parents=ot.parents, grow=20)
        # graph.apply alone: the applier as one launch per step
        b = random_batch(rng, n, s, d, 800)
        g.apply(_db(b))
        og.apply(_ob(b))
        csr, want = g.to_csr(), og.to_csr()
        np.testing.assert_array_equal(csr.row_ptr, want["row_ptr"])
        np.testing.assert_array_equal(csr.col_ind, want["col"])
        np.testing.assert_array_equal(csr.weights.reshape(-1), want["w"].reshape(-1))
    finally:
        res.set_test_hooks()
