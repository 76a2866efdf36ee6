"""The learned scheduler on the GPU: its kernels against the numpy restatement (inference,
bit-exact) and a torch fp32 reference (gradients), training, the device features, and updates
under the learned schedule against plain updates (bit-exact)."""
import numpy as np
import pytest

from tests.helpers import random_graph, random_batch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def D():
    import dyng_b200
    return dyng_b200


def _batch(D, b):
    return D.EdgeBatch.from_arrays(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"],
                                   b["del_dst"])


def _random_features(rng, n):
    x = rng.normal(size=(n, 12)).astype(np.float32) * 3 + 5
    return x


def test_forward_bit_exact_with_numpy(D):
    from dyng_b200 import scheduler as S
    rng = np.random.default_rng(1)
    sch = S.Scheduler(seed=3)
    x = _random_features(rng, 300)
    mean, scale = S.standardization(x)
    params = (rng.normal(size=S.num_params()) * 0.3).astype(np.float32)
    sch.set_params(params, mean, scale)
    got = sch.forward(x)
    want = S.reference_forward(params, mean, scale, x)
    assert np.array_equal(got, want)
    assert np.array_equal(sch.predict(x), S.classes_of(want))
    p, m, s = sch.get_params()
    assert np.array_equal(p, params) and np.array_equal(m, mean) and np.array_equal(s, scale)


def _torch_loss_and_grad(params, mean, scale, x, y):
    import torch
    from dyng_b200 import scheduler as S
    P = torch.tensor(params, dtype=torch.float32, requires_grad=True)
    parts, off = {}, 0
    for name, shape in S.param_shapes():
        size = int(np.prod(shape))
        parts[name] = P[off:off + size].reshape(shape)
        off += size

    def bfr(t):  # bf16 rounding with a straight-through gradient
        return t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()

    xs = (torch.tensor(x) - torch.tensor(mean)) * torch.tensor(scale)
    h = bfr(xs)
    h1 = bfr(torch.relu(h @ bfr(parts["w1"]).T + parts["b1"]))
    h2 = bfr(torch.relu(h1 @ bfr(parts["w2"]).T + parts["b2"]))
    lo = h2 @ bfr(parts["w3"]).T + parts["b3"]
    yt = torch.tensor(y, dtype=torch.int64)
    loss = 0
    for head, (b, n) in enumerate(S.HEADS):
        loss = loss + torch.nn.functional.cross_entropy(lo[:, b:b + n], yt[:, head])
    loss.backward()
    return float(loss.detach()), P.grad.numpy()


def test_gradients_match_torch_fp32(D):
    from dyng_b200 import scheduler as S
    rng = np.random.default_rng(2)
    sch = S.Scheduler(seed=5)
    x = _random_features(rng, 517)
    y = np.stack([rng.integers(0, n, x.shape[0]) for _, n in S.HEADS], axis=1).astype(np.int32)
    mean, scale = S.standardization(x)
    sch.set_params(feature_mean=mean, feature_scale=scale)
    params = sch.get_params()[0]
    loss, grad = sch.gradients(x, y)
    want_loss, want_grad = _torch_loss_and_grad(params, mean, scale, x, y)
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, abs(want_loss))
    # fp32 sums in a different order: relative 1e-3 of the largest gradient entry
    tol = 1e-3 * float(np.abs(want_grad).max())
    assert np.abs(grad - want_grad).max() <= tol
    assert np.abs(grad).max() > 0


def test_training_learns_a_separable_rule(D):
    from dyng_b200 import scheduler as S
    rng = np.random.default_rng(3)
    x = _random_features(rng, 2000)
    # width class from feature 0, switch class from the sign of feature 1 - 5, grid from feature 2
    y = np.stack([np.clip(((x[:, 0] - 5) / 1.5 + 4).astype(int), 0, 7),
                  (x[:, 1] > 5).astype(int) * 2,
                  np.clip(((x[:, 2] - 5) / 2 + 1).astype(int), 0, 2)], axis=1).astype(np.int32)
    sch = S.Scheduler(seed=1)
    mean, scale = S.standardization(x)
    sch.set_params(feature_mean=mean, feature_scale=scale)
    loss0, _ = sch.gradients(x, y)
    loss = sch.train(x, y, epochs=60, batch_size=64, learning_rate=3e-3, seed=2)
    assert loss < 0.5 * loss0
    acc = (sch.predict(x) == y).mean(axis=0)
    assert acc[1] > 0.97 and acc[0] > 0.8 and acc[2] > 0.85


def _expected_features(n, m, src_deg, ins, dels, tree_dels, delta, hist):
    ops = ins + dels
    lg = lambda v: np.float32(np.log2(1.0 + max(v, 0)))  # noqa: E731
    f = [lg(ops), ins / ops if ops else 0.0, tree_dels / dels if dels else 0.0,
         lg(np.mean(src_deg) if len(src_deg) else 0.0), lg(max(src_deg) if len(src_deg) else 0),
         lg(n), lg(m / n), lg(delta), lg(hist[0]), lg(abs(hist[1])), lg(abs(hist[2])), lg(hist[3])]
    return np.asarray(f, np.float32)


def test_device_features_of_a_hand_case(D):
    # path 0 -> 1 -> 2 -> 3 plus 0 -> 2 (weight 5) and 1 -> 3 (weight 7); the tree from 0 uses the
    # path edges; the batch deletes tree edge 1 -> 2 and non-tree edge 0 -> 2 and inserts 3 -> 0
    src = np.array([0, 1, 2, 0, 1], np.int32)
    dst = np.array([1, 2, 3, 2, 3], np.int32)
    w = np.array([1, 1, 1, 5, 7], np.int32)
    g = D.Graph.from_edges(src, dst, w, num_vertices=4)
    tree = D.sssp.compute(g, 0)
    b = D.EdgeBatch.from_arrays([3], [0], [2], [1, 0], [2, 2])
    st = D.sssp.update(g, b, tree, schedule=D.sssp.Schedule(record_features=True))
    got = np.asarray(st.features, np.float32)
    # the history is that of compute(): nothing invalidated
    assert got[8] == 0.0
    # out-degrees of the sources 3, 1, 0 before the batch: 0, 2, 2
    want = _expected_features(4, 5, [0, 2, 2], 1, 2, 1, st.delta, (0, 0, 0, 0))
    assert np.allclose(got[:8], want[:8], rtol=1e-6, atol=1e-6), (got, want)
    # a second update sees the first one's record: one tree edge deleted invalidated 2 vertices
    st2 = D.sssp.update(g, D.EdgeBatch.from_arrays([1], [2], [1]), tree,
                        schedule=D.sssp.Schedule(record_features=True))
    assert st2.features[8] == pytest.approx(np.log2(1 + st.invalidated))
    assert st2.features[11] == pytest.approx(np.log2(1 + st.iterations + st.epochs))


def test_learned_updates_equal_plain_updates(D):
    from dyng_b200 import scheduler as S
    rng = np.random.default_rng(9)
    n, s, d, w = random_graph(rng, "sparse", 3000)
    g1 = D.Graph.from_edges(s, d, w, num_vertices=n)
    g2 = D.Graph.from_edges(s, d, w, num_vertices=n)
    t1 = D.sssp.compute(g1, 0)
    t2 = D.sssp.compute(g2, 0)
    sch = S.Scheduler(seed=4)
    seen = set()
    for step in range(24):
        # random weights give a spread of classes
        sch.set_params((rng.normal(size=S.num_params()) * 0.5).astype(np.float32))
        b = _batch(D, random_batch(rng, n, s, d, 2 + int(rng.integers(0, 2000)),
                                   tree_parents=t1.parents))
        st1 = D.sssp.update(g1, b, t1)
        st2 = D.sssp.update(g2, b, t2, scheduler=sch)
        assert np.array_equal(t1.distances, t2.distances)
        assert np.array_equal(t1.parents, t2.parents)
        assert (st1.invalidated, st1.affected) == (st2.invalidated, st2.affected)
        cls = st2.schedule_classes
        assert all(0 <= c < nh for c, (_, nh) in zip(cls, S.HEADS))
        # the schedule that ran is the one the classes name
        want = S.schedule_for(cls, st1.delta, st1.grid_blocks)
        assert st2.delta == want.delta
        assert st2.grid_blocks == (want.grid_blocks or st1.grid_blocks)
        seen.add(tuple(cls))
        # the device's choice equals the numpy restatement on the device's own features
        p, m, sc = sch.get_params()
        assert tuple(S.classes_of(S.reference_forward(p, m, sc, np.asarray(st2.features)))[0]) \
            == tuple(cls)
    assert len(seen) >= 3


def test_outside_its_trained_range_the_scheduler_keeps_the_plain_schedule(D):
    from dyng_b200 import scheduler as S
    rng = np.random.default_rng(12)
    n, s, d, w = random_graph(rng, "sparse", 2000)
    g1 = D.Graph.from_edges(s, d, w, num_vertices=n)
    g2 = D.Graph.from_edges(s, d, w, num_vertices=n)
    t1, t2 = D.sssp.compute(g1, 0), D.sssp.compute(g2, 0)
    sch = S.Scheduler(seed=5)
    sch.set_params((rng.normal(size=S.num_params()) * 0.5).astype(np.float32))
    # a range that excludes this graph's size feature (log2(1 + n) ~ 11)
    lo = np.full(12, -100, np.float32)
    hi = np.full(12, 100, np.float32)
    hi[5] = 5.0
    sch.set_feature_range(lo, hi)
    assert np.array_equal(sch.get_feature_range()[1], hi)
    for step in range(3):
        b = _batch(D, random_batch(rng, n, s, d, 500, tree_parents=t1.parents))
        st1 = D.sssp.update(g1, b, t1)
        st2 = D.sssp.update(g2, b, t2, scheduler=sch)
        assert tuple(st2.schedule_classes) == (-2, -2, -2)
        assert (st2.delta, st2.grid_blocks) == (st1.delta, st1.grid_blocks)
        assert np.array_equal(t1.distances, t2.distances)
        assert np.array_equal(t1.parents, t2.parents)
    # inside the range it chooses again
    sch.set_feature_range(None, None)
    st2 = D.sssp.update(g2, _batch(D, random_batch(rng, n, s, d, 500, tree_parents=t2.parents)),
                        t2, scheduler=sch)
    assert all(c >= 0 for c in st2.schedule_classes)


def test_snapshot_restore_replays_a_batch(D):
    rng = np.random.default_rng(12)
    n, s, d, w = random_graph(rng, "hub", 2000)
    g = D.Graph.from_edges(s, d, w, num_vertices=n)
    tree = D.sssp.compute(g, 0)
    gs, ts = g.clone(), tree.clone()
    b = _batch(D, random_batch(rng, n, s, d, 800, tree_parents=tree.parents))
    st_a = D.sssp.update(g, b, tree)
    dist_a, par_a, csr_a = tree.distances, tree.parents, g.to_csr()
    g.copy_from(gs)
    tree.copy_from(ts)
    assert g.version() == gs.version()
    st_b = D.sssp.update(g, b, tree, schedule=D.sssp.Schedule(delta=7, invalidation=1))
    assert np.array_equal(dist_a, tree.distances) and np.array_equal(par_a, tree.parents)
    csr_b = g.to_csr()
    assert all(np.array_equal(x, y) for x, y in zip(csr_a, csr_b))
    assert (st_a.invalidated, st_a.affected) == (st_b.invalidated, st_b.affected)
