"""Parity with the oracle at the sizes the benchmark's metric is quoted on.

The smaller cases (tests/test_gpu_parity.py) pin the CUDA path on the reference's goldens and
random shapes; these run the benchmark workloads themselves through the C ABI and compare every
batch with the oracle (bit-exact int64 distances, int32 parents, `invalidated`, `affected` and
the apply summary):

  - directed R-MAT scale 22, edge factor 16, weights uniform in [1, 1000], source 0: ten
    consecutive batches of each size 1k, 10k, 100k and 1M changes (75 % insertions of uniform
    pairs, 25 % deletions, half of them current tree edges), under the plain schedule and under
    the learned scheduler, on two graphs side by side;
  - the 4096 x 4096 grid (bidirectional 4-neighbour edges, 0.1 % shortcuts, lognormal weights,
    source at the centre) with near-source churn batches of 10k and 100k changes (50/50), whose
    deletions cut subtrees spanning most of the grid.

The oracle runs on every host core (its batch application and repair are threaded, with results
identical to its sequential engine, which tests/test_oracle.py checks).
"""
import os

import numpy as np
import pytest

import dyng_b200 as D
from dyng_b200 import generators as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dyng_b200",
                       "data", "scheduler_weights.npz")


def _cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


@pytest.fixture
def oracle_threads():
    O.set_threads(_cores())
    yield
    O.set_threads(1)


def _gpu_batch(b):
    return D.EdgeBatch.from_arrays(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                   b.delete_dst)


def _oracle_batch(b):
    return O.Batch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src, b.delete_dst)


def _check(label, t, st, ot, ost, osm):
    np.testing.assert_array_equal(t.distances, ot.distances, err_msg=label)
    np.testing.assert_array_equal(t.parents, ot.parents, err_msg=label)
    assert (st.invalidated, st.affected) == (ost["invalidated"], ost["affected"]), label
    assert (st.batch.inserted_edges, st.batch.deleted_edges, st.batch.updated_edges,
            st.batch.ignored_deletions) == (osm["inserted_edges"], osm["deleted_edges"],
                                            osm["updated_edges"], osm["ignored_deletions"]), label


def test_rmat_scale22_batch_sweep_matches_the_oracle(oracle_threads):
    from dyng_b200 import scheduler as S
    e = G.rmat(22, 16, w_max=1000, seed=1, device="cuda")
    rp, col, w = e.csr()
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    ot, _ = O.compute(og, 0, rule=1)
    plain_g = D.Graph.from_csr(rp, col, w)
    learned_g = D.Graph.from_csr(rp, col, w)
    plain_t = D.sssp.compute(plain_g, 0)
    np.testing.assert_array_equal(plain_t.distances, ot.distances)
    np.testing.assert_array_equal(plain_t.parents, ot.parents)
    learned_t = D.sssp.compute(learned_g, 0)
    sched = S.Scheduler.load(WEIGHTS, resources=learned_g._res)
    stream = G.BatchStream(e, seed=7)
    for size in (1_000, 10_000, 100_000, 1_000_000):
        for step in range(10):
            b = stream.next(size, 0.75, 0.5, parents=ot.parents)
            ost, osm = O.update(og, _oracle_batch(b), ot)
            st = D.sssp.update(plain_g, _gpu_batch(b), plain_t)
            _check(f"plain {size} step {step}", plain_t, st, ot, ost, osm)
            st = D.sssp.update(learned_g, _gpu_batch(b), learned_t, scheduler=sched)
            _check(f"learned {size} step {step}", learned_t, st, ot, ost, osm)
    assert plain_g.num_edges() == og.m and learned_g.num_edges() == og.m
    # every finite distance of the final tree fits in 31 bits (the int32 claim of the workload)
    d = ot.distances
    assert d[d < O.INF // 2].max() < 2**31


def test_grid_4096_near_source_churn_matches_the_oracle(oracle_threads):
    side = 4096
    source = (side // 2) * side + side // 2
    e = G.grid(side, seed=1)
    rp, col, w = e.csr()
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    ot, _ = O.compute(og, source, rule=1)
    g = D.Graph.from_csr(rp, col, w)
    t = D.sssp.compute(g, source)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)
    churn = G.NearSourceChurn(G.BatchStream(e, seed=7), side, source)
    for step, size in enumerate((10_000, 100_000, 10_000)):
        b = churn.next(size)
        ost, osm = O.update(og, _oracle_batch(b), ot)
        st = D.sssp.update(g, _gpu_batch(b), t)
        _check(f"grid {size} step {step}", t, st, ot, ost, osm)
        # the deletions near the source invalidate most of the grid: the repair is near a full solve
        assert st.invalidated > side * side // 2
