"""The serving loop on the GPU: every request's result in a mix equals the same batches run
alone, in order, on a copy of its graph, with one lane and with large batches on a lane of
their own beside the small rounds (their persistent grids sharing the SMs); rounds group small
batches of different graphs; admission refuses what does not fit; a bad batch fails alone."""
import threading

import numpy as np
import pytest

import dyng_b200 as D
from dyng_b200.serving import Server
from tests.helpers import random_graph, random_batch

pytestmark = pytest.mark.gpu

SHAPES = ("sparse", "hub", "grid", "chain")


def _batch(b):
    return D.EdgeBatch.from_arrays(b["ins_src"], b["ins_dst"], b["ins_w"], b["del_src"],
                                   b["del_dst"])


def _workload(seed, per_graph=12):
    rng = np.random.default_rng(seed)
    graphs = []
    for i, shape in enumerate(SHAPES):
        n, s, d, w = random_graph(rng, shape, 1500 + 500 * i)
        sizes = rng.integers(1, 3000, per_graph)
        sizes[::5] = 20000  # some batches above small_changes: rounds of their own
        batches = [random_batch(rng, n, s, d, int(z)) for z in sizes]
        graphs.append(((n, s, d, w), batches))
    return graphs


def _alone(spec, batches):
    n, s, d, w = spec
    g = D.Graph.from_edges(s, d, w, num_vertices=n)
    t = D.sssp.compute(g, 0)
    out = []
    for b in batches:
        st = D.sssp.update(g, _batch(b), t)
        out.append((st.invalidated, st.affected, st.batch.inserted_edges, st.batch.deleted_edges))
    return out, t.distances, t.parents


@pytest.mark.parametrize("lanes", [1, 2, 4])
@pytest.mark.parametrize("learned", [False, True])
def test_mix_equals_alone(learned, lanes):
    work = _workload(3)
    sched = None
    if learned:
        from dyng_b200 import scheduler as S
        sched = S.Scheduler(seed=11)
        sched.set_params((np.random.default_rng(5).normal(size=S.num_params()) * 0.5)
                         .astype(np.float32))
    server = Server(scheduler=sched, max_group=8, small_changes=10000, lanes=lanes)
    handles, slots = [], []
    for spec, _ in work:
        n, s, d, w = spec
        g = D.Graph.from_edges(s, d, w, num_vertices=n)
        t = D.sssp.compute(g, 0)
        handles.append((g, t))
        slots.append(server.add(g, t))
    results = {}

    def submitter(which):
        # each thread owns some graphs, so each graph's batches arrive in order
        for i in which:
            tickets = [server.submit(slots[i], _batch(b)) for b in work[i][1]]
            results[i] = [server.wait(tk) for tk in tickets]

    threads = [threading.Thread(target=submitter, args=([0, 2],)),
               threading.Thread(target=submitter, args=([1, 3],))]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    info = server.info()
    server.drain()
    for i, (spec, batches) in enumerate(work):
        want, dist, par = _alone(spec, batches)
        got = [(st.invalidated, st.affected, st.batch.inserted_edges, st.batch.deleted_edges)
               for st, _ in results[i]]
        assert got == want
        g, t = handles[i]
        assert np.array_equal(t.distances, dist) and np.array_equal(t.parents, par)
    groups = [tm["group_size"] for i in results for _, tm in results[i]]
    assert info["completed"] == sum(len(b) for _, b in work) and info["failed"] == 0
    lanes_used = [tm["lane"] for i in results for _, tm in results[i]]
    if lanes <= 2:
        assert max(groups) >= 2  # small batches of different graphs shared rounds
    else:
        # small batches of different graphs ran side by side on the small lanes
        assert len({ln for ln in lanes_used if ln < lanes - 1}) >= 2
    assert info["lanes"] == lanes
    if lanes >= 2:
        # the 20000-change batches ran on the large lane (the last), everything else on the
        # small ones
        sizes = [len(b["ins_src"]) + len(b["del_src"]) for _, bs in work for b in bs]
        assert info["large_rounds"] == sum(z > 10000 for z in sizes) > 0
        assert sum(ln == lanes - 1 for ln in lanes_used) == info["large_rounds"]
        assert all((ln == lanes - 1) == (z > 10000) for ln, z in
                   zip([tm["lane"] for i in sorted(results) for _, tm in results[i]],
                       [len(b["ins_src"]) + len(b["del_src"]) for i in sorted(results)
                        for b in work[i][1]]))
    else:
        assert not any(lanes_used) and info["large_rounds"] == 0
    assert all(tm["total_ms"] >= tm["service_ms"] >= 0 for i in results for _, tm in results[i])
    server.close()


def test_admission_and_errors():
    rng = np.random.default_rng(4)
    n, s, d, w = random_graph(rng, "sparse", 1000)
    g = D.Graph.from_edges(s, d, w, num_vertices=n)
    t = D.sssp.compute(g, 0)
    # a reserve larger than the device: the graph is not admitted
    big = Server(hbm_reserve_bytes=1 << 50)
    with pytest.raises(D.OutOfMemoryError):
        big.add(g, t)
    big.close()
    server = Server()
    slot = server.add(g, t)
    with pytest.raises(D.InvalidArgumentError):
        server.submit(slot + 5, _batch(random_batch(rng, n, s, d, 10)))
    bad = server.submit(slot, D.EdgeBatch.from_arrays([-1], [2], [3]))  # negative id
    ok = server.submit(slot, _batch(random_batch(rng, n, s, d, 50)))
    with pytest.raises(D.InvalidArgumentError):
        server.wait(bad)
    st, _ = server.wait(ok)  # the failed batch changed nothing; the next one runs
    assert st.batch.num_vertices_after == n
    server.close()
    assert np.array_equal(t.distances, D.sssp.compute(g, 0).distances)
