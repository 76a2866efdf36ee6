"""Small workloads that run each kernel family of the library a few times, for profiling with ncu
(one kernel per capture: ``ncu -k regex:<kernel> -c <n> python -m dyng_b200.profile_cases <case>``).

Cases (each a few GB of device memory at most, inputs larger than L2 where the kernel streams):

  operators    R-MAT scale 20, compute and four 100k-change updates with the operators engine
               (``k_op_*``, the applier as ``k_apply_step``)
  maintenance  R-MAT scale 18 under a stream of insertion-heavy batches until the arenas have
               grown, been compacted and the edge index rebuilt (``k_index_*``, ``k_compact_*``),
               then a deletion of the only maximum-weight edge (``k_rescan_*``)
  multigraph   a graph with parallel edges allowed (the applier's row scans instead of the index)
  canonicalize an imported tree canonicalised and repacked (``k_canonicalize``, ``k_pack``)
  mlp          the learned scheduler trained for a few epochs on the shipped traces
               (``k_mlp_grad``, ``k_adam``, ``k_refresh_bf16``, ``k_mlp_forward``)

Every case checks its own result (against a from-scratch compute, or the training loss) and
exits non-zero on a mismatch.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np


def _check(ok: bool, what: str) -> None:
    if not ok:
        print(f"profile_cases: {what} failed", file=sys.stderr)
        sys.exit(1)


def _same_as_compute(D, g, t, source=0, options=None):
    fresh = D.sssp.compute(g, source, options)
    return bool(np.array_equal(fresh.distances, t.distances) and
                np.array_equal(fresh.parents, t.parents))


def case_operators(D, G):
    e = G.rmat(20, 16, w_max=1000, seed=1)
    rp, col, w = e.csr()
    g = D.Graph.from_csr(rp, col, w)
    opt = D.sssp.Options(cuda_engine="operators")
    t = D.sssp.compute(g, 0, opt)
    stream = G.BatchStream(e, seed=7)
    for _ in range(4):
        b = stream.next(100_000, 0.75, 0.5, parents=t.parents)
        st = D.sssp.update(g, D.EdgeBatch.from_arrays(b.insert_src, b.insert_dst,
                                                      b.insert_weights, b.delete_src,
                                                      b.delete_dst), t)
        _check(st.engine_used == "operators", "engine")
    _check(_same_as_compute(D, g, t, 0, opt), "operators update vs compute")


def case_maintenance(D, G):
    e = G.rmat(18, 16, w_max=1000, seed=2)
    rp, col, w = e.csr()
    g = D.Graph.from_csr(rp, col, w)
    t = D.sssp.compute(g, 0)
    n = g.num_vertices()
    rng = np.random.default_rng(5)
    for step in range(40):
        st = g.storage()
        if st["compactions"] >= 1 and st["arena_growths"] >= 1 and st["index_builds"] >= 2:
            break
        ni, nd = 400_000, 100_000
        csr = g.to_csr()
        rows = rng.integers(0, n, nd)
        has = csr.row_ptr[rows] < csr.row_ptr[rows + 1]
        du = rows[has].astype(np.int32)
        dv = csr.col_ind[csr.row_ptr[du]].astype(np.int32)
        b = D.EdgeBatch.from_arrays(rng.integers(0, n, ni).astype(np.int32),
                                    rng.integers(0, n, ni).astype(np.int32),
                                    rng.integers(1, 1000, ni, endpoint=True).astype(np.int32),
                                    du, dv)
        D.sssp.update(g, b, t)
    st = g.storage()
    print({k: st[k] for k in ("compactions", "arena_growths", "index_builds")})
    _check(_same_as_compute(D, g, t), "maintenance update vs compute")
    # the only edge of the maximum weight deleted: the column statistics are rescanned
    D.sssp.update(g, D.EdgeBatch.from_arrays([1], [2], [1_000_000], [], []), t)
    D.sssp.update(g, D.EdgeBatch.from_arrays([], [], [], [1], [2]), t)
    t2 = D.sssp.compute(g, 0)
    _check(_same_as_compute(D, g, t2), "after rescan")


def case_multigraph(D, G):
    e = G.rmat(18, 16, w_max=1000, seed=3)
    props = D.GraphProperties(allow_multi=True)
    g = D.Graph.from_edges(e.src, e.dst, e.weights, e.num_vertices, props)
    t = D.sssp.compute(g, 0)
    stream = G.BatchStream(e, seed=8)
    for _ in range(4):
        b = stream.next(50_000, 0.75, 0.5, parents=t.parents)
        D.sssp.update(g, D.EdgeBatch.from_arrays(b.insert_src, b.insert_dst, b.insert_weights,
                                                 b.delete_src, b.delete_dst), t)
    _check(_same_as_compute(D, g, t), "multigraph update vs compute")


def case_canonicalize(D, G):
    e = G.rmat(20, 16, w_max=1000, seed=4)
    rp, col, w = e.csr()
    g = D.Graph.from_csr(rp, col, w)
    t = D.sssp.compute(g, 0)
    for _ in range(3):
        imp = D.sssp.Result.from_arrays(g, 0, t.distances, t.parents, canonicalize=True)
        _check(bool(np.array_equal(imp.parents, t.parents)), "canonicalize")


def case_mlp(D, G):
    from dyng_b200 import scheduler as S
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                        "scheduler_traces.npz")
    with np.load(path) as z:
        traces = {k: z[k] for k in z.files}
    sch, report = S.train_on_traces(traces, epochs=3, batch_size=32, learning_rate=2e-3, seed=0)
    print(report)
    _check(sch is not None, "training")


CASES = {"operators": case_operators, "maintenance": case_maintenance,
         "multigraph": case_multigraph, "canonicalize": case_canonicalize, "mlp": case_mlp}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m dyng_b200.profile_cases")
    ap.add_argument("case", choices=sorted(CASES))
    a = ap.parse_args(argv)
    import dyng_b200 as D
    from dyng_b200 import generators as G
    CASES[a.case](D, G)
    print(f"profile_cases {a.case}: ok")


if __name__ == "__main__":
    main()
