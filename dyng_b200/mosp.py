"""dyng_b200.mosp: dynamic multi-objective shortest paths (the reference's dyng.mosp,
python/dyng/mosp.py, over cpp/include/dyng/mosp.hpp).

A graph with K weight columns and a source: the K canonical shortest-path trees (sssp results of
the first K columns), the combined graph they span (an edge of m of the trees weighs
L (K + 1) - sum of L / Pref_i over those trees, L = lcm(Pref)), its shortest-path tree (the MOSP
tree) and the K objective values of every MOSP path.  update() applies a batch once, updates the
K trees (dyng::update_each) and solves the combined graph again, all on the device; the path
costs are copied to host memory, as the reference keeps them.

    r = mosp.compute(g, 0, preferences=[4, 1, 4])
    st = mosp.update(g, batch, r)
    r.combined_parents, r.path_costs
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field, replace

import numpy as np

from . import _native as N
from .graph import ApplySummary, EdgeBatch, Graph, InvalidArgumentError, check
from .sssp import Result as _SsspResult
from .sssp import Stats as _SsspStats

HOST, DEVICE = 0, 1


@dataclass
class Options:
    """mosp::options (mosp.hpp:79-101)."""

    preferences: list = field(default_factory=list)
    delta: int = 0
    compute_path_costs: bool = True
    validate_inputs: bool = True
    num_objectives: int = 0

    def _to_native(self):
        prefs = [int(p) for p in self.preferences]
        arr = (ctypes.c_int32 * max(len(prefs), 1))(*prefs)
        o = N.MospOptions(int(self.num_objectives), len(prefs),
                          ctypes.cast(arr, ctypes.POINTER(ctypes.c_int32)) if prefs else None,
                          int(self.delta), int(bool(self.compute_path_costs)),
                          int(bool(self.validate_inputs)))
        return o, arr  # the array must outlive the call


@dataclass(frozen=True)
class Stats:
    """mosp::stats (mosp.hpp:115-125): the batch, `affected` (vertices whose combined distance or
    MOSP parent changed), the combined graph's edges, L, and the K sssp updates."""

    affected: int
    iterations: int
    converged: bool
    batch: ApplySummary
    objectives: tuple
    combined_edges: int
    preference_scale: int
    combine_ms: float
    solve_ms: float
    costs_ms: float


class _Tree(_SsspResult):
    """The sssp tree of one objective, owned by its mosp result (never destroyed here)."""

    def __init__(self, handle, graph: Graph, owner: "Result"):
        super().__init__(handle, graph)
        self._owner = owner

    def __del__(self):
        pass


class Result:
    """mosp::result (mosp.hpp:138-348): the K trees, the MOSP tree and the path costs."""

    def __init__(self, handle, graph: Graph, options: Options):
        self._h = handle
        self._graph = graph
        self._res = graph._res
        self._options = options

    def __del__(self):
        try:
            if getattr(self, "_h", None) and self._h.value:
                N.lib().dyngb200_mosp_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass

    def _info(self):
        k, n, scale, src, ver = (ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64(),
                                 ctypes.c_int32(), ctypes.c_uint64())
        check(N.lib().dyngb200_mosp_info(self._h, ctypes.byref(k), ctypes.byref(n),
                                         ctypes.byref(scale), ctypes.byref(src), ctypes.byref(ver)))
        return k.value, n.value, scale.value, src.value, ver.value

    @property
    def num_objectives(self) -> int:
        return self._info()[0]

    @property
    def preference_scale(self) -> int:
        return self._info()[2]

    @property
    def source(self) -> int:
        return self._info()[3]

    @property
    def graph_version(self) -> int:
        return self._info()[4]

    @property
    def options(self) -> Options:
        return replace(self._options)

    def tree(self, objective: int) -> _SsspResult:
        """The sssp result of one objective (owned by this result)."""
        h = ctypes.c_void_p()
        check(N.lib().dyngb200_mosp_tree(self._h, int(objective), ctypes.byref(h)))
        return _Tree(h, self._graph, self)

    def distances(self, objective: int) -> np.ndarray:
        return self.tree(objective).distances

    def parents(self, objective: int) -> np.ndarray:
        return self.tree(objective).parents

    @property
    def combined_distances(self) -> np.ndarray:
        """Distances in the combined graph, in units of 1/L (INF if unreachable)."""
        n = self._info()[1]
        out = np.zeros(n, np.int64)
        check(N.lib().dyngb200_mosp_combined(self._h, out.ctypes.data_as(N.c_i64p) if n else None,
                                             None, HOST))
        return out

    @property
    def combined_parents(self) -> np.ndarray:
        """The MOSP tree (-1 for the source and unreachable vertices)."""
        n = self._info()[1]
        out = np.zeros(n, np.int32)
        check(N.lib().dyngb200_mosp_combined(self._h, None,
                                             out.ctypes.data_as(N.c_i32p) if n else None, HOST))
        return out

    @property
    def path_costs(self) -> np.ndarray:
        """n x K objective values of every MOSP path (INF if unreachable)."""
        k, n = self._info()[:2]
        out = np.zeros((n, k), np.int64)
        check(N.lib().dyngb200_mosp_path_costs(self._h,
                                               out.ctypes.data_as(N.c_i64p) if out.size else None))
        return out

    def path_costs_over(self, columns: int) -> np.ndarray:
        """n x columns path costs along the MOSP tree over the graph's first `columns` weight
        columns (MOSP's mospCosts.txt covers every column of the graph)."""
        n = self._info()[1]
        out = np.zeros((n, int(columns)), np.int64)
        check(N.lib().dyngb200_mosp_path_costs_columns(
            self._res._h, self._graph._h, self._h, int(columns),
            out.ctypes.data_as(N.c_i64p) if out.size else None))
        return out

    def set_options(self, options: Options | None = None, **kwargs) -> None:
        opt = replace(options or self._options, **kwargs)
        o, keep = opt._to_native()
        check(N.lib().dyngb200_mosp_set_options(self._h, ctypes.byref(o)))
        self._options = opt

    @classmethod
    def from_arrays(cls, graph: Graph, source: int, distances, parents, canonicalize: bool = True,
                    options: Options | None = None, **kwargs) -> "Result":
        """mosp::result::from_arrays (mosp.hpp:300-347): adopt K trees of `graph`."""
        opt = replace(options or Options(), **kwargs)
        ds = [np.ascontiguousarray(np.asarray(d, np.int64)) for d in distances]
        ps = [np.ascontiguousarray(np.asarray(p, np.int32)) for p in parents]
        if len(ds) != len(ps):
            raise InvalidArgumentError("mosp.Result.from_arrays: as many distance as parent arrays")
        n = ds[0].size if ds else 0
        dp = (N.c_i64p * max(len(ds), 1))(*[d.ctypes.data_as(N.c_i64p) for d in ds])
        pp = (N.c_i32p * max(len(ps), 1))(*[p.ctypes.data_as(N.c_i32p) for p in ps])
        o, keep = opt._to_native()
        h = ctypes.c_void_p()
        check(N.lib().dyngb200_mosp_from_arrays(graph._res._h, graph._h, int(source), len(ds), dp,
                                                pp, n, HOST, int(bool(canonicalize)),
                                                ctypes.byref(o), ctypes.byref(h)))
        return cls(h, graph, opt)


def compute(graph: Graph, source: int, options: Options | None = None, **kwargs) -> Result:
    """mosp::compute (mosp.hpp:444-449): the K trees, the combined graph, the MOSP tree and the
    path costs of `graph` from `source`."""
    opt = replace(options or Options(), **kwargs)
    o, keep = opt._to_native()
    h = ctypes.c_void_p()
    check(N.lib().dyngb200_mosp_compute(graph._res._h, graph._h, int(source), ctypes.byref(o),
                                        ctypes.byref(h)))
    return Result(h, graph, opt)


def update(graph: Graph, batch: EdgeBatch, result: Result) -> Stats:
    """mosp::update (mosp.hpp:502-506): the batch applied once, the K trees updated, the
    combined graph solved again and the path costs recomputed."""
    nb = batch._to_native()
    st = N.MospStats()
    k = result.num_objectives
    per = (N.Stats * max(k, 1))()
    check(N.lib().dyngb200_mosp_update(graph._res._h, graph._h, ctypes.byref(nb), result._h,
                                       ctypes.byref(st), per))
    return Stats(int(st.affected), int(st.iterations), bool(st.converged),
                 ApplySummary._from_native(st.batch),
                 tuple(_SsspStats(per[i]) for i in range(k)), int(st.combined_edges),
                 int(st.preference_scale), float(st.combine_ms), float(st.solve_ms),
                 float(st.costs_ms))


def main(argv=None):
    """python -m dyng_b200.mosp: time mosp.update on a synthetic multi-objective graph.

    A side x side grid (4-neighbour, bidirectional, 0.1% shortcuts; a road-network stand-in) or
    an R-MAT graph with K weight columns U[1,100], source 0, batches of `--batch` changes (half
    insertions, half deletions of live edges), `--steps` timed updates after `--warmup`.  Prints
    one JSON line: per-update ms (p50), the K sssp updates and the finalize stages, and checks the
    result against mosp.compute on the final graph."""
    import argparse
    import json
    import time
    from .generators import BatchStream, grid, rmat
    ap = argparse.ArgumentParser(prog="python -m dyng_b200.mosp")
    ap.add_argument("--graph", default="grid", choices=["grid", "rmat"])
    ap.add_argument("--side", type=int, default=1024)
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("-k", type=int, default=3)
    ap.add_argument("--batch", type=int, default=50_000)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(12345)
    e = grid(a.side, seed=3) if a.graph == "grid" else rmat(a.scale, 16, w_max=100, seed=3)
    w = rng.integers(1, 101, (a.k, e.src.size)).astype(np.int32)
    rp = np.zeros(e.num_vertices + 1, np.int64)
    order = np.lexsort((e.dst, e.src))
    src, dst = e.src[order], e.dst[order]
    np.add.at(rp, src.astype(np.int64) + 1, 1)
    rp = np.cumsum(rp)
    g = Graph.from_csr(rp, dst, w[:, order], num_weights=a.k)
    t0 = time.perf_counter()
    r = compute(g, 0)
    compute_ms = 1000 * (time.perf_counter() - t0)
    stream = BatchStream(e, seed=777)
    lat, parts = [], []
    for step in range(a.warmup + a.steps):
        b = stream.next(a.batch, 0.5, 0.0, parents=None)
        iw = rng.integers(1, 101, b.insert_src.size * a.k).astype(np.int32)
        eb = EdgeBatch.from_arrays(b.insert_src, b.insert_dst, iw, b.delete_src, b.delete_dst,
                                   num_weights=a.k)
        t0 = time.perf_counter()
        st = update(g, eb, r)
        dt = 1000 * (time.perf_counter() - t0)
        if step >= a.warmup:
            lat.append(dt)
            parts.append([sum(o.apply_ms + o.sssp_ms for o in st.objectives),
                          sum(o.sssp_ms for o in st.objectives), st.combine_ms, st.solve_ms,
                          st.costs_ms])
    fresh = compute(g, 0)
    same = bool(np.array_equal(fresh.combined_distances, r.combined_distances) and
                np.array_equal(fresh.combined_parents, r.combined_parents) and
                np.array_equal(fresh.path_costs, r.path_costs))
    p = np.mean(np.array(parts), axis=0)
    print(json.dumps({
        "workload": (f"grid-{a.side}x{a.side}" if a.graph == "grid" else f"rmat-s{a.scale}-ef16")
                    + f"-K{a.k}-w100-batch{a.batch}",
        "vertices": int(e.num_vertices), "edges": int(e.src.size), "K": a.k,
        "update_ms_p50": float(np.percentile(lat, 50)), "update_ms_mean": float(np.mean(lat)),
        "objectives_ms": round(float(p[0]), 3), "objectives_sssp_ms": round(float(p[1]), 3),
        "sssp_ms_per_objective": round(float(p[1]) / a.k, 3),
        "combine_ms": round(float(p[2]), 3), "combined_solve_ms": round(float(p[3]), 3),
        "path_costs_ms": round(float(p[4]), 3), "compute_ms": round(compute_ms, 1),
        "combined_edges": st.combined_edges, "equals_compute": same}), flush=True)


if __name__ == "__main__":
    main()
