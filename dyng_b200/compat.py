"""python -m dyng_b200.compat: the SOSP part of MOSP's `mosp` driver and `mospPrep init`, on the
B200 path (the reference's tools/compat/mosp/mosp_compat.cpp, update and init modes).

Update mode reads <prefix>{RowPtr,ColInd,Values}.txt, <changes>/insert.txt and delete.txt and
the initial trees <init>/obj<k>/{distancesOriginal,SSSPTreeOriginal}.txt, applies the batch once
to a graph with graph_properties::mosp_compatible() and updates the K trees with update_each,
then writes <out>/obj<k>/{distancesUpdated,SSSPTreeUpdated}.txt in MOSP's format and one report
line per objective ("obj<k> invalidated <n>").  With --mosp it runs the whole MOSP update
(dyng_b200.mosp: the K trees adopted, the batch, the combined graph, the MOSP tree and the path
costs; mosp_compat.cpp:517-640) and also writes <out>/combinedGraph/{distancesCsr,SSSPTreeCsr,
mospCosts}.txt (the costs over every weight column of the graph, as MOSP's driver writes them).
Init mode writes <out>/obj<k>/{distancesOriginal,SSSPTreeOriginal}.txt with sssp.compute().

    python -m dyng_b200.compat --graph <prefix> --changes <dir> --init <dir> [--out dir]
                               [-k K] [--source s] [--delta D] [--canonicalize]
                               [--no-validate-inputs] [--no-output]
                               [--mosp [--pref p1,..,pK] [--no-path-costs]]
    python -m dyng_b200.compat init <prefix> <outDir> [--source s] [-k K]
"""
from __future__ import annotations

import argparse
import os
import sys

from . import mosp_io as io
from .graph import EdgeBatch, Graph, GraphProperties
from .sssp import Options, Result, compute, update_each


def _graph(prefix: str):
    row_ptr, col, w = io.read_csr(prefix)
    k = w.shape[0]
    g = Graph.from_csr(row_ptr, col, w.reshape(-1), GraphProperties.mosp_compatible(),
                       num_weights=k)
    return g, k


def run_update(graph: str, changes: str, init: str, out: str = "mosp-output", k: int | None = None,
               source: int = 0, delta: int = 0, canonicalize: bool = False,
               validate: bool = True, write: bool = True, log=print) -> list:
    g, cols = _graph(graph)
    k = cols if k is None else k
    if not 1 <= k <= cols:
        raise ValueError(f"-k {k}: the graph has {cols} weight column(s)")
    trees = []
    for j in range(k):
        d = io.read_distances(os.path.join(init, f"obj{j}", "distancesOriginal.txt"))
        p = io.read_tree(os.path.join(init, f"obj{j}", "SSSPTreeOriginal.txt"))
        trees.append(Result.from_arrays(g, source, d, p, canonicalize=canonicalize,
                                        options=Options(delta=delta, objective=j,
                                                        validate_inputs=validate)))
    s, t, w, ds, dd = io.read_changes(changes, cols)
    stats = update_each(g, EdgeBatch.from_arrays(s, t, w.reshape(-1), ds, dd, num_weights=cols),
                        trees)
    for j, (tr, st) in enumerate(zip(trees, stats)):
        if write:
            io.write_distances(os.path.join(out, f"obj{j}", "distancesUpdated.txt"), tr.distances)
            io.write_tree(os.path.join(out, f"obj{j}", "SSSPTreeUpdated.txt"), tr.parents)
        log(f"obj{j} invalidated {st.invalidated}")
    return stats


def run_mosp(graph: str, changes: str, init: str, out: str = "mosp-output", k: int | None = None,
             source: int = 0, delta: int = 0, canonicalize: bool = False, validate: bool = True,
             write: bool = True, pref=(), path_costs: bool = True, log=print):
    """The whole MOSP update (mosp_compat.cpp:517-640); returns the mosp.Stats."""
    from . import mosp
    g, cols = _graph(graph)
    k = cols if k is None else k
    if not 1 <= k <= cols:
        raise ValueError(f"-k {k}: the graph has {cols} weight column(s)")
    ds, ps = [], []
    for j in range(k):
        ds.append(io.read_distances(os.path.join(init, f"obj{j}", "distancesOriginal.txt")))
        ps.append(io.read_tree(os.path.join(init, f"obj{j}", "SSSPTreeOriginal.txt")))
    r = mosp.Result.from_arrays(g, source, ds, ps, canonicalize=canonicalize,
                                options=mosp.Options(preferences=list(pref), delta=delta,
                                                     validate_inputs=validate, num_objectives=k,
                                                     compute_path_costs=path_costs and write))
    s, t, w, dd, de = io.read_changes(changes, cols)
    st = mosp.update(g, EdgeBatch.from_arrays(s, t, w.reshape(-1), dd, de, num_weights=cols), r)
    for j, o in enumerate(st.objectives):
        if write:
            io.write_distances(os.path.join(out, f"obj{j}", "distancesUpdated.txt"),
                               r.distances(j))
            io.write_tree(os.path.join(out, f"obj{j}", "SSSPTreeUpdated.txt"), r.parents(j))
        log(f"obj{j} invalidated {o.invalidated}")
    if write:
        cd = os.path.join(out, "combinedGraph")
        io.write_distances(os.path.join(cd, "distancesCsr.txt"), r.combined_distances)
        io.write_tree(os.path.join(cd, "SSSPTreeCsr.txt"), r.combined_parents)
        if path_costs:
            io.write_path_costs(os.path.join(cd, "mospCosts.txt"),
                                r.path_costs if k == cols else r.path_costs_over(cols))
    log(f"combined: L={st.preference_scale} edges {st.combined_edges} affected {st.affected}")
    return st


def run_init(graph: str, out: str, k: int | None = None, source: int = 0) -> None:
    g, cols = _graph(graph)
    k = cols if k is None else k
    for j in range(k):
        r = compute(g, source, Options(objective=j))
        io.write_distances(os.path.join(out, f"obj{j}", "distancesOriginal.txt"), r.distances)
        io.write_tree(os.path.join(out, f"obj{j}", "SSSPTreeOriginal.txt"), r.parents)


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if argv and argv[0] == "init":
        ap = argparse.ArgumentParser(prog="python -m dyng_b200.compat init")
        ap.add_argument("graph")
        ap.add_argument("out")
        ap.add_argument("--source", type=int, default=0)
        ap.add_argument("-k", type=int, default=None)
        a = ap.parse_args(argv[1:])
        run_init(a.graph, a.out, a.k, a.source)
        return 0
    ap = argparse.ArgumentParser(prog="python -m dyng_b200.compat")
    ap.add_argument("--graph", required=True)
    ap.add_argument("--changes", required=True)
    ap.add_argument("--init", required=True)
    ap.add_argument("--out", default="mosp-output")
    ap.add_argument("-k", type=int, default=None)
    ap.add_argument("--source", type=int, default=0)
    ap.add_argument("--delta", type=int, default=0)
    ap.add_argument("--canonicalize", action="store_true")
    ap.add_argument("--no-validate-inputs", action="store_true")
    ap.add_argument("--no-output", action="store_true")
    ap.add_argument("--mosp", action="store_true", help="the whole MOSP update and combinedGraph/")
    ap.add_argument("--pref", default="", help="with --mosp: preferences p1,..,pK")
    ap.add_argument("--no-path-costs", action="store_true")
    a = ap.parse_args(argv)
    if a.mosp:
        pref = [int(x) for x in a.pref.split(",")] if a.pref else []
        run_mosp(a.graph, a.changes, a.init, a.out, a.k, a.source, a.delta, a.canonicalize,
                 not a.no_validate_inputs, not a.no_output, pref, not a.no_path_costs)
        return 0
    run_update(a.graph, a.changes, a.init, a.out, a.k, a.source, a.delta, a.canonicalize,
               not a.no_validate_inputs, not a.no_output)
    return 0


if __name__ == "__main__":
    sys.exit(main())
