"""ctypes wrapper of the CPU oracle (oracle/sssp_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and by the
cpu_baseline / ``--impl reference`` legs of bench.py, always as the checker or as the timed CPU
restatement of the reference, never as part of the product path.

The oracle restates dynG's host path (cpp/src/graph/apply_host.cpp:57-518,
cpp/src/algorithms/sssp/sequential.cpp:57-381, cpp/src/algorithms/sssp/sssp.cpp:136-165,
377-460, 563-576, 643-689) and mosp's finalize step (cpp/src/algorithms/mosp/sequential.cpp:33-232,
mosp.cpp:108-131, 259-301) in plain C.  Its parity with the reference is pinned by
tests/test_oracle.py against the reference's golden fixtures (tests/golden/).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
INF = (2**63 - 1) // 4  # sssp_infinity (cpp/src/algorithms/sssp/problem.hpp:340-341)

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class Props(ctypes.Structure):
    """graph_properties + batch_semantics (cpp/include/dyng/graph/graph_properties.hpp:67-241)."""

    _fields_ = [
        ("directed", ctypes.c_int),
        ("sorted", ctypes.c_int),
        ("allow_multi", ctypes.c_int),
        ("on_existing_insert", ctypes.c_int),
        ("on_missing_delete", ctypes.c_int),
        ("on_self_loop", ctypes.c_int),
        ("deletions_first", ctypes.c_int),
        ("allow_vertex_growth", ctypes.c_int),
    ]


def default_props(**kw) -> Props:
    """The default graph_properties: directed, sorted rows, a simple graph, upsert_last_wins."""
    p = Props(1, 1, 0, 0, 0, 0, 1, 1)
    for k, v in kw.items():
        setattr(p, k, int(v))
    return p


def mosp_props(**kw) -> Props:
    """graph_properties::mosp_compatible(): append order, parallel edges allowed."""
    p = Props(1, 0, 1, 0, 0, 0, 1, 1)
    for k, v in kw.items():
        setattr(p, k, int(v))
    return p


class Summary(ctypes.Structure):
    """apply_summary (cpp/include/dyng/graph/apply_summary.hpp)."""

    _fields_ = [(name, ctypes.c_int64) for name in (
        "inserted_edges", "deleted_edges", "updated_edges", "ignored_insertions",
        "ignored_deletions", "dropped_self_loops", "inserted_vertices", "num_vertices_after")]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class Stats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in (
        "invalidated", "affected", "iterations", "epochs", "pushes", "packed_parents", "delta",
        "max_weight")]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class OracleError(RuntimeError):
    pass


def build() -> str:
    """Compile oracle/liboracle.so (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
                os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "sssp_oracle.c"))):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_graph_from_edges.restype = ctypes.c_void_p
        L.orc_graph_from_edges.argtypes = [ctypes.c_int64, ctypes.c_int64, _i32p, _i32p, _i32p,
                                           ctypes.c_int, ctypes.POINTER(Props), ctypes.c_char_p,
                                           ctypes.c_size_t]
        L.orc_graph_from_csr.restype = ctypes.c_void_p
        L.orc_graph_from_csr.argtypes = [ctypes.c_int64, _i64p, _i32p, _i32p, ctypes.c_int,
                                         ctypes.POINTER(Props), ctypes.c_char_p, ctypes.c_size_t]
        L.orc_graph_free.argtypes = [ctypes.c_void_p]
        L.orc_graph_num_vertices.restype = ctypes.c_int64
        L.orc_graph_num_vertices.argtypes = [ctypes.c_void_p]
        L.orc_graph_num_edges.restype = ctypes.c_int64
        L.orc_graph_num_edges.argtypes = [ctypes.c_void_p]
        L.orc_graph_export.argtypes = [ctypes.c_void_p, _i64p, _i32p, _i32p, _i64p, _i32p, _i32p]
        L.orc_graph_num_changes.restype = ctypes.c_int64
        L.orc_graph_num_changes.argtypes = [ctypes.c_void_p, _i64p]
        L.orc_graph_delta.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p, _u8p]
        L.orc_graph_apply.restype = ctypes.c_int
        L.orc_graph_apply.argtypes = [ctypes.c_void_p, ctypes.c_int64, _i32p, _i32p, _i32p,
                                      ctypes.c_int64, _i32p, _i32p, ctypes.POINTER(Summary),
                                      ctypes.c_char_p, ctypes.c_size_t]
        L.orc_sssp_compute.restype = ctypes.c_int
        L.orc_sssp_compute.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int,
                                       ctypes.c_int64, ctypes.c_int, _i64p, _i32p,
                                       ctypes.POINTER(Stats), ctypes.c_char_p, ctypes.c_size_t]
        L.orc_sssp_update.restype = ctypes.c_int
        L.orc_sssp_update.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int,
                                      ctypes.c_int64, ctypes.c_int, ctypes.c_int64, _i32p, _i32p,
                                      _i32p, ctypes.c_int64, _i32p, _i32p, _i64p, _i32p,
                                      ctypes.POINTER(Stats), ctypes.POINTER(Summary),
                                      ctypes.c_char_p, ctypes.c_size_t]
        L.orc_canonicalize.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int, _i64p, _i32p]
        L.orc_validate_tree.restype = ctypes.c_int
        L.orc_validate_tree.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int, _i64p,
                                        _i32p, ctypes.c_char_p, ctypes.c_size_t]
        L.orc_default_delta.restype = ctypes.c_int64
        L.orc_default_delta.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]
        L.orc_packs_parents.restype = ctypes.c_int
        L.orc_packs_parents.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        L.orc_distances_fit.restype = ctypes.c_int
        L.orc_distances_fit.argtypes = [ctypes.c_int64, ctypes.c_int64]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        L.orc_mosp_combine.restype = ctypes.c_int64
        L.orc_mosp_combine.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int, _i32p, _i32p,
                                       ctypes.c_int32, _i32p, _i32p, _i32p, _i64p]
        L.orc_mosp_path_costs.restype = ctypes.c_int32
        L.orc_mosp_path_costs.argtypes = [ctypes.c_void_p, _i32p, ctypes.c_int32, ctypes.c_int,
                                          _i64p]
        _lib = L
    return _lib


def _p32(a):
    return a.ctypes.data_as(_i32p) if a is not None and a.size else None


def _p64(a):
    return a.ctypes.data_as(_i64p) if a is not None and a.size else None


def _arr32(x, n=None):
    a = np.ascontiguousarray(np.asarray(x if x is not None else [], dtype=np.int32).ravel())
    return a


@dataclass
class Batch:
    """An edge batch (edge_batch_view, cpp/include/dyng/graph/edge_batch.hpp:38-76):
    insertion weights are insertion-major (num_weights per insertion)."""

    insert_src: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    insert_dst: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    insert_weights: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    delete_src: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    delete_dst: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    num_weights: int = 1

    def normalized(self) -> "Batch":
        return Batch(_arr32(self.insert_src), _arr32(self.insert_dst), _arr32(self.insert_weights),
                     _arr32(self.delete_src), _arr32(self.delete_dst), self.num_weights)


class Graph:
    """A host CSR graph of the oracle (owns an orc_graph handle)."""

    def __init__(self, handle, k):
        self._h = handle
        self.k = k

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_graph_free(self._h)
            self._h = None

    @staticmethod
    def from_edges(n, src, dst, weights, num_weights=1, props=None) -> "Graph":
        props = props or default_props()
        s, d, w = _arr32(src), _arr32(dst), _arr32(weights)
        err = ctypes.create_string_buffer(256)
        h = lib().orc_graph_from_edges(n, s.size, _p32(s), _p32(d), _p32(w), num_weights,
                                       ctypes.byref(props), err, 256)
        if not h:
            raise OracleError(err.value.decode())
        return Graph(h, num_weights)

    @staticmethod
    def from_csr(row_ptr, col, weights_objective_major, num_weights=1, props=None) -> "Graph":
        props = props or default_props()
        rp = np.ascontiguousarray(np.asarray(row_ptr, dtype=np.int64))
        c, w = _arr32(col), _arr32(weights_objective_major)
        err = ctypes.create_string_buffer(256)
        h = lib().orc_graph_from_csr(rp.size - 1, _p64(rp), _p32(c), _p32(w), num_weights,
                                     ctypes.byref(props), err, 256)
        if not h:
            raise OracleError(err.value.decode())
        return Graph(h, num_weights)

    @property
    def n(self) -> int:
        return int(lib().orc_graph_num_vertices(self._h))

    @property
    def m(self) -> int:
        return int(lib().orc_graph_num_edges(self._h))

    def to_csr(self):
        n, m, k = self.n, self.m, self.k
        rp = np.zeros(n + 1, np.int64)
        col = np.zeros(m, np.int32)
        w = np.zeros(m * k, np.int32)
        irp = np.zeros(n + 1, np.int64)
        icol = np.zeros(m, np.int32)
        iw = np.zeros(m * k, np.int32)
        lib().orc_graph_export(self._h, _p64(rp), _p32(col), _p32(w), _p64(irp), _p32(icol),
                               _p32(iw))
        return {"row_ptr": rp, "col": col, "w": w.reshape(k, m) if k else w,
                "in_row_ptr": irp, "in_col": icol, "in_w": iw.reshape(k, m) if k else iw}

    def delta(self):
        nd = ctypes.c_int64(0)
        ni = int(lib().orc_graph_num_changes(self._h, ctypes.byref(nd)))
        nd = nd.value
        a = [np.zeros(ni, np.int32), np.zeros(ni, np.int32), np.zeros(nd, np.int32),
             np.zeros(nd, np.int32)]
        inc = np.zeros(ni * self.k, np.uint8)
        lib().orc_graph_delta(self._h, _p32(a[0]), _p32(a[1]), _p32(a[2]), _p32(a[3]),
                              inc.ctypes.data_as(_u8p) if inc.size else None)
        return {"insert_src": a[0], "insert_dst": a[1], "delete_src": a[2], "delete_dst": a[3],
                "weight_increased": inc.reshape(ni, self.k) if self.k else inc}

    def apply(self, batch: Batch) -> dict:
        b = batch.normalized()
        sm = Summary()
        err = ctypes.create_string_buffer(256)
        st = lib().orc_graph_apply(self._h, b.insert_src.size, _p32(b.insert_src),
                                   _p32(b.insert_dst), _p32(b.insert_weights), b.delete_src.size,
                                   _p32(b.delete_src), _p32(b.delete_dst), ctypes.byref(sm), err,
                                   256)
        if st != 0:
            raise OracleError(err.value.decode())
        return sm.as_dict()


class Tree:
    """An sssp::result held by the oracle: int64 distances, int32 parents."""

    def __init__(self, source, distances, parents, objective=0, delta=0, rule=0):
        self.source = int(source)
        self.distances = distances
        self.parents = parents
        self.objective = objective
        self.delta = delta
        self.rule = rule


def compute(g: Graph, source: int, objective: int = 0, delta: int = 0, rule: int = 0):
    """sssp::compute (the Dijkstra tree with lowest-id ties). rule 0 = host packing rule
    (sequential/OpenMP backends), rule 1 = the CUDA engines' packing rule."""
    n = g.n
    d = np.zeros(n, np.int64)
    p = np.zeros(n, np.int32)
    st = Stats()
    err = ctypes.create_string_buffer(256)
    rc = lib().orc_sssp_compute(g._h, source, objective, delta, rule, _p64(d), _p32(p),
                                ctypes.byref(st), err, 256)
    if rc != 0:
        raise OracleError(err.value.decode())
    return Tree(source, d, p, objective, delta, rule), st.as_dict()


def update(g: Graph, batch: Batch, tree: Tree):
    """sssp::update: applies the batch to g and repairs tree in place; returns (stats, summary)."""
    b = batch.normalized()
    n_cap = g.n
    if b.insert_src.size:
        n_cap = max(n_cap, int(max(b.insert_src.max(), b.insert_dst.max())) + 1)
    d = np.full(n_cap, INF, np.int64)
    p = np.full(n_cap, -1, np.int32)
    d[:tree.distances.size] = tree.distances
    p[:tree.parents.size] = tree.parents
    st = Stats()
    sm = Summary()
    err = ctypes.create_string_buffer(256)
    rc = lib().orc_sssp_update(g._h, tree.source, tree.objective, tree.delta, tree.rule,
                               b.insert_src.size, _p32(b.insert_src), _p32(b.insert_dst),
                               _p32(b.insert_weights), b.delete_src.size, _p32(b.delete_src),
                               _p32(b.delete_dst), _p64(d), _p32(p), ctypes.byref(st),
                               ctypes.byref(sm), err, 256)
    if rc != 0:
        raise OracleError(err.value.decode())
    n = g.n
    tree.distances = d[:n].copy()
    tree.parents = p[:n].copy()
    return st.as_dict(), sm.as_dict()


def from_arrays(g: Graph, source, distances, parents, canonicalize=True, objective=0,
                validate=True, delta=0, rule=0) -> Tree:
    """sssp::result::from_arrays (sssp.cpp:1118-1197): normalise INF, optional canonicalisation
    and validation."""
    d = np.ascontiguousarray(np.asarray(distances, dtype=np.int64)).copy()
    p = np.ascontiguousarray(np.asarray(parents, dtype=np.int32)).copy()
    if np.any((p < -1) | (p >= g.n)):
        raise OracleError("parent outside [-1, n)")
    d[d >= INF // 2] = INF
    if canonicalize:
        lib().orc_canonicalize(g._h, source, objective, _p64(d), _p32(p))
    if validate:
        err = ctypes.create_string_buffer(256)
        if lib().orc_validate_tree(g._h, source, objective, _p64(d), _p32(p), err, 256) != 0:
            raise OracleError(err.value.decode())
    return Tree(source, d, p, objective, delta, rule)


def default_delta(m, n, weight_sum) -> int:
    return int(lib().orc_default_delta(m, n, weight_sum))


def packs_parents(n, max_weight, rule=0) -> bool:
    return bool(lib().orc_packs_parents(n, max_weight, rule))


def preference_scale(preferences, num_objectives: int) -> int:
    """L = lcm(preferences), 1 for none (mosp.cpp:108-131); each >= 1, L <= 2^20."""
    if not preferences:
        return 1
    if len(preferences) != num_objectives:
        raise OracleError("one preference per objective")
    scale = 1
    for p in preferences:
        if int(p) < 1:
            raise OracleError("a preference must be >= 1")
        scale = scale // np.gcd(scale, int(p)) * int(p)
        if scale > 1 << 20:
            raise OracleError("lcm(preferences) exceeds 2^20")
    return int(scale)


@dataclass
class MospTree:
    distances: np.ndarray   # combined distances, in units of 1/L
    parents: np.ndarray     # the MOSP tree
    costs: np.ndarray       # n x columns path costs (INF where unreachable)
    combined_edges: int
    scale: int


def mosp_finalize(g: Graph, source: int, parents, preferences=None, cost_columns=None) -> MospTree:
    """Steps 2-3 of MOSP_Update on K trees of g (mosp.cpp:259-301): the combined graph, its tree
    (sssp::compute with lowest-id ties) and the path costs over the first `cost_columns` weight
    columns (K by default)."""
    K = len(parents)
    n = g.n
    L = preference_scale(preferences, K)
    terms = np.asarray([L if not preferences else L // int(p) for p in (preferences or [1] * K)],
                       np.int32)
    base = int(L * (K + 1))
    par = np.ascontiguousarray(np.stack([np.asarray(p, np.int32) for p in parents]))
    cap = max(1, K * n)
    src, dst, w = (np.zeros(cap, np.int32) for _ in range(3))
    wsum = ctypes.c_int64(0)
    m = int(lib().orc_mosp_combine(n, int(source), K, _p32(par), _p32(terms), base, _p32(src),
                                   _p32(dst), _p32(w), ctypes.byref(wsum)))
    cg = Graph.from_edges(n, src[:m], dst[:m], w[:m], 1)
    tree, _ = compute(cg, int(source), rule=1)
    C = K if cost_columns is None else int(cost_columns)
    costs = np.zeros(max(1, n * C), np.int64)
    missing = int(lib().orc_mosp_path_costs(g._h, _p32(tree.parents), int(source), C,
                                            _p64(costs)))
    if missing >= 0:
        raise OracleError(f"the MOSP tree edge ({int(tree.parents[missing])}, {missing}) is not "
                          "an edge of the graph")
    return MospTree(tree.distances, tree.parents, costs[:n * C].reshape(n, C), m, L)


def set_threads(threads: int) -> int:
    """Threads of the oracle's parallel loops (CSR assembly, transposition); 1 = sequential.
    Results are identical for every count.  Returns the count in effect."""
    lib().orc_set_threads(int(threads))
    return int(lib().orc_get_threads())
