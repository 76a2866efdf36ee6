"""Resources, graphs and edge batches over the C ABI (mirrors the reference's python/dyng/graph.py,
batch.py, resources.py and errors.py for the sssp path)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

from . import _native as N

HOST, DEVICE = 0, 1


class DyngError(RuntimeError):
    """Base of the library's errors (cpp/include/dyng/core/error.hpp)."""


class InvalidArgumentError(DyngError, ValueError):
    pass


class NotSupportedError(DyngError):
    pass


class StaleResultError(DyngError):
    pass


class OutOfMemoryError(DyngError, MemoryError):
    pass


class CudaError(DyngError):
    pass


class CapacityError(DyngError):
    pass


class InternalError(DyngError):
    pass


_ERRORS = {1: InvalidArgumentError, 2: NotSupportedError, 3: StaleResultError,
           4: OutOfMemoryError, 5: CudaError, 6: CapacityError, 7: InternalError}


def check(status: int) -> None:
    if status != 0:
        msg = N.lib().dyngb200_last_error_message().decode(errors="replace")
        raise _ERRORS.get(status, DyngError)(msg)


def _ptr32(a):
    return a.ctypes.data_as(N.c_i32p) if a is not None and a.size else None


def _ptr64(a):
    return a.ctypes.data_as(N.c_i64p) if a is not None and a.size else None


def _i32(x):
    return np.ascontiguousarray(np.asarray(x if x is not None else [], dtype=np.int32).ravel())


class Resources:
    """resources::cuda(device): the device, a stream and the pooled workspace."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = ctypes.c_void_p()
        check(N.lib().dyngb200_context_create(device, stream, ctypes.byref(h)))
        self._h = h
        self.device = device

    @staticmethod
    def cuda(device: int = 0) -> "Resources":
        return Resources(device)

    def synchronize(self) -> None:
        check(N.lib().dyngb200_context_synchronize(self._h))

    def set_test_hooks(self, barrier_timeout_ns: int = 0, barrier_extra_arrivals: int = 0,
                       no_cooperative_launch: bool = False, barrier_kernel: int = 0) -> None:
        """Host-side failure injection for tests (dyngb200_test_hooks); no argument clears.
        barrier_kernel: the kernel the phantom arrivals hold up (0 both, 1 the batch applier,
        2 the sssp kernel)."""
        h = N.TestHooks(int(barrier_timeout_ns), int(barrier_extra_arrivals),
                        int(bool(no_cooperative_launch)), int(barrier_kernel))
        check(N.lib().dyngb200_context_set_test_hooks(self._h, ctypes.byref(h)))

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            N.lib().dyngb200_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = None


def default_resources() -> Resources:
    global _default
    if _default is None:
        _default = Resources(0)
    return _default


@dataclass
class GraphProperties:
    """graph_properties + batch_semantics (graph_properties.hpp:67-241)."""

    directed: bool = True
    sorted: bool = True
    allow_multi: bool = False
    on_existing_insert: str = "upsert"  # upsert | error | ignore
    on_missing_delete: str = "ignore"   # ignore | error
    on_self_loop: str = "keep"          # keep | drop | error
    deletions_first: bool = True
    allow_vertex_growth: bool = True
    headroom: float = 0.125

    @classmethod
    def mosp_compatible(cls) -> "GraphProperties":
        return cls(sorted=False, allow_multi=True)

    def _to_native(self) -> N.Props:
        return N.Props(int(self.directed), int(self.sorted), int(self.allow_multi),
                       {"upsert": 0, "error": 1, "ignore": 2}[self.on_existing_insert],
                       {"ignore": 0, "error": 1}[self.on_missing_delete],
                       {"keep": 0, "drop": 1, "error": 2}[self.on_self_loop],
                       int(self.deletions_first), int(self.allow_vertex_growth),
                       float(self.headroom))


@dataclass(frozen=True)
class ApplySummary:
    inserted_edges: int = 0
    deleted_edges: int = 0
    updated_edges: int = 0
    ignored_insertions: int = 0
    ignored_deletions: int = 0
    dropped_self_loops: int = 0
    inserted_vertices: int = 0
    num_vertices_after: int = 0

    @classmethod
    def _from_native(cls, s: N.ApplySummary) -> "ApplySummary":
        return cls(*(int(getattr(s, f)) for f, _ in N.ApplySummary._fields_))


class CSR(NamedTuple):
    row_ptr: np.ndarray
    col_ind: np.ndarray
    weights: np.ndarray  # (num_weights, m), objective-major


class EdgeBatch:
    """An edge batch (edge_batch.hpp:88-404; python/dyng/batch.py): insertions (upserts under the
    default semantics) and deletions.

    ``EdgeBatch(insert=(src, dst[, weights]), delete=(src, dst))`` as in the reference; weights
    of shape (n,) or (n, K) (insertion-major); insertions without weights get weight 1.  Also
    built edge by edge (``insert_edge`` / ``delete_edge``), from flat arrays (``from_arrays``) or
    from device pointers (``device``)."""

    def __init__(self, insert=None, delete=None, *, num_weights: int | None = None):
        self.num_weights = 1 if num_weights is None else int(num_weights)
        self._ins_src, self._ins_dst, self._ins_w = [], [], []
        self._del_src, self._del_dst = [], []
        self._arrays = None
        self._device = None
        if insert is not None or delete is not None:
            ins = tuple(insert) if insert is not None else ((), ())
            dele = tuple(delete) if delete is not None else ((), ())
            if len(ins) not in (2, 3) or len(dele) != 2:
                raise InvalidArgumentError("EdgeBatch: insert is (src, dst[, weights]), delete "
                                           "is (src, dst)")
            s, d = _i32(ins[0]), _i32(ins[1])
            if s.size != d.size:
                raise InvalidArgumentError("EdgeBatch: the insert src and dst differ in length")
            if len(ins) == 3 and ins[2] is not None:
                w = np.asarray(ins[2])
                if w.ndim == 2:
                    if num_weights is None:
                        self.num_weights = int(w.shape[1])
                    if w.shape != (s.size, self.num_weights):
                        raise InvalidArgumentError("EdgeBatch: weights must be (n,) or (n, K)")
                elif w.size != s.size * self.num_weights:
                    raise InvalidArgumentError("EdgeBatch: one weight per insertion expected")
                w = _i32(w.reshape(-1))
            else:
                w = np.ones(s.size * self.num_weights, np.int32)
            ds, dd = _i32(dele[0]), _i32(dele[1])
            if ds.size != dd.size:
                raise InvalidArgumentError("EdgeBatch: the delete src and dst differ in length")
            self._arrays = (s, d, w, ds, dd)

    @property
    def num_insertions(self) -> int:
        return self._device[3] if self._device else self.arrays()[0].size

    @property
    def num_deletions(self) -> int:
        return self._device[6] if self._device else self.arrays()[3].size

    def insert_edge(self, u: int, v: int, weights=(1,)) -> "EdgeBatch":
        w = list(weights) if np.ndim(weights) else [weights]
        if len(w) != self.num_weights:
            raise InvalidArgumentError(f"insert_edge: {len(w)} weights, expected {self.num_weights}")
        self._ins_src.append(u)
        self._ins_dst.append(v)
        self._ins_w.extend(w)
        self._arrays = None
        return self

    def delete_edge(self, u: int, v: int) -> "EdgeBatch":
        self._del_src.append(u)
        self._del_dst.append(v)
        self._arrays = None
        return self

    def clear(self) -> None:
        self.__init__(num_weights=self.num_weights)

    @classmethod
    def from_arrays(cls, insert_src=None, insert_dst=None, insert_weights=None, delete_src=None,
                    delete_dst=None, num_weights: int = 1) -> "EdgeBatch":
        b = cls(num_weights=num_weights)
        b._arrays = (_i32(insert_src), _i32(insert_dst), _i32(insert_weights), _i32(delete_src),
                     _i32(delete_dst))
        return b

    @classmethod
    def device(cls, insert_src: int, insert_dst: int, insert_weights: int, num_insertions: int,
               delete_src: int, delete_dst: int, num_deletions: int,
               num_weights: int = 1) -> "EdgeBatch":
        """A batch whose arrays already live in device memory (raw CUDA pointers)."""
        b = cls(num_weights=num_weights)
        b._device = (insert_src, insert_dst, insert_weights, num_insertions, delete_src,
                     delete_dst, num_deletions)
        return b

    def arrays(self):
        if self._arrays is None:
            self._arrays = (_i32(self._ins_src), _i32(self._ins_dst), _i32(self._ins_w),
                            _i32(self._del_src), _i32(self._del_dst))
        return self._arrays

    def _to_native(self) -> N.Batch:
        if self._device is not None:
            d = self._device
            cast = lambda p: ctypes.cast(ctypes.c_void_p(p), N.c_i32p) if p else None  # noqa: E731
            return N.Batch(cast(d[0]), cast(d[1]), cast(d[2]), d[3], cast(d[4]), cast(d[5]), d[6],
                           self.num_weights, DEVICE)
        s, t, w, ds, dt = self.arrays()
        return N.Batch(_ptr32(s), _ptr32(t), _ptr32(w), s.size, _ptr32(ds), _ptr32(dt), ds.size,
                       self.num_weights, HOST)


class Graph:
    """A device-resident graph<int32, int64, int32> in slack rows (graph.hpp:96-508)."""

    def __init__(self, handle, resources: Resources):
        self._h = handle
        self._res = resources

    def __del__(self):
        try:
            if getattr(self, "_h", None) and self._h.value:
                N.lib().dyngb200_graph_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass

    @classmethod
    def from_edges(cls, src, dst, weights, num_vertices: int | None = None,
                   properties: GraphProperties | None = None, num_weights: int = 1,
                   resources: Resources | None = None) -> "Graph":
        res = resources or default_resources()
        s, d, w = _i32(src), _i32(dst), _i32(weights)
        if num_vertices is None:
            num_vertices = int(max(s.max(initial=-1), d.max(initial=-1))) + 1
        props = (properties or GraphProperties())._to_native()
        h = ctypes.c_void_p()
        check(N.lib().dyngb200_graph_from_edges(res._h, num_vertices, _ptr32(s), _ptr32(d),
                                                _ptr32(w), s.size, num_weights, HOST,
                                                ctypes.byref(props), ctypes.byref(h)))
        return cls(h, res)

    @classmethod
    def from_csr(cls, row_ptr, col_ind, weights, properties: GraphProperties | None = None,
                 num_weights: int = 1, resources: Resources | None = None) -> "Graph":
        """weights objective-major: shape (num_weights, m) or flat."""
        res = resources or default_resources()
        rp = np.ascontiguousarray(np.asarray(row_ptr, dtype=np.int64))
        c, w = _i32(col_ind), _i32(weights)
        props = (properties or GraphProperties())._to_native()
        h = ctypes.c_void_p()
        check(N.lib().dyngb200_graph_from_csr(res._h, rp.size - 1, _ptr64(rp), _ptr32(c),
                                              _ptr32(w), num_weights, HOST, ctypes.byref(props),
                                              ctypes.byref(h)))
        return cls(h, res)

    def _info(self):
        n, m, k, ver = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32(), ctypes.c_uint64()
        check(N.lib().dyngb200_graph_info(self._h, ctypes.byref(n), ctypes.byref(m),
                                          ctypes.byref(k), ctypes.byref(ver)))
        return n.value, m.value, k.value, ver.value

    def num_vertices(self) -> int:
        return self._info()[0]

    def num_edges(self) -> int:
        return self._info()[1]

    def num_weights(self) -> int:
        return self._info()[2]

    def version(self) -> int:
        return self._info()[3]

    def device_bytes(self) -> int:
        b = ctypes.c_int64()
        check(N.lib().dyngb200_graph_device_bytes(self._h, ctypes.byref(b)))
        return b.value

    def storage(self) -> dict:
        """The slack-row storage: arena slots, tops, abandoned slots, growths, compactions."""
        st = N.GraphStorage()
        check(N.lib().dyngb200_graph_storage_get(self._h, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in N.GraphStorage._fields_}

    def clone(self) -> "Graph":
        """A new graph with this graph's contents (results of this graph are not bound to it)."""
        h = ctypes.c_void_p()
        check(N.lib().dyngb200_graph_clone(self._res._h, self._h, ctypes.byref(h)))
        return Graph(h, self._res)

    def copy_from(self, other: "Graph") -> None:
        """Take other's contents; results bound to this graph stay bound to it."""
        check(N.lib().dyngb200_graph_copy_from(self._res._h, self._h, other._h))

    def apply(self, batch: EdgeBatch, classify: bool = False):
        """graph::apply; with classify also the weight-increase mask (insertions x num_weights)."""
        sm = N.ApplySummary()
        nb = batch._to_native()
        if classify:
            mask = np.zeros(max(batch.num_insertions, 1) * batch.num_weights, np.uint8)
            check(N.lib().dyngb200_graph_apply_classified(
                self._res._h, self._h, ctypes.byref(nb), ctypes.byref(sm),
                mask.ctypes.data_as(N.c_u8p)))
            k = batch.num_weights
            return ApplySummary._from_native(sm), mask[:batch.num_insertions * k].reshape(-1, k)
        check(N.lib().dyngb200_graph_apply(self._res._h, self._h, ctypes.byref(nb),
                                           ctypes.byref(sm)))
        return ApplySummary._from_native(sm)

    def to_csr(self, transposed: bool = False) -> CSR:
        n, m, k, _ = self._info()
        rp = np.zeros(n + 1, np.int64)
        col = np.zeros(m, np.int32)
        w = np.zeros(m * k, np.int32)
        if transposed:
            check(N.lib().dyngb200_graph_to_csr(self._res._h, self._h, None, None, None,
                                                _ptr64(rp), _ptr32(col), _ptr32(w)))
        else:
            check(N.lib().dyngb200_graph_to_csr(self._res._h, self._h, _ptr64(rp), _ptr32(col),
                                                _ptr32(w), None, None, None))
        return CSR(rp, col, w.reshape(k, m))


def device_allocations() -> int:
    """Device allocations the library has made in this process so far."""
    n = ctypes.c_int64()
    check(N.lib().dyngb200_debug_device_allocations(ctypes.byref(n)))
    return n.value


def fail_device_allocation(nth: int) -> None:
    """The nth device allocation from now fails with OutOfMemoryError (0 disarms): the
    allocation-failure sweeps of the reference's tests/support/failing_allocator.hpp."""
    check(N.lib().dyngb200_debug_fail_device_allocation(int(nth)))
