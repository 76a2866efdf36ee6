"""dyng_b200.sssp: dynamic single-source shortest paths on B200 (mirrors the reference's
python/dyng/sssp.py: Options, Stats, Result, compute, update, INFINITE_DISTANCE).

:func:`compute` builds the canonical shortest-path tree (ties to the lowest parent id);
:func:`update` applies an edge batch to the device-resident graph and repairs the tree.  The
distances, parents, ``invalidated`` and ``affected`` equal the reference's sequential backend bit
for bit (cpp/include/dyng/sssp.hpp:23-73).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .graph import (DEVICE, HOST, ApplySummary, EdgeBatch, Graph, InvalidArgumentError, check,
                    _ptr32, _ptr64)

INFINITE_DISTANCE: int = (2**63 - 1) // 4

_ENGINES = {"automatic": 0, "fused": 1, "operators": 2}


@dataclass
class Options:
    """sssp::options (sssp.hpp:78-94)."""

    delta: int = 0
    objective: int = 0
    cuda_engine: str = "automatic"
    validate_inputs: bool = True

    def _to_native(self) -> N.Options:
        if self.cuda_engine not in _ENGINES:
            raise InvalidArgumentError(f"unknown cuda_engine {self.cuda_engine!r}")
        return N.Options(int(self.delta), int(self.objective), _ENGINES[self.cuda_engine],
                         int(bool(self.validate_inputs)))


@dataclass
class Schedule:
    """The schedule of one update (what the learned scheduler picks; never changes results)."""

    delta: int = 0
    grid_blocks: int = 0
    invalidation: int = 0
    small_frontier: int = 0
    heavy_degree: int = 0
    record_features: bool = False  # report the learned scheduler's features in the stats

    def _to_native(self) -> N.Schedule:
        return N.Schedule(int(self.delta), int(self.grid_blocks), int(self.invalidation),
                          int(self.small_frontier), int(self.heavy_degree),
                          int(bool(self.record_features)))


class Stats:
    """sssp::stats (sssp.hpp:100-117) plus the schedule that ran and the device times.

    A view of the native stats record: fields are converted when first read, so an update pays
    no Python conversion for the fields its caller never looks at."""

    WORK_NAMES = ("round_visits", "jumps", "invalidated", "pull_candidates", "pull_slots",
                  "pull_words", "pushes", "push_slots", "push_words", "atomics", "appends",
                  "unpacked", "atomic_attempts", "step0_max_warp_ns", "step0_sum_warp_ns",
                  "step0_warps", "step0_light_ns", "step0_medium_ns", "step0_heavy_ns",
                  "step0_max_light_ns", "step0_max_medium_ns", "step0_max_heavy_ns",
                  "pj_seeded", "pull_atomics", "pull_appends", "pair_visits", "walk_rows",
                  "walk_slots", "stamps_scanned")
    # Algorithmic bytes per unit of work (4-byte ids / weights, 8-byte packed words and rows):
    #   pointer-jumping visit 8 (ancestor + flag), jump 12 (ancestor[a], flag[a], write),
    #   invalidated vertex 12 (word set to INF, candidate entry), pull candidate / pushed vertex
    #   20 (list entry, row descriptor, own word), row slot 8 (column + weight), word read 8,
    #   successful atomicMin 8, frontier append 12 (entry + stamp), compared vertex 20 (word, old
    #   distance and parent), seeded vertex 12 (stamp, parent, ancestor written), change pair 16
    #   (list entry, flags, key), walk row 12 (entry, descriptor), walk slot 8 (column, parent),
    #   scanned change stamp 4; attempted atomics and the balance probes are diagnostics (0 bytes).
    WORK_BYTES = ((8, 12, 12, 20, 8, 8, 20, 8, 8, 8, 12, 20) + (0,) * 10 +
                  (12, 8, 12, 16, 12, 8, 4) + (0,) * 3)
    # The work counters of each phase of the kernel (indices into WORK_NAMES), and the phases'
    # device times (indices into PHASES): the per-phase roofline.
    PHASE_WORK = {"roots_heads": ((25,), (0, 3)),
                  "invalidation": ((0, 1, 2, 22, 26, 27), (1, 2)),
                  "pull": ((3, 4, 5, 23, 24), (4,)),
                  "near_far": ((6, 7, 8, 9, 10), (5,)),
                  "unpack": ((11, 28), (6,))}
    PHASES = ("roots", "invalidation", "invalidate_scan", "heads", "pull", "near_far", "unpack")
    _SCALARS = ("invalidated", "affected", "iterations", "epochs", "pushes", "delta",
                "max_weight", "grid_blocks", "invalidation", "rounds", "touched",
                "kernel_launches")

    __slots__ = ("_s",)

    def __init__(self, native: N.Stats | None = None):
        self._s = native if native is not None else N.Stats()

    @classmethod
    def _from_native(cls, s: N.Stats) -> "Stats":
        return cls(s)

    def __getattr__(self, name):
        if name in Stats._SCALARS:
            return int(getattr(self._s, name))
        raise AttributeError(name)

    @property
    def batch(self) -> ApplySummary:
        return ApplySummary._from_native(self._s.batch)

    @property
    def packed_parents(self) -> bool:
        return bool(self._s.packed_parents)

    @property
    def engine_used(self) -> str:
        engines = {v: k for k, v in _ENGINES.items()}
        return engines.get(self._s.engine_used, "fused")

    @property
    def apply_ms(self) -> float:
        return float(self._s.apply_ms)

    @property
    def sssp_ms(self) -> float:
        return float(self._s.sssp_ms)

    @property
    def work(self) -> tuple:
        return tuple(int(x) for x in self._s.work)

    @property
    def phase_ms(self) -> tuple:
        return tuple(float(x) for x in self._s.phase_ms)

    @property
    def trace(self) -> tuple:
        """(light, heavy chunks, start us) per near-far step; light < 0: an epoch."""
        s = self._s
        return tuple((int(s.trace_light[i]), int(s.trace_heavy[i]), float(s.trace_us[i]))
                     for i in range(min(int(s.trace_len), 64)))

    @property
    def pj_rounds_us(self) -> tuple:
        """Start of each pointer-jumping round (us since the kernel began)."""
        return tuple(float(self._s.pj_round_us[i]) for i in range(min(int(self._s.rounds), 24)))

    @property
    def pj_done_us(self) -> tuple:
        """The last block's arrival at the barrier ending each pointer-jumping round (us)."""
        return tuple(float(self._s.pj_done_us[i]) for i in range(min(int(self._s.rounds), 24)))

    @property
    def apply_step_us(self) -> tuple:
        """The batch applier kernel: the end of each step (us since it began; 0: not reached)."""
        return tuple(float(x) for x in self._s.apply_step_us)

    @property
    def host_us(self) -> tuple:
        """Host time of the call (us): checks and staging, queuing the applier, queuing the sssp
        kernel and the read-back, waiting for the device."""
        return tuple(float(x) for x in self._s.host_us)

    @property
    def features(self) -> tuple:
        return tuple(float(x) for x in self._s.features)

    @property
    def schedule_classes(self) -> tuple:
        return tuple(int(x) for x in self._s.schedule_classes)

    @property
    def algorithmic_bytes(self) -> int:
        return int(sum(a * b for a, b in zip(self.work, self.WORK_BYTES)))

    # The reference's profiler stages (parity/timed_regions/sssp.toml) -> this update's device
    # times: the commit is the batch applier (the in-edge mirror is kept in place inside it, so
    # graph.transpose has no time of its own), and the sssp kernel's phases map onto the stages
    # of the update's Steps 1 and 2.
    STAGES = {"sssp.identify_affected": (0, 1, 2), "sssp.seed": (3, 4), "sssp.loop": (5,),
              "sssp.finalize": (6,)}

    def stages_ms(self) -> dict:
        """Device time (ms) under the reference's profiler stage names (sssp.update >
        sssp.commit > graph.apply, sssp.identify_affected, sssp.seed, sssp.loop, sssp.finalize)."""
        ms = self.phase_ms
        out = {"sssp.update": self.apply_ms + self.sssp_ms, "sssp.commit": self.apply_ms,
               "graph.apply": self.apply_ms, "graph.transpose": 0.0}
        for name, phases in self.STAGES.items():
            out[name] = float(sum(ms[i] for i in phases))
        return out

    def phase_bytes_ms(self) -> dict:
        """Per phase of the kernel: (algorithmic bytes, device ms).  The unpack also counts the
        12 bytes it writes per affected vertex."""
        work, ms = self.work, self.phase_ms
        out = {}
        for name, (units, phases) in self.PHASE_WORK.items():
            b = sum(work[i] * self.WORK_BYTES[i] for i in units)
            if name == "unpack":
                b += 12 * self.affected
            out[name] = (int(b), float(sum(ms[i] for i in phases)))
        return out

    def __repr__(self):
        return (f"Stats(invalidated={self.invalidated}, affected={self.affected}, "
                f"iterations={self.iterations}, epochs={self.epochs}, delta={self.delta}, "
                f"apply_ms={self.apply_ms:.3f}, sssp_ms={self.sssp_ms:.3f})")


class Result:
    """sssp::result: int64 distances and int32 parents in device memory (sssp.hpp:153-310)."""

    def __init__(self, handle, graph: Graph):
        self._h = handle
        self._graph = graph
        self._res = graph._res

    def __del__(self):
        try:
            if getattr(self, "_h", None) and self._h.value:
                N.lib().dyngb200_tree_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass

    def _info(self):
        src, n, ver, poisoned = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_uint64(), ctypes.c_int32()
        opt = N.Options()
        check(N.lib().dyngb200_tree_info(self._h, ctypes.byref(src), ctypes.byref(n),
                                         ctypes.byref(ver), ctypes.byref(poisoned),
                                         ctypes.byref(opt)))
        return src.value, n.value, ver.value, bool(poisoned.value), opt

    @property
    def source(self) -> int:
        return self._info()[0]

    @property
    def graph_version(self) -> int:
        return self._info()[2]

    @property
    def poisoned(self) -> bool:
        return self._info()[3]

    @property
    def distances(self) -> np.ndarray:
        n = self._info()[1]
        out = np.zeros(n, np.int64)
        check(N.lib().dyngb200_tree_distances(self._res._h, self._h, _ptr64(out), HOST))
        return out

    @property
    def parents(self) -> np.ndarray:
        n = self._info()[1]
        out = np.zeros(n, np.int32)
        check(N.lib().dyngb200_tree_parents(self._res._h, self._h, _ptr32(out), HOST))
        return out

    def device_arrays(self):
        """Raw device pointers (int64 distances, int32 parents), valid until the next update."""
        d, p = N.c_i64p(), N.c_i32p()
        check(N.lib().dyngb200_tree_device_arrays(self._h, ctypes.byref(d), ctypes.byref(p)))
        return ctypes.cast(d, ctypes.c_void_p).value, ctypes.cast(p, ctypes.c_void_p).value

    @property
    def options(self) -> Options:
        o = self._info()[4]
        engines = {v: k for k, v in _ENGINES.items()}
        return Options(o.delta, o.objective, engines.get(o.cuda_engine, "automatic"),
                       bool(o.validate_inputs))

    def set_options(self, options: Options) -> None:
        o = options._to_native()
        check(N.lib().dyngb200_tree_set_options(self._h, ctypes.byref(o)))

    def clone(self) -> "Result":
        h = ctypes.c_void_p()
        check(N.lib().dyngb200_tree_clone(self._res._h, self._h, ctypes.byref(h)))
        return Result(h, self._graph)

    def copy_from(self, other: "Result") -> None:
        """Take other's distances, parents and history; this result stays bound to its graph."""
        check(N.lib().dyngb200_tree_copy_from(self._res._h, self._h, other._h))

    @classmethod
    def from_arrays(cls, graph: Graph, source: int, distances, parents, canonicalize: bool = True,
                    options: Options | None = None) -> "Result":
        d = np.ascontiguousarray(np.asarray(distances, dtype=np.int64))
        p = np.ascontiguousarray(np.asarray(parents, dtype=np.int32))
        if d.size != p.size:
            raise InvalidArgumentError("from_arrays: distances and parents differ in length")
        o = (options or Options())._to_native()
        h = ctypes.c_void_p()
        check(N.lib().dyngb200_tree_from_arrays(graph._res._h, graph._h, source, _ptr64(d),
                                                _ptr32(p), d.size, HOST, int(canonicalize),
                                                ctypes.byref(o), ctypes.byref(h)))
        return cls(h, graph)


def compute(graph: Graph, source: int = 0, options: Options | None = None,
            stats: bool = False):
    """sssp::compute(resources::cuda(), g, source, opt) (sssp.hpp:415-421)."""
    o = (options or Options())._to_native()
    h = ctypes.c_void_p()
    st = N.Stats()
    check(N.lib().dyngb200_sssp_compute(graph._res._h, graph._h, int(source), ctypes.byref(o),
                                        ctypes.byref(h), ctypes.byref(st)))
    r = Result(h, graph)
    return (r, Stats._from_native(st)) if stats else r


def update_each(graph: Graph, batch: EdgeBatch, results) -> list:
    """dyng::update_each (update.hpp:331) for sssp results: the batch is applied once and every
    result (e.g. one per objective) is updated; one Stats per result, in order."""
    results = list(results)
    nb = batch._to_native()
    handles = (ctypes.c_void_p * max(len(results), 1))(*[r._h.value for r in results])
    out = (N.Stats * max(len(results), 1))()
    check(N.lib().dyngb200_sssp_update_each(graph._res._h, graph._h, ctypes.byref(nb), handles,
                                            len(results), out))
    return [Stats(out[i]) for i in range(len(results))]


def update(graph: Graph, batch: EdgeBatch, tree: Result, schedule: Schedule | None = None,
           scheduler=None) -> Stats:
    """sssp::update(resources::cuda(), g, batch, tree) (sssp.hpp:484-489).

    ``schedule`` fixes the schedule; ``scheduler`` (a :class:`dyng_b200.scheduler.Scheduler`)
    picks it on the device for this batch.  Neither changes the results."""
    nb = batch._to_native()
    st = N.Stats()
    if scheduler is not None:
        if schedule is not None:
            raise InvalidArgumentError("update: give a schedule or a scheduler, not both")
        check(N.lib().dyngb200_sssp_update_learned(graph._res._h, graph._h, ctypes.byref(nb),
                                                   tree._h, scheduler._h, ctypes.byref(st)))
    elif schedule is None:
        check(N.lib().dyngb200_sssp_update(graph._res._h, graph._h, ctypes.byref(nb), tree._h,
                                           ctypes.byref(st)))
    else:
        sc = schedule._to_native()
        check(N.lib().dyngb200_sssp_update_scheduled(graph._res._h, graph._h, ctypes.byref(nb),
                                                     tree._h, ctypes.byref(sc), ctypes.byref(st)))
    return Stats._from_native(st)
