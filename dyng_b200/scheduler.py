"""dyng_b200.scheduler: the learned schedule of sssp updates.

A 12 -> 64 -> 64 -> 15 MLP (bf16 weights and activations, fp32 accumulation) whose three heads
pick, per batch, the near-far width class, the invalidation / small-frontier switch and the
persistent-grid size.  Training, inference and feature extraction all run in the library's own
CUDA kernels (dyng_b200/csrc/mlp.cu); this module holds the handle, the class tables, a numpy
restatement of the inference arithmetic (bit-exact with the kernels), the trace recorder and the
trainer.  The schedule changes the order of the work only: distances, parents, ``invalidated`` and
``affected`` are the same under every schedule.

The fixed heuristic -- the automatic width, pointer jumping with the small-frontier switch at 256
vertices, the full occupancy grid -- is class (2, 0, 2) and the fallback when no scheduler is given.

Command line (on a GPU):
    python -m dyng_b200.scheduler record --out traces.npz     # sweep schedules, record timings
    python -m dyng_b200.scheduler train traces.npz --out weights.npz
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .graph import InvalidArgumentError, Resources, check, default_resources

NUM_FEATURES = 12
NUM_OUTPUTS = 15
HEADS = ((0, 8), (8, 4), (12, 3))  # (first logit, classes): width, switch, grid
DEFAULT_CLASSES = (2, 0, 2)
FEATURE_NAMES = (
    "log2_ops", "insert_fraction", "tree_deletion_fraction", "log2_mean_src_degree",
    "log2_max_src_degree", "log2_n", "log2_avg_degree", "log2_auto_delta", "log2_prev_invalidated",
    "log2_prev_frontier0", "log2_prev_frontier_max", "log2_prev_steps")
SWITCH_CLASSES = (  # (invalidation, small_frontier)
    (0, 256), (0, -1), (1, 256), (1, -1))
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
PRETRAINED = os.path.join(DATA_DIR, "scheduler_weights.npz")


def num_params() -> int:
    return int(N.lib().dyngb200_scheduler_num_params())


def param_shapes():
    """(name, shape) of the flat parameter vector, in order."""
    h = 64
    return (("w1", (h, NUM_FEATURES)), ("b1", (h,)), ("w2", (h, h)), ("b2", (h,)),
            ("w3", (NUM_OUTPUTS, h)), ("b3", (NUM_OUTPUTS,)))


def unflatten(params: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shape in param_shapes():
        size = int(np.prod(shape))
        out[name] = params[off:off + size].reshape(shape)
        off += size
    assert off == params.size, "parameter count"
    return out


def all_settings():
    """The 96 (width, switch, grid) class triples the trace recorder sweeps."""
    return [(d, s, g) for d in range(HEADS[0][1]) for s in range(HEADS[1][1])
            for g in range(HEADS[2][1])]


def width_for(cls: int, base: int) -> int:
    """The near-far width of width class `cls` given the automatic width `base` (the kernel's rule)."""
    base = max(int(base), 1)
    if cls >= 2:
        sh = 2 * (cls - 2)
        d = (1 << 40) if base > ((1 << 40) >> sh) else base << sh
    else:
        d = base >> (2 * (2 - cls))
    return max(d, 1)


def grid_for(cls: int, full_grid: int) -> int:
    """Persistent-grid size of grid class `cls` (0: the full occupancy grid)."""
    return 0 if cls == 2 else max(1, int(full_grid) >> (2 - cls))


def schedule_for(classes, base_delta: int, full_grid: int):
    """The explicit Schedule equal to what the device picks for `classes`."""
    from .sssp import Schedule
    d, s, g = classes
    inval, small = SWITCH_CLASSES[s]
    return Schedule(delta=width_for(d, base_delta), grid_blocks=grid_for(g, full_grid),
                    invalidation=inval, small_frontier=small)


# ---- numpy restatement of the device inference (bit-exact) ------------------------------------

def bf16_round(x: np.ndarray) -> np.ndarray:
    """fp32 -> bf16 -> fp32 with round-to-nearest-even (finite inputs)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def reference_forward(params: np.ndarray, mean: np.ndarray, scale: np.ndarray,
                      features: np.ndarray) -> np.ndarray:
    """Logits of raw feature rows with the kernels' arithmetic: standardize in fp32, round the
    input, the weights and each ReLU output to bf16, accumulate bias + sum_i w_i x_i in fp32 in
    input order (every product of two bf16 values is exact in fp32, so fp32 adds reproduce the
    kernels' fused multiply-adds)."""
    p = unflatten(np.asarray(params, np.float32))
    x = np.atleast_2d(np.asarray(features, np.float32))
    xs = (x - np.asarray(mean, np.float32)) * np.asarray(scale, np.float32)
    h = bf16_round(xs)
    for layer, relu in (("1", True), ("2", True), ("3", False)):
        w = bf16_round(p["w" + layer])
        acc = np.broadcast_to(p["b" + layer], (h.shape[0], w.shape[0])).astype(np.float32).copy()
        for i in range(w.shape[1]):
            acc = (acc + (h[:, i:i + 1] * w[None, :, i])).astype(np.float32)
        h = bf16_round(np.maximum(acc, np.float32(0))) if relu else acc
    return h


def within_range(classes: np.ndarray, features: np.ndarray, lo, hi) -> np.ndarray:
    """The classes the update runs with: the plain schedule's where a feature row leaves the
    trained range [lo, hi] (as the inference kernel decides; no range: unchanged)."""
    c = np.array(classes, np.int32, copy=True).reshape(-1, 3)
    if lo is None:
        return c
    x = np.atleast_2d(np.asarray(features, np.float32))
    out = ((x < np.asarray(lo, np.float32)) | (x > np.asarray(hi, np.float32))).any(axis=1)
    c[out] = DEFAULT_CLASSES
    return c


def classes_of(logits: np.ndarray) -> np.ndarray:
    """Per-head argmax (first maximum wins, as in the kernel)."""
    lo = np.atleast_2d(logits)
    return np.stack([np.argmax(lo[:, b:b + n], axis=1) for b, n in HEADS], axis=1).astype(np.int32)


# ---- the device scheduler ---------------------------------------------------------------------

def _f32(a):
    a = np.ascontiguousarray(np.asarray(a, np.float32))
    return a, a.ctypes.data_as(N.c_f32p)


class Scheduler:
    """The learned scheduler on one device: fp32 master weights, their bf16 copies, Adam state."""

    def __init__(self, resources: Resources | None = None, seed: int = 0):
        self._res = resources or default_resources()
        self._h = ctypes.c_void_p()
        check(N.lib().dyngb200_scheduler_create(self._res._h, int(seed), ctypes.byref(self._h)))

    def __del__(self):
        try:
            if getattr(self, "_h", None) and self._h.value:
                N.lib().dyngb200_scheduler_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass

    def get_params(self):
        """(params, feature_mean, feature_scale) as numpy arrays."""
        p = np.zeros(num_params(), np.float32)
        m = np.zeros(NUM_FEATURES, np.float32)
        s = np.zeros(NUM_FEATURES, np.float32)
        check(N.lib().dyngb200_scheduler_get_params(self._res._h, self._h,
                                                    p.ctypes.data_as(N.c_f32p),
                                                    m.ctypes.data_as(N.c_f32p),
                                                    s.ctypes.data_as(N.c_f32p)))
        return p, m, s

    def set_params(self, params=None, feature_mean=None, feature_scale=None) -> None:
        args = []
        keep = []
        for a, n in ((params, num_params()), (feature_mean, NUM_FEATURES),
                     (feature_scale, NUM_FEATURES)):
            if a is None:
                args.append(None)
                continue
            arr, ptr = _f32(a)
            if arr.size != n:
                raise InvalidArgumentError(f"scheduler: expected {n} values, got {arr.size}")
            keep.append(arr)
            args.append(ptr)
        check(N.lib().dyngb200_scheduler_set_params(self._res._h, self._h, *args))

    def set_feature_range(self, lo=None, hi=None) -> None:
        """The raw feature range of the training set: outside it an update keeps the plain
        schedule (stats.schedule_classes == (-2, -2, -2)).  None, None: no range."""
        if lo is None and hi is None:
            check(N.lib().dyngb200_scheduler_set_feature_range(self._h, None, None))
            return
        a, pa = _f32(lo)
        b, pb = _f32(hi)
        if a.size != NUM_FEATURES or b.size != NUM_FEATURES:
            raise InvalidArgumentError("scheduler.set_feature_range: 12 values per bound")
        check(N.lib().dyngb200_scheduler_set_feature_range(self._h, pa, pb))

    def get_feature_range(self):
        lo = np.zeros(NUM_FEATURES, np.float32)
        hi = np.zeros(NUM_FEATURES, np.float32)
        has = ctypes.c_int32()
        check(N.lib().dyngb200_scheduler_get_feature_range(self._h, lo.ctypes.data_as(N.c_f32p),
                                                           hi.ctypes.data_as(N.c_f32p),
                                                           ctypes.byref(has)))
        return (lo, hi) if has.value else (None, None)

    def forward(self, features) -> np.ndarray:
        """Logits (n x 15) of raw feature rows, computed by the device kernels."""
        x, px = _f32(np.atleast_2d(features))
        if x.shape[1] != NUM_FEATURES:
            raise InvalidArgumentError("scheduler.forward: rows of 12 features expected")
        out = np.zeros((x.shape[0], NUM_OUTPUTS), np.float32)
        check(N.lib().dyngb200_scheduler_forward(self._res._h, self._h, px, x.shape[0],
                                                 out.ctypes.data_as(N.c_f32p)))
        return out

    def predict(self, features) -> np.ndarray:
        """The classes updates with these features run with (the trained range applied)."""
        return within_range(classes_of(self.forward(features)), features,
                            *self.get_feature_range())

    def gradients(self, features, labels):
        """(mean loss, gradient of the flat parameters) over all samples, without a step."""
        x, px = _f32(np.atleast_2d(features))
        y = np.ascontiguousarray(np.asarray(labels, np.int32).reshape(-1, 3))
        g = np.zeros(num_params(), np.float32)
        loss = ctypes.c_double()
        check(N.lib().dyngb200_scheduler_gradients(self._res._h, self._h, px,
                                                   y.ctypes.data_as(N.c_i32p), x.shape[0],
                                                   g.ctypes.data_as(N.c_f32p), ctypes.byref(loss)))
        return loss.value, g

    def train(self, features, labels, epochs: int = 200, batch_size: int = 64,
              learning_rate: float = 3e-3, seed: int = 0) -> float:
        """Minibatch Adam on the device; returns the mean loss of the last pass."""
        x, px = _f32(np.atleast_2d(features))
        y = np.ascontiguousarray(np.asarray(labels, np.int32).reshape(-1, 3))
        loss = ctypes.c_double()
        check(N.lib().dyngb200_scheduler_train(self._res._h, self._h, px,
                                               y.ctypes.data_as(N.c_i32p), x.shape[0], int(epochs),
                                               int(batch_size), float(learning_rate), int(seed),
                                               ctypes.byref(loss)))
        return loss.value

    def save(self, path: str, **extra) -> None:
        p, m, s = self.get_params()
        lo, hi = self.get_feature_range()
        rng = {} if lo is None else {"feature_lo": lo, "feature_hi": hi}
        np.savez(path, params=p, feature_mean=m, feature_scale=s, **rng, **extra)

    @classmethod
    def load(cls, path: str = PRETRAINED, resources: Resources | None = None) -> "Scheduler":
        with np.load(path) as z:
            sch = cls(resources)
            sch.set_params(z["params"], z["feature_mean"], z["feature_scale"])
            if "feature_lo" in z.files:
                sch.set_feature_range(z["feature_lo"], z["feature_hi"])
        return sch


def feature_range(features: np.ndarray, margin: float = 0.5):
    """The range of a training set, widened by `margin` (features are log2-scaled counts and
    fractions: 0.5 is a factor 1.4 on a count) or a tenth of the span, whichever is larger."""
    x = np.asarray(features, np.float64)
    lo, hi = x.min(axis=0), x.max(axis=0)
    pad = np.maximum(margin, 0.1 * (hi - lo))
    return (lo - pad).astype(np.float32), (hi + pad).astype(np.float32)


def standardization(features: np.ndarray):
    """Feature mean and scale (1 / std, 1 for constant features) of a training set."""
    x = np.asarray(features, np.float64)
    mean = x.mean(axis=0)
    std = x.std(axis=0)
    scale = np.where(std > 1e-6, 1.0 / np.maximum(std, 1e-6), 1.0)
    return mean.astype(np.float32), scale.astype(np.float32)


# ---- traces: one batch under every schedule ---------------------------------------------------

@dataclass
class Workload:
    """A graph family the recorder sweeps: name, a builder of its edge list, batches to record."""
    name: str
    build: object
    batches: int
    max_batch: int = 1_000_000
    source: int = 0
    churn_side: int = 0  # > 0: a grid of this side, batches churn around the source


def default_workloads():
    from .generators import grid, rmat
    return [
        Workload("rmat-s20-ef16", lambda: rmat(20, 16, w_max=1000, seed=3), 44, 1_000_000),
        Workload("rmat-s21-ef16", lambda: rmat(21, 16, w_max=1000, seed=5), 40, 1_000_000),
        Workload("rmat-s22-ef16", lambda: rmat(22, 16, w_max=1000, seed=1, device="cuda"), 84,
                 1_000_000),
        Workload("grid-2048", lambda: grid(2048, seed=2), 40, 1_000_000),
        Workload("grid-4096-centre", lambda: grid(4096, seed=1), 30, 1_000_000,
                 source=2048 * 4096 + 2048, churn_side=4096),
    ]


def record_traces(workloads=None, seed: int = 11, resources: Resources | None = None,
                  log=print) -> dict:
    """For each workload: build the graph, compute the tree from vertex 0, then for each of its
    seeded batches (sizes log-uniform in [100, max_batch], insertion fraction and tree-deletion
    fraction drawn per batch) snapshot the graph and the tree, run the batch once with the default
    schedule recording the features, once under each of the 96 settings (restoring the snapshot
    before each), and once more with the default schedule, which also advances the stream.
    Times are the library's device times of the update (applier + sssp kernel)."""
    from .graph import EdgeBatch, Graph
    from .generators import BatchStream, NearSourceChurn
    from .sssp import Schedule, compute, update
    res = resources or default_resources()
    workloads = workloads or default_workloads()
    rng = np.random.default_rng(seed)
    settings = all_settings()
    rows = {k: [] for k in ("workload", "size", "insert_fraction", "tree_fraction", "features",
                            "base_delta", "full_grid", "times", "default_times", "affected",
                            "invalidated")}
    for wi, wl in enumerate(workloads):
        edges = wl.build()
        g = Graph.from_csr(*edges.csr(), resources=res)
        tree = compute(g, wl.source)
        g_snap, t_snap = g.clone(), tree.clone()
        stream = BatchStream(edges, seed=seed + 101 * wi)
        churn = NearSourceChurn(stream, wl.churn_side, wl.source) if wl.churn_side else None
        log(f"{wl.name}: n={edges.num_vertices} m={edges.src.size}")
        for bi in range(wl.batches):
            size = int(round(np.exp(rng.uniform(np.log(100), np.log(wl.max_batch)))))
            ins_frac = float(rng.choice([0.0, 0.25, 0.5, 0.75, 1.0, rng.uniform()]))
            tree_frac = float(rng.uniform(0.0, 0.6))
            if churn is not None:
                ins_frac, tree_frac = churn.insert_fraction, 0.0
                b = churn.next(size)
            else:
                b = stream.next(size, insert_fraction=ins_frac, tree_fraction=tree_frac,
                                parents=tree.parents)
            eb = EdgeBatch.from_arrays(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                       b.delete_dst)
            g_snap.copy_from(g)
            t_snap.copy_from(tree)
            st0 = update(g, eb, tree, Schedule(record_features=True))
            times = np.zeros(len(settings), np.float32)
            for k, cls in enumerate(settings):
                g.copy_from(g_snap)
                tree.copy_from(t_snap)
                st = update(g, eb, tree, schedule_for(cls, st0.delta, st0.grid_blocks))
                if st.affected != st0.affected or st.invalidated != st0.invalidated:
                    raise RuntimeError(f"schedule {cls} changed the result of batch {bi}")
                times[k] = st.apply_ms + st.sssp_ms
            g.copy_from(g_snap)
            tree.copy_from(t_snap)
            st1 = update(g, eb, tree)
            rows["workload"].append(wi)
            rows["size"].append(b.size)
            rows["insert_fraction"].append(ins_frac)
            rows["tree_fraction"].append(tree_frac)
            rows["features"].append(np.asarray(st0.features, np.float32))
            rows["base_delta"].append(st0.delta)
            rows["full_grid"].append(st0.grid_blocks)
            rows["times"].append(times)
            rows["default_times"].append((st0.apply_ms + st0.sssp_ms, st1.apply_ms + st1.sssp_ms))
            rows["affected"].append(st0.affected)
            rows["invalidated"].append(st0.invalidated)
            best = int(np.argmin(times))
            log(f"  batch {bi} size {b.size}: default {rows['default_times'][-1][1]:.3f} ms, "
                f"best {times[best]:.3f} ms at {settings[best]}")
        del g_snap, t_snap, tree, g
    out = {k: np.asarray(v) for k, v in rows.items()}
    out["settings"] = np.asarray(settings, np.int32)
    out["workload_names"] = np.asarray([w.name for w in workloads])
    return out


def merge_traces(parts) -> dict:
    """One trace set from several (same 96 settings); workload indices renumbered."""
    settings = np.asarray(parts[0]["settings"])
    out = {}
    names = []
    offset = 0
    for t in parts:
        if not np.array_equal(np.asarray(t["settings"]), settings):
            raise InvalidArgumentError("merge_traces: the trace sets swept different settings")
        for k, v in t.items():
            if k in ("settings", "workload_names"):
                continue
            v = np.asarray(v)
            if k == "workload":
                v = v + offset
            out.setdefault(k, []).append(v)
        names += [str(x) for x in t["workload_names"]]
        offset += len(t["workload_names"])
    merged = {k: np.concatenate(v) for k, v in out.items()}
    merged["settings"] = settings
    merged["workload_names"] = np.asarray(names)
    return merged


def labels_of(traces: dict) -> np.ndarray:
    """Per batch, the classes of its fastest setting."""
    settings = np.asarray(traces["settings"])
    return settings[np.argmin(np.asarray(traces["times"]), axis=1)].astype(np.int32)


def holdout_mask(traces: dict, every: int = 5) -> np.ndarray:
    """Batches held out of training: every `every`-th batch of each workload."""
    w = np.asarray(traces["workload"])
    idx = np.zeros(w.size, np.int64)
    for k in np.unique(w):
        sel = np.nonzero(w == k)[0]
        idx[sel] = np.arange(sel.size)
    return (idx % every) == every - 1


def evaluate(classes: np.ndarray, traces: dict, mask=None) -> dict:
    """Summed device time of the chosen settings against the fixed heuristic and the best."""
    settings = [tuple(s) for s in np.asarray(traces["settings"]).tolist()]
    index = {s: i for i, s in enumerate(settings)}
    times = np.asarray(traces["times"], np.float64)
    sel = np.ones(times.shape[0], bool) if mask is None else np.asarray(mask, bool)
    chosen = np.array([times[r, index[tuple(int(x) for x in classes[r])]]
                       for r in range(times.shape[0])])
    default = times[:, index[DEFAULT_CLASSES]]
    best = times.min(axis=1)
    out = {"batches": int(sel.sum()), "default_ms": float(default[sel].sum()),
           "learned_ms": float(chosen[sel].sum()), "best_ms": float(best[sel].sum())}
    out["gain"] = out["default_ms"] / max(out["learned_ms"], 1e-9)
    out["best_gain"] = out["default_ms"] / max(out["best_ms"], 1e-9)
    return out


def train_on_traces(traces: dict, epochs: int = 400, batch_size: int = 32,
                    learning_rate: float = 2e-3, seed: int = 0, holdout_every: int = 5,
                    resources: Resources | None = None):
    """Train a scheduler on the device on the non-held-out batches; returns it and a report."""
    x = np.asarray(traces["features"], np.float32)
    y = labels_of(traces)
    hold = holdout_mask(traces, holdout_every)
    mean, scale = standardization(x[~hold])
    sch = Scheduler(resources, seed=seed)
    sch.set_params(feature_mean=mean, feature_scale=scale)
    sch.set_feature_range(*feature_range(x[~hold]))
    loss = sch.train(x[~hold], y[~hold], epochs=epochs, batch_size=batch_size,
                     learning_rate=learning_rate, seed=seed)
    pred = sch.predict(x)
    report = {"final_loss": loss, "train": evaluate(pred, traces, ~hold),
              "heldout": evaluate(pred, traces, hold)}
    return sch, report


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m dyng_b200.scheduler")
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("record", help="sweep the 96 settings per batch and record device times")
    r.add_argument("--out", required=True)
    r.add_argument("--seed", type=int, default=11)
    r.add_argument("--scale-batches", type=float, default=1.0,
                   help="multiply every workload's batch count (0.1: a quick run)")
    r.add_argument("--workloads", default="", help="comma-separated names (default: all)")
    mg = sub.add_parser("merge", help="concatenate trace files recorded with the same settings")
    mg.add_argument("inputs", nargs="+")
    mg.add_argument("--out", required=True)
    t = sub.add_parser("train", help="train on recorded traces (on the GPU)")
    t.add_argument("traces")
    t.add_argument("--out", required=True)
    t.add_argument("--epochs", type=int, default=400)
    t.add_argument("--batch-size", type=int, default=32)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    if a.cmd == "merge":
        parts = []
        for path in a.inputs:
            with np.load(path) as z:
                parts.append({k: z[k] for k in z.files})
        np.savez_compressed(a.out, **merge_traces(parts))
        return
    if a.cmd == "record":
        wls = default_workloads()
        if a.workloads:
            keep = set(a.workloads.split(","))
            wls = [w for w in wls if w.name in keep]
        for w in wls:
            w.batches = max(1, int(round(w.batches * a.scale_batches)))
        traces = record_traces(wls, seed=a.seed, log=lambda s: print(s, flush=True))
        np.savez_compressed(a.out, **traces)
        print(json.dumps(evaluate(labels_of(traces), traces)))
    else:
        with np.load(a.traces) as z:
            traces = {k: z[k] for k in z.files}
        sch, report = train_on_traces(traces, a.epochs, a.batch_size, a.lr, a.seed)
        sch.save(a.out)
        print(json.dumps(report))


if __name__ == "__main__":
    main()
