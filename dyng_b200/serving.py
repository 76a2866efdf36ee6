"""dyng_b200.serving: several resident graphs updated by batches that arrive at any time.

The loop itself is native (dyng_b200/csrc/serve.cu): per-graph FIFO order (every result equals
running the same batches alone, in order), continuous batching of small batches of different
graphs into one round on one stream, large batches on a lane of their own that shares the SMs
with the small rounds (lanes=2, the default), admission by free HBM.  This module is its Python
face and the load generator that measures it:

    python -m dyng_b200.serving --rates 10,100,500,2000 --seconds 5

builds 8 R-MAT graphs (scales 18, 19, 20, 20, 21, 21, 22, 22; edge factor 16; weights 1..1000),
sends Poisson arrivals at each aggregate rate, batch sizes log-uniform in [100, 1M], the target
graph drawn from Zipf(1.1), and prints p50 / p99 latency (submit to result) per rate.
"""
from __future__ import annotations

import ctypes
import threading
import time

import numpy as np

from . import _native as N
from .graph import EdgeBatch, Graph, Resources, check, default_resources
from .sssp import Result, Stats


class Server:
    """A serving loop on one GPU.  Graphs and trees added to it belong to it until close()."""

    def __init__(self, resources: Resources | None = None, scheduler=None, max_group: int = 8,
                 small_changes: int = 65536, hbm_reserve_bytes: int = 1 << 30, lanes: int = 2):
        self._res = resources or default_resources()
        cfg = N.ServerConfig(self._res.device, int(max_group), int(small_changes),
                             int(hbm_reserve_bytes), int(lanes))
        self._h = ctypes.c_void_p()
        self._keep = [scheduler]
        check(N.lib().dyngb200_server_create(ctypes.byref(cfg),
                                             scheduler._h if scheduler is not None else None,
                                             ctypes.byref(self._h)))

    def add(self, graph: Graph, tree: Result) -> int:
        slot = ctypes.c_int32()
        check(N.lib().dyngb200_server_add_graph(self._h, graph._h, tree._h, ctypes.byref(slot)))
        self._keep += [graph, tree]
        return slot.value

    def submit(self, slot: int, batch: EdgeBatch) -> int:
        """Queue a batch for the graph in `slot` (copied: the arrays may be reused at once)."""
        nb = batch._to_native()
        ticket = ctypes.c_uint64()
        check(N.lib().dyngb200_server_submit(self._h, int(slot), ctypes.byref(nb),
                                             ctypes.byref(ticket)))
        return ticket.value

    def wait(self, ticket: int):
        """(Stats, times) of a request; raises its update's error.  times: queued_ms,
        service_ms, total_ms, group_size, begin_ms, round_ms, copy_ms, lane (lanes - 1: the
        large lane)."""
        st = N.Stats()
        tm = N.RequestTimes()
        check(N.lib().dyngb200_server_wait(self._h, int(ticket), ctypes.byref(st),
                                           ctypes.byref(tm)))
        return Stats._from_native(st), {"queued_ms": tm.queued_ms, "service_ms": tm.service_ms,
                                        "total_ms": tm.total_ms, "group_size": tm.group_size,
                                        "begin_ms": tm.begin_ms, "round_ms": tm.round_ms,
                                        "copy_ms": tm.copy_ms, "lane": tm.lane}

    def drain(self) -> None:
        check(N.lib().dyngb200_server_drain(self._h))

    def info(self) -> dict:
        i = N.ServerInfo()
        check(N.lib().dyngb200_server_info_get(self._h, ctypes.byref(i)))
        return {n: int(getattr(i, n)) for n, _ in N.ServerInfo._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            check(N.lib().dyngb200_server_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- the load generator ------------------------------------------------------------------------

SCALES = (18, 19, 20, 20, 21, 21, 22, 22)


class _Pool:
    """Random change material for one graph: a window of it is a batch (no per-request copy)."""

    def __init__(self, edges, rng, size=1 << 21):
        n = edges.num_vertices
        self.ins_src = rng.integers(0, n, size).astype(np.int32)
        self.ins_dst = rng.integers(0, n, size).astype(np.int32)
        self.ins_w = rng.integers(1, 1001, size).astype(np.int32)
        pick = rng.integers(0, edges.src.size, size)
        self.del_src = edges.src[pick].copy()
        self.del_dst = edges.dst[pick].copy()
        self.size = size

    def batch(self, rng, changes, insert_fraction=0.75):
        ni = int(round(changes * insert_fraction))
        nd = changes - ni
        a = int(rng.integers(0, self.size - ni + 1))
        b = int(rng.integers(0, self.size - nd + 1))
        return EdgeBatch.from_arrays(self.ins_src[a:a + ni], self.ins_dst[a:a + ni],
                                     self.ins_w[a:a + ni], self.del_src[b:b + nd],
                                     self.del_dst[b:b + nd])


def zipf_weights(n, s=1.1):
    w = 1.0 / np.arange(1, n + 1) ** s
    return w / w.sum()


def run_load(server, slots, pools, rate, seconds, rng, size_range=(100, 1_000_000)):
    """Poisson arrivals at `rate` batches/s for `seconds`; returns per-request records."""
    n_req = max(1, int(rng.poisson(rate * seconds)))
    gaps = rng.exponential(1.0 / rate, n_req)
    targets = rng.choice(len(slots), n_req, p=zipf_weights(len(slots)))
    lo, hi = np.log(size_range[0]), np.log(size_range[1])
    sizes = np.exp(rng.uniform(lo, hi, n_req)).round().astype(np.int64)
    batches = [pools[t].batch(rng, int(s)) for t, s in zip(targets, sizes)]
    tickets = []
    done = []

    def collect():
        for i, tk in enumerate(iter(tickets_q.get, None)):
            st, tm = server.wait(tk[0])
            done.append((tk[1], tk[2], tm["total_ms"], tm["queued_ms"], tm["group_size"],
                         tm["service_ms"], tm["begin_ms"], tm["round_ms"], tm["copy_ms"], tk[3],
                         tm["lane"]))

    import queue
    tickets_q = queue.Queue()
    th = threading.Thread(target=collect, daemon=True)
    th.start()
    t0 = time.perf_counter()
    due = t0
    for i in range(n_req):
        due += gaps[i]
        now = time.perf_counter()
        if due > now:
            time.sleep(due - now)
        t_sub = time.perf_counter() - t0
        tk = server.submit(slots[targets[i]], batches[i])
        tickets.append(tk)
        tickets_q.put((tk, int(targets[i]), int(sizes[i]), t_sub))
    tickets_q.put(None)
    th.join()
    wall = time.perf_counter() - t0
    return done, wall


def summarize(done, wall, rate):
    lat = np.array([d[2] for d in done])
    changes = sum(d[1] for d in done)
    return {"rate": rate, "requests": len(done), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "p99_over_p50": float(np.percentile(lat, 99) / max(np.percentile(lat, 50), 1e-9)),
            "max_ms": float(lat.max()),
            "service_max_ms": float(max(d[5] for d in done)),
            "changed_edges_per_s": changes / wall,
            "mean_group": float(np.mean([d[4] for d in done])),
            "parts_p50_ms": {k: float(np.percentile([d[i] for d in done], 50))
                             for k, i in PARTS},
            "parts_p99_ms": {k: float(np.percentile([d[i] for d in done], 99))
                             for k, i in PARTS},
            "by_size": by_size(done)}


def graph_waits(done):
    """Per request: how long it waited for its own graph's earlier requests to finish (the
    batches of one graph apply in arrival order, so a request cannot start before its
    predecessor on the same graph is done).  Records are in completion order; submission times
    (submitted_s) order them per graph."""
    wait = [0.0] * len(done)
    by_graph = {}
    for i, d in enumerate(done):
        by_graph.setdefault(d[0], []).append(i)
    for idx in by_graph.values():
        idx.sort(key=lambda i: done[i][9])
        prev_finish = -1.0
        for i in idx:
            submit_ms = done[i][9] * 1000.0
            wait[i] = max(0.0, prev_finish - submit_ms)
            prev_finish = max(prev_finish, submit_ms + done[i][2])
    return wait


def by_size(done):
    """p50 / p99 latency per decade of batch size (the load mixes 100 .. 1M changes, whose own
    service times differ by 10x, so the overall p99 / p50 mostly measures the mix); `own_*`
    leaves out the wait for the same graph's earlier requests (graph_waits): the latency the
    serving loop adds to the order it must keep."""
    out = {}
    gw = graph_waits(done)
    for lo in (100, 1_000, 10_000, 100_000):
        sel = [i for i, d in enumerate(done)
               if lo <= d[1] < lo * 10 or (lo == 100_000 and d[1] >= lo)]
        if sel:
            lat = [done[i][2] for i in sel]
            own = [done[i][2] - gw[i] for i in sel]
            out[f"{lo}+"] = {"n": len(lat), "p50_ms": float(np.percentile(lat, 50)),
                             "p99_ms": float(np.percentile(lat, 99)),
                             "own_p50_ms": float(np.percentile(own, 50)),
                             "own_p99_ms": float(np.percentile(own, 99)),
                             "graph_wait_p99_ms": float(np.percentile([gw[i] for i in sel], 99))}
    return out


STORAGE_KEYS = ("arena_growths", "compactions", "index_builds", "grow_ms", "compact_ms",
                "index_ms", "maintenance_ms_max")
PARTS = (("queued", 3), ("service", 5), ("begin", 6), ("round", 7), ("copy", 8))
RECORD = ("graph", "changes", "total_ms", "queued_ms", "group_size", "service_ms", "begin_ms",
          "round_ms", "copy_ms", "submitted_s", "lane")


def main(argv=None):
    import argparse
    import json
    from .generators import rmat
    from .sssp import compute
    ap = argparse.ArgumentParser(prog="python -m dyng_b200.serving")
    ap.add_argument("--rates", default="10,100,500,2000")
    ap.add_argument("--seconds", type=float, default=5.0)
    ap.add_argument("--scales", default=",".join(str(s) for s in SCALES))
    ap.add_argument("--max-batch", type=int, default=1_000_000)
    ap.add_argument("--learned", default="", help="scheduler weights (.npz); empty: heuristic")
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--dump", default="", help="write every request's record to this .npz")
    ap.add_argument("--small-changes", type=int, default=65536,
                    help="batches up to this many changes run in the small lane's rounds")
    ap.add_argument("--lanes", type=int, default=2,
                    help="2: large batches on their own lane beside small rounds; 1: one lane; "
                         "3..8: lanes - 1 small lanes side by side beside the large one")
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    res = Resources(0)
    sched = None
    if a.learned:
        from .scheduler import Scheduler
        sched = Scheduler.load(a.learned, resources=res)
    server = Server(res, scheduler=sched, lanes=a.lanes, small_changes=a.small_changes)
    slots, pools, keep = [], [], []
    for i, sc in enumerate(int(x) for x in a.scales.split(",")):
        edges = rmat(sc, 16, w_max=1000, seed=100 + i, device="cuda")
        g = Graph.from_csr(*edges.csr(), resources=res)
        t = compute(g, 0)
        slots.append(server.add(g, t))
        pools.append(_Pool(edges, rng))
        keep.append((g, t))
        print(f"graph {i}: scale {sc}, {edges.src.size} edges", flush=True)
    # warm-up (not measured): every graph sees the largest batch size twice, so workspaces,
    # pair tables, pinned copies and the edge indexes have grown before the timed loads
    for _ in range(2):
        tickets = [server.submit(sl, pools[i].batch(rng, a.max_batch)) for i, sl in enumerate(slots)]
        for tk in tickets:
            server.wait(tk)
    records = {}
    for rate in (float(r) for r in a.rates.split(",")):
        done, wall = run_load(server, slots, pools, rate, a.seconds, rng, (100, a.max_batch))
        out = summarize(done, wall, rate)
        out["info"] = server.info()
        out["storage"] = [{k: round(v, 3) for k, v in g.storage().items()
                           if k in STORAGE_KEYS} for g, _ in keep]
        print(json.dumps(out), flush=True)
        records[f"rate{rate:g}"] = np.array(done, dtype=np.float64)
    if a.dump:
        np.savez(a.dump, fields=np.array(RECORD), **records)
    server.close()


if __name__ == "__main__":
    main()
