"""Benchmark: batch-dynamic SSSP update on one B200 (changed edges/s, p50/p99 update latency).

Workload (the headline configuration): directed R-MAT, scale 22 (4,194,304 vertices), edge
factor 16, (a, b, c) = (0.57, 0.19, 0.19), self-loops and duplicate pairs dropped, int32 weights
uniform in [1, 1000], source 0; consecutive 100k-change batches, 75% insertions of uniform
random pairs, 25% deletions (half current tree edges parent[v] -> v, half uniform other edges).
Seeded synthetic data (the reference publishes no number for this configuration).

A step is one sssp::update of one batch.  `value` times the update with the batch already in
device memory (CUDA events on the library's stream); `e2e` times the public call with the batch
in pinned host memory (the copy to the device and the read-back of the stats inside the timed
region).  Two arms run on the same batches from the same starting graph and tree (a device
snapshot restored in between): the plain schedule (the fixed heuristic) and the learned
scheduler (dyng_b200/data/scheduler_weights.npz); `--schedule` picks the headline arm and
config.schedules reports both.  Every run checks that both arms end in the same tree and that
the final tree equals a from-scratch compute (distances and parents bit-exact).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch 100000] [--scale 22]
    python bench.py --graph grid [--side 4096] [--batch 10000]   # the high-diameter workload
    python bench.py --impl reference ...   # the reference algorithm's CPU restatement (oracle)
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "changed edges/s and p50/p99 update latency, learned vs plain schedule, 1 B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=100_000)
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--graph", default="rmat", choices=["rmat", "grid"],
                    help="rmat: R-MAT ef16 (headline); grid: side x side 4-neighbour grid with "
                         "0.1%% shortcuts, lognormal weights, source at the centre, 50/50 batches "
                         "whose deletions concentrate within 64 hops of the source")
    ap.add_argument("--side", type=int, default=4096)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--schedule", default="learned", choices=["plain", "learned"],
                    help="the headline arm; both arms run when scheduler weights exist")
    ap.add_argument("--scheduler-weights", default=os.path.join(ROOT, "dyng_b200", "data",
                                                                "scheduler_weights.npz"))
    ap.add_argument("--invalidation", type=int, default=0, help="0 pointer jumping, 1 subtree walk")
    ap.add_argument("--delta", type=int, default=0)
    ap.add_argument("--grid-blocks", type=int, default=0)
    ap.add_argument("--heavy-degree", type=int, default=0)
    ap.add_argument("--small", type=int, default=0, help="small-frontier size (0 default, -1 off)")
    ap.add_argument("--engine", default="automatic", choices=["automatic", "fused", "operators"],
                    help="sssp options.cuda_engine (automatic: fused with cooperative launch)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-verify", action="store_true")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic(args):
    """DRAM bytes per k_sssp launch from the committed ncu capture of this workload (None when
    the workload differs from the captured one)."""
    path = os.path.join(ROOT, "profiles", "k_sssp_dram_rmat-s22_batch100k.json")
    if not os.path.exists(path) or (args.graph, args.scale, args.batch) != ("rmat", 22, 100_000):
        return None
    with open(path) as f:
        return int(json.load(f)["dram_bytes_per_launch"])


def make_workload(args, device):
    from dyng_b200 import generators as G
    t0 = time.time()
    if args.graph == "grid":
        edges = G.grid(args.side, seed=1)
    else:
        edges = G.rmat(args.scale, 16, w_max=1000, seed=1, device=device)
    return edges, time.time() - t0


def workload_name(args):
    if args.graph == "grid":
        return f"grid-{args.side}x{args.side}-lognormal-batch{args.batch}"
    return f"rmat-s{args.scale}-ef16-w1000-batch{args.batch}"


def source_of(args):
    """R-MAT: vertex 0; grid: the centre vertex."""
    return (args.side // 2) * args.side + args.side // 2 if args.graph == "grid" else 0


def insert_fraction(args):
    return 0.5 if args.graph == "grid" else 0.75


L2_BYTES = 126 * 1024 * 1024


def l2_note(num_edges):
    """How the timed steps stand to the 126 MB L2: no flush runs between steps, so the graph's
    arenas (out and in, a 4-byte column and a 4-byte weight per slot each) must exceed it."""
    arenas = 16 * int(num_edges)
    if arenas > L2_BYTES:
        return f"inputs larger than L2 (graph arenas ~{arenas / 1e9:.1f} GB, L2 126 MB)"
    return (f"inputs smaller than L2 (graph arenas ~{arenas / 1e6:.0f} MB, L2 126 MB) and no "
            "flush between steps: a small configuration, not a timing of record")


def batch_maker(args, stream):
    """next(parents) -> one batch of the workload.  R-MAT: 75% insertions, half of the deletions
    tree edges.  Grid: 50/50; the deletions concentrate within 64 lattice hops of the source (a
    quarter of the live edges there per batch, the rest uniform over the live edges) and the
    near edges deleted by the previous batch come back as insertions (the rest uniform pairs),
    so the region around the source churns without being cut off."""
    if args.graph != "grid":
        return lambda parents: stream.next(args.batch, 0.75, 0.5, parents=parents)
    from dyng_b200 import generators as G
    churn = G.NearSourceChurn(stream, args.side, source_of(args))
    return lambda parents: churn.next(args.batch)


def oracle_replay(edges, source, init_tree, batches, gpu_stats, final_tree, budget_s=90.0):
    """The CPU leg: the oracle (the reference's algorithm restated in C, batch application and
    repair on every host core, as the reference's OpenMP host path) computes the initial tree of
    the same graph itself, then replays the GPU arm's batches in order, timing each update.

    It is also the full-size parity check of the GPU arm: the oracle's initial tree against the
    GPU's compute, every batch's `invalidated` / `affected` and apply summary against the GPU's
    stats of the same batch, and, when every batch was replayed within the budget, the final
    tree against the GPU's (distances and parents bit for bit)."""
    from oracle import oracle as O
    cores = O.set_threads(host_cores())
    rp, col, w = edges.csr()
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    t0 = time.perf_counter()
    ot, _ = O.compute(og, source, rule=1)
    compute_s = time.perf_counter() - t0
    check = {"compute_equal": bool(np.array_equal(ot.distances, init_tree[0]) and
                                   np.array_equal(ot.parents, init_tree[1])),
             "batches": len(batches), "replayed": 0, "stats_equal": True, "final_tree_equal": None,
             "first_mismatch": None, "oracle_compute_s": round(compute_s, 1)}
    done, changes, spent = 0, 0, 0.0
    for i, (b, gs) in enumerate(zip(batches, gpu_stats)):
        t0 = time.perf_counter()
        ost, osm = O.update(og, O.Batch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                                        b.delete_dst), ot)
        spent += time.perf_counter() - t0
        done += 1
        changes += b.size
        got = (gs.invalidated, gs.affected, gs.batch.inserted_edges, gs.batch.deleted_edges,
               gs.batch.updated_edges)
        want = (ost["invalidated"], ost["affected"], osm["inserted_edges"], osm["deleted_edges"],
                osm["updated_edges"])
        if got != want and check["stats_equal"]:
            check["stats_equal"] = False
            check["first_mismatch"] = {"batch": i, "gpu": list(got), "oracle": list(want)}
        if spent > budget_s:
            break
    check["replayed"] = done
    if done == len(batches):
        check["final_tree_equal"] = bool(np.array_equal(ot.distances, final_tree[0]) and
                                         np.array_equal(ot.parents, final_tree[1]))
    O.set_threads(1)
    check["verified"] = bool(check["compute_equal"] and check["stats_equal"] and
                             check["final_tree_equal"])
    return changes / spent, done, spent, cores, check


def host_cores() -> int:
    """The host cores this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    """--impl reference: the reference's CPU algorithm (the oracle port) on this workload.

    Nothing of this package's CUDA library runs here: the synthetic graph is generated with
    torch tensor ops (on the GPU when one is present: input generation only, outside the timed
    steps), and the oracle computes the initial tree and applies every batch."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    device = "cuda" if torch.cuda.is_available() else None
    edges, _ = make_workload(args, device)
    from dyng_b200 import generators as G
    from oracle import oracle as O
    cores = O.set_threads(host_cores())
    rp, col, w = edges.csr()
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    ot, _ = O.compute(og, source_of(args), rule=1)
    stream = G.BatchStream(edges, seed=7)
    make_batch = batch_maker(args, stream)
    times, sizes = [], []
    for step in range(args.warmup + args.steps):
        b = make_batch(ot.parents)
        t0 = time.perf_counter()
        O.update(og, O.Batch(b.insert_src, b.insert_dst, b.insert_weights, b.delete_src,
                             b.delete_dst), ot)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
            sizes.append(b.size)
    total = sum(times)
    value = sum(sizes) / total
    line = {"metric": METRIC, "value": value, "unit": "changed edges/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(args),
                       "vertices": int(edges.num_vertices), "edges": int(edges.src.size),
                       "batch_changes": args.batch, "insert_fraction": insert_fraction(args),
                       "source": source_of(args), "parallelism": f"replicas{args.gpus}",
                       "l2": l2_note(edges.src.size),
                       "p50_ms": 1000 * float(np.percentile(times, 50)),
                       "p99_ms": 1000 * float(np.percentile(times, 99))},
            "cpu_baseline": {"value": value, "unit": "changed edges/s", "cores": cores,
                             "kind": "port",
                             "sample": f"{len(times)} consecutive {args.batch}-change batches; "
                                       f"apply and repair on {cores} threads"},
            "e2e": {"value": value, "unit": "changed edges/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


class Arm:
    """One schedule's pass over the benchmark batches: W warm-up steps, then K timed steps, each
    timed with CUDA events on the library's stream (max over ranks)."""

    def __init__(self, name, schedule=None, scheduler=None):
        self.name, self.schedule, self.scheduler = name, schedule, scheduler
        self.lat, self.sizes, self.stats, self.host = [], [], [], []
        self.all_stats = []  # every step's stats, warm-up included (the oracle replay checks them)
        self.total_ms = 0.0

    def summary(self, world):
        from dyng_b200.replicas import whole_job_rate
        v = whole_job_rate(sum(self.sizes), self.total_ms, world)
        return {"value": v, "ms_per_step": self.total_ms / max(len(self.lat), 1),
                "p50_ms": float(np.percentile(self.lat, 50)),
                "p99_ms": float(np.percentile(self.lat, 99)),
                "apply_ms_mean": float(np.mean([s.apply_ms for s in self.stats])),
                "sssp_ms_mean": float(np.mean([s.sssp_ms for s in self.stats])),
                # per timed step: the update (events around the call), its applier and sssp
                # kernel times, and the host time of the call
                "steps": [[round(t, 3), round(s.apply_ms, 3), round(s.sssp_ms, 3),
                           round(1000 * h, 3)]
                          for t, s, h in zip(self.lat, self.stats, self.host)],
                "maintenance": getattr(self, "maintenance", None)}


def run_arm(env, arm, next_batch, nvtx=False):
    D, torch, g, tree, stream, args, world, local = env
    import gc
    gc.collect()  # no collection of leftover objects (and their device frees) inside a timed step
    gc.disable()
    try:
        return _run_arm(env, arm, next_batch, nvtx)
    finally:
        gc.enable()


def _run_arm(env, arm, next_batch, nvtx):
    D, torch, g, tree, stream, args, world, local = env
    for step in range(args.warmup + args.steps):
        b = next_batch(step)
        ts = [torch.from_numpy(np.ascontiguousarray(x)).to(f"cuda:{local}") for x in
              (b.insert_src, b.insert_dst, b.insert_weights, b.delete_src, b.delete_dst)]
        db = D.EdgeBatch.device(ts[0].data_ptr(), ts[1].data_ptr(), ts[2].data_ptr(),
                                b.insert_src.size, ts[3].data_ptr(), ts[4].data_ptr(),
                                b.delete_src.size)
        torch.cuda.synchronize()
        if step == args.warmup:
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            storage0 = g.storage()
            if nvtx:
                torch.cuda.nvtx.range_push("timed")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        h0 = time.perf_counter()
        e0.record(stream)
        st = D.sssp.update(g, db, tree, schedule=arm.schedule, scheduler=arm.scheduler)
        e1.record(stream)
        e1.synchronize()
        arm.all_stats.append(st)
        if step >= args.warmup:
            arm.host.append(time.perf_counter() - h0)
            arm.lat.append(e0.elapsed_time(e1))
            arm.sizes.append(b.size)
            arm.stats.append(st)
        del ts
    torch.cuda.synchronize()
    if nvtx:
        torch.cuda.nvtx.range_pop()
    # storage maintenance inside the timed steps (edge-index builds, arena growths, compactions)
    storage1 = g.storage()
    arm.maintenance = {k: round(storage1[k] - storage0[k], 3) for k in
                       ("index_builds", "arena_growths", "compactions", "index_ms", "grow_ms",
                        "compact_ms")}
    from dyng_b200.replicas import max_over_ranks
    arm.total_ms = max_over_ranks(float(sum(arm.lat)))
    return arm


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import dyng_b200 as D
    from dyng_b200 import generators as G
    from dyng_b200 import scheduler as S

    # replicas only: every rank runs the same independent workload on its own GPU
    stream = torch.cuda.Stream()
    res = D.Resources(local, stream.cuda_stream)
    edges, gen_s = make_workload(args, "cuda")
    rp, col, w = edges.csr()
    t0 = time.time()
    g = D.Graph.from_csr(rp, col, w, resources=res)
    source = source_of(args)
    options = D.sssp.Options(cuda_engine=args.engine)
    tree = D.sssp.compute(g, source, options)
    build_s = time.time() - t0
    # the oracle replay (CPU leg, rank 0) starts from its own compute and checks it against this
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    init_tree = (tree.distances, tree.parents) if cpu_leg else None
    bs = G.BatchStream(edges, seed=7)
    make_batch = batch_maker(args, bs)
    env = (D, torch, g, tree, stream, args, world, local)

    fixed = None
    if args.invalidation or args.delta or args.grid_blocks or args.heavy_degree or args.small:
        fixed = D.sssp.Schedule(delta=args.delta, grid_blocks=args.grid_blocks,
                                invalidation=args.invalidation, heavy_degree=args.heavy_degree,
                                small_frontier=args.small)
    weights = args.scheduler_weights
    learned = None
    if os.path.exists(weights):
        learned = S.Scheduler.load(weights, resources=res)
    elif args.schedule == "learned":
        print(f"bench: no scheduler weights at {weights}; timing the plain schedule only",
              file=sys.stderr)
        args.schedule = "plain"

    # the plain arm generates the batches (deletions drawn from the current tree); the learned arm
    # replays them from the same starting graph and tree (a device snapshot restored in between)
    recorded = []

    def generate(step):
        b = make_batch(tree.parents)
        recorded.append(b)
        return b

    sampler = ClockSampler(local)
    sampler.start()
    arms = {}
    if learned is not None:
        g_snap, t_snap = g.clone(), tree.clone()
    arms["plain"] = run_arm(env, Arm("plain", schedule=fixed), generate,
                            nvtx=args.schedule == "plain")
    same = None
    final_plain = (tree.distances, tree.parents)
    if learned is not None:
        d_plain, p_plain = final_plain
        g.copy_from(g_snap)
        tree.copy_from(t_snap)
        del g_snap, t_snap
        arms["learned"] = run_arm(env, Arm("learned", scheduler=learned), lambda i: recorded[i],
                                  nvtx=args.schedule == "learned")
        same = bool(np.array_equal(d_plain, tree.distances) and
                    np.array_equal(p_plain, tree.parents))
    clocks = sampler.stop()
    head = arms[args.schedule]
    summ = {k: a.summary(world) for k, a in arms.items()}
    value = summ[args.schedule]["value"]
    timed_stats = head.stats
    # end to end: batches in pinned host memory through the public call, headline schedule
    e2e_lat, e2e_sizes, e2e_stats = [], [], []
    h2d = 0
    import gc
    for step in range(args.steps):
        b = make_batch(tree.parents)
        pinned = [torch.from_numpy(np.ascontiguousarray(x)).pin_memory() for x in
                  (b.insert_src, b.insert_dst, b.insert_weights, b.delete_src, b.delete_dst)]
        arrs = [p.numpy() for p in pinned]
        hb = D.EdgeBatch.from_arrays(*arrs)
        torch.cuda.synchronize()
        gc.collect()  # as in the arms: no collection (and device free) inside the timed call
        gc.disable()
        t0 = time.perf_counter()
        st = D.sssp.update(g, hb, tree, schedule=head.schedule, scheduler=head.scheduler)
        e2e_lat.append(time.perf_counter() - t0)
        gc.enable()
        e2e_sizes.append(b.size)
        e2e_stats.append(st)
        h2d = sum(a.nbytes for a in arrs)
    e2e_value = world * sum(e2e_sizes) / sum(e2e_lat)
    # where an end-to-end call's time goes (us, means): the library's host phases (checks and
    # staging with the batch copies queued, queuing the applier, queuing the sssp kernel and the
    # read-back, waiting for the device) and the two kernels' device times
    e2e_parts = {"host_us": [round(float(np.mean([s.host_us[i] for s in e2e_stats])), 1)
                             for i in range(4)],
                 "apply_us": round(1000 * float(np.mean([s.apply_ms for s in e2e_stats])), 1),
                 "sssp_us": round(1000 * float(np.mean([s.sssp_ms for s in e2e_stats])), 1)}

    # correctness at full size: the updated tree equals a from-scratch compute on the new graph
    verified = None
    compute_info = None
    if not args.no_verify:
        fresh, cst = D.sssp.compute(g, source, options, stats=True)
        verified = bool(np.array_equal(fresh.distances, tree.distances) and
                        np.array_equal(fresh.parents, tree.parents))
        # the same kernel on bulk work: a from-scratch solve of the final graph
        cbytes = cst.algorithmic_bytes
        compute_info = {"sssp_ms": round(cst.sssp_ms, 3), "alg_bytes": int(cbytes),
                        "achieved_gbs": round(cbytes / (cst.sssp_ms / 1000.0) / 1e9, 1)
                        if cst.sssp_ms > 0 else None,
                        "iterations": int(cst.iterations), "epochs": int(cst.epochs)}
        del fresh

    # roofline of the dominant kernel (the sssp persistent kernel): algorithmic bytes counted by
    # the kernel (Stats.work x Stats.WORK_BYTES) over its CUDA-event time on the launching stream
    sssp_ms = [s.sssp_ms for s in timed_stats]
    engine = timed_stats[0].engine_used
    peak, peak_kind = peaks()
    alg = [s.algorithmic_bytes + 12 * s.affected for s in timed_stats]
    achieved = float(np.sum(alg) / (np.sum(sssp_ms) / 1000.0) / 1e9) if sssp_ms else 0.0
    work = {name: int(np.mean([s.work[i] for s in timed_stats]))
            for i, name in enumerate(timed_stats[0].WORK_NAMES)}
    phases = {name: round(float(np.mean([s.phase_ms[i] for s in timed_stats])), 3)
              for i, name in enumerate(timed_stats[0].PHASES)}
    stages = {name: round(float(np.mean([s.stages_ms()[name] for s in timed_stats])), 4)
              for name in timed_stats[0].stages_ms()}
    # the batch applier's steps: the end of each (us since it began; 0: not reached)
    apply_steps = {name: [round(float(np.mean([s.apply_step_us[i] for s in a.stats])), 1)
                          for i in range(1, 12)]
                   for name, a in arms.items()}
    shape = {k: float(np.mean([getattr(s, k) for s in timed_stats]))
             for k in ("iterations", "epochs", "pushes", "invalidated", "affected", "rounds",
                       "touched", "delta", "grid_blocks")}
    classes = [list(s.schedule_classes) for s in timed_stats] if args.schedule == "learned" else None
    # the same roofline per phase of the kernel (bytes and device time of each phase, summed over
    # the timed steps): the kernel-wide fraction blends O(n) streaming passes with the latency-
    # bound frontier phases
    per_step = [s.phase_bytes_ms() for s in timed_stats]
    phase_roof = {}
    for name in timed_stats[0].PHASE_WORK:
        pb = float(sum(x[name][0] for x in per_step))
        pm = float(sum(x[name][1] for x in per_step))
        gbs = pb / (pm / 1000.0) / 1e9 if pm > 0 else None
        phase_roof[name] = {"bytes_per_update": round(pb / len(per_step)),
                            "ms_per_update": round(pm / len(per_step), 4),
                            "achieved_gbs": round(gbs, 1) if gbs is not None else None,
                            "frac": round(gbs / peak, 4) if gbs is not None and peak else None}

    cpu = None
    oracle_check = None
    if cpu_leg:
        try:
            v, done, spent, cores, oracle_check = oracle_replay(
                edges, source, init_tree, recorded, arms["plain"].all_stats, final_plain)
            cpu = {"value": v, "unit": "changed edges/s", "cores": cores, "kind": "port",
                   "sample": f"oracle sssp::update on {done} of the GPU arm's {len(recorded)} "
                             f"{args.batch}-change batches ({spent:.1f} s), same graph, from the "
                             f"oracle's own compute; apply and repair on {cores} threads"}
        except Exception as exc:  # noqa: BLE001
            cpu = {"value": None, "unit": "changed edges/s", "cores": host_cores(),
                   "kind": "port", "sample": f"failed: {exc}"}
        del init_tree
    del final_plain

    if rank == 0:
        compare = {k: {kk: round(vv, 4) if kk not in ("value", "steps", "maintenance") else vv
                       for kk, vv in v.items()}
                   for k, v in summ.items()}
        if "learned" in summ:
            compare["learned_over_plain"] = summ["learned"]["value"] / summ["plain"]["value"]
            compare["learned_equals_plain"] = same
        line = {
            "metric": METRIC, "value": value, "unit": "changed edges/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": summ[args.schedule]["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": {"workload": workload_name(args),
                       "vertices": int(edges.num_vertices), "edges": int(edges.src.size),
                       "batch_changes": args.batch, "insert_fraction": insert_fraction(args),
                       "source": source,
                       "schedule": args.schedule, "engine": engine,
                       "parallelism": f"replicas{world}",
                       "l2": l2_note(edges.src.size),
                       "p50_ms": summ[args.schedule]["p50_ms"],
                       "p99_ms": summ[args.schedule]["p99_ms"],
                       "apply_ms_mean": summ[args.schedule]["apply_ms_mean"],
                       "sssp_ms_mean": summ[args.schedule]["sssp_ms_mean"],
                       "host_ms_p50": 1000 * float(np.percentile(head.host, 50)),
                       "schedules": compare, "learned_classes": classes,
                       "sssp_phases_ms": phases, "stages_ms": stages, "sssp_work": work,
                       "apply_steps_end_us": apply_steps,
                       "update_shape": shape,
                       "alg_bytes_per_update": float(np.mean(alg)),
                       "trace_last_update": [list(t) for t in timed_stats[-1].trace],
                       "pj_rounds_us_last_update": list(timed_stats[-1].pj_rounds_us),
                       "pj_done_us_last_update": list(timed_stats[-1].pj_done_us),
                       "verified_vs_compute": verified, "compute_from_scratch": compute_info,
                       "verified_vs_oracle": oracle_check["verified"] if oracle_check else None,
                       "oracle_check": oracle_check,
                       "setup_s": {"generate": round(gen_s, 1), "build_and_compute": round(build_s, 1)}},
            "e2e": {"value": e2e_value, "unit": "changed edges/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": ctypes.sizeof(D._native.Stats),
                    "p50_ms": 1000 * float(np.percentile(e2e_lat, 50)),
                    "p99_ms": 1000 * float(np.percentile(e2e_lat, 99)), "parts": e2e_parts},
            "gpu_launches": int(sum(s.kernel_launches for s in timed_stats)),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None,
                         "traffic": traffic(args) if engine == "fused" else None,
                         "peak_kind": peak_kind,
                         "kernel": "k_sssp" if engine == "fused" else
                                   "k_op_* (the operators engine's launches and host steps)",
                         "phases": phase_roof},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()

if __name__ == "__main__":
    main()
