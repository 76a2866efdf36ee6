"""Seeded synthetic inputs of the benchmark workloads (the reference ships no R-MAT or grid
generator; these are this package's own, written from the workload descriptions):

  - R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): every edge picks one of the four adjacency
    quadrants per level with probabilities (a, b, c, d); directed; self-loops and duplicate pairs
    dropped; int32 weights uniform in [1, w_max];
  - a side x side 2D grid with bidirectional 4-neighbour edges plus a fraction of random directed
    long-range shortcuts, weights round(lognormal(mu, sigma)) clamped to [1, w_max];
  - change batches: insertions of uniform random (u, v) pairs and deletions drawn from current
    tree edges (parent[v] -> v) and uniformly from the other edges.

Everything is a pure function of its seed (a counter-based hash for R-MAT, numpy PCG64 for the
rest), so the CPU oracle and the GPU path see the same inputs.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class EdgeList:
    num_vertices: int
    src: np.ndarray  # int32, sorted by (src, dst), unique pairs
    dst: np.ndarray
    weights: np.ndarray  # int32

    def csr(self):
        row_ptr = np.zeros(self.num_vertices + 1, np.int64)
        np.cumsum(np.bincount(self.src, minlength=self.num_vertices), out=row_ptr[1:])
        return row_ptr, self.dst, self.weights


_M1 = 0x9E3779B97F4A7C15
_M2 = 0xBF58476D1CE4E5B9
_M3 = 0x94D049BB133111EB
_F1 = 0xFF51AFD7ED558CCD
_F2 = 0xC4CEB9FE1A85EC53


def _hash32_np(idx: np.ndarray, level: int, seed: int) -> np.ndarray:
    """Counter-based uniform u32 of (edge index, level, seed): a Weyl sum through the murmur3
    64-bit finalizer, high 32 bits.  Identical in _hash32_torch."""
    with np.errstate(over="ignore"):
        x = (idx.astype(np.uint64) * np.uint64(_M1) + np.uint64(((level + 1) * _M2) & 0xFFFFFFFFFFFFFFFF)
             + np.uint64((seed * _M3) & 0xFFFFFFFFFFFFFFFF))
        x ^= x >> np.uint64(33)
        x *= np.uint64(_F1)
        x ^= x >> np.uint64(33)
        x *= np.uint64(_F2)
        x ^= x >> np.uint64(33)
    return (x >> np.uint64(32)).astype(np.int64)


def _s64(c: int) -> int:
    c &= 0xFFFFFFFFFFFFFFFF
    return c - (1 << 64) if c >= 1 << 63 else c


def _hash32_torch(idx, level: int, seed: int):
    import torch
    def lsr(x, k):  # logical shift right of int64 bit patterns
        return (x >> k) & ((1 << (64 - k)) - 1)
    x = idx * _s64(_M1) + _s64((level + 1) * _M2) + _s64(seed * _M3)
    x = x ^ lsr(x, 33)
    x = x * _s64(_F1)
    x = x ^ lsr(x, 33)
    x = x * _s64(_F2)
    x = x ^ lsr(x, 33)
    return lsr(x, 32)


def _thresholds(a, b, c):
    t = 1 << 32
    return int(a * t), int((a + b) * t), int((a + b + c) * t)


def rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, w_max=1000, seed=1,
         w_min=1, device=None) -> EdgeList:
    """Directed R-MAT graph with 2**scale vertices and edge_factor * 2**scale drawn edges.

    Edge i picks its quadrant at level l from the counter-based hash of (i, l, seed), so the
    numpy path and the torch path (device="cuda", for large scales) give identical graphs.  The
    weight of the j-th pair in sorted order is w_min + hash(j, scale, seed + 1) mod the range."""
    n = 1 << scale
    m = edge_factor * n
    A, AB, ABC = _thresholds(a, b, c)
    if device is not None:
        import torch
        key_parts = []
        chunk = 1 << 24
        for lo in range(0, m, chunk):
            hi = min(m, lo + chunk)
            idx = torch.arange(lo, hi, device=device, dtype=torch.int64)
            s = torch.zeros_like(idx)
            t = torch.zeros_like(idx)
            for level in range(scale):
                r = _hash32_torch(idx, level, seed)
                bit = 1 << (scale - 1 - level)
                s |= (r >= AB).to(torch.int64) * bit
                t |= (((r >= A) & (r < AB)) | (r >= ABC)).to(torch.int64) * bit
            keep = s != t
            key_parts.append((s[keep] << 32) | t[keep])
        key = torch.unique(torch.cat(key_parts))
        j = torch.arange(key.numel(), device=device, dtype=torch.int64)
        w = w_min + _hash32_torch(j, scale, seed + 1) % (w_max - w_min + 1)
        key = key.cpu().numpy()
        w = w.to(torch.int32).cpu().numpy()
    else:
        keys = []
        chunk = 1 << 22
        for lo in range(0, m, chunk):
            hi = min(m, lo + chunk)
            idx = np.arange(lo, hi, dtype=np.int64)
            s = np.zeros(hi - lo, np.int64)
            t = np.zeros(hi - lo, np.int64)
            for level in range(scale):
                r = _hash32_np(idx, level, seed)
                bit = np.int64(1 << (scale - 1 - level))
                s |= (r >= AB).astype(np.int64) * bit
                t |= (((r >= A) & (r < AB)) | (r >= ABC)).astype(np.int64) * bit
            keep = s != t
            keys.append((s[keep] << 32) | t[keep])
        key = np.unique(np.concatenate(keys))
        j = np.arange(key.size, dtype=np.int64)
        w = (w_min + _hash32_np(j, scale, seed + 1) % (w_max - w_min + 1)).astype(np.int32)
    src = (key >> 32).astype(np.int32)
    dst = (key & 0xFFFFFFFF).astype(np.int32)
    return EdgeList(n, src, dst, w)


def grid(side: int = 4096, shortcut_fraction=0.001, mu=3.0, sigma=1.0, w_max=10000,
         seed=1) -> EdgeList:
    """side x side grid, bidirectional 4-neighbour edges plus random directed shortcuts."""
    rng = np.random.default_rng(seed)
    n = side * side
    v = np.arange(n, dtype=np.int64)
    x = v % side
    y = v // side
    right = v[x + 1 < side]
    down = v[y + 1 < side]
    src = np.concatenate([right, right + 1, down, down + side])
    dst = np.concatenate([right + 1, right, down + side, down])
    k = int(round(shortcut_fraction * src.size))
    src = np.concatenate([src, rng.integers(0, n, k)]).astype(np.int32)
    dst = np.concatenate([dst, rng.integers(0, n, k)]).astype(np.int32)
    keep = src != dst
    key = np.unique((src[keep].astype(np.int64) << 32) | dst[keep].astype(np.int64))
    s = (key >> 32).astype(np.int32)
    d = (key & 0xFFFFFFFF).astype(np.int32)
    w = np.clip(np.rint(rng.lognormal(mu, sigma, s.size)), 1, w_max).astype(np.int32)
    return EdgeList(n, s, d, w)


@dataclass
class Batch:
    insert_src: np.ndarray
    insert_dst: np.ndarray
    insert_weights: np.ndarray
    delete_src: np.ndarray
    delete_dst: np.ndarray

    @property
    def size(self) -> int:
        return int(self.insert_src.size + self.delete_src.size)


class BatchStream:
    """Consecutive seeded batches on a graph whose live edges it tracks (base edges minus the
    deleted ones, plus the inserted pairs)."""

    def __init__(self, edges: EdgeList, seed: int = 7, w_min=1, w_max=1000):
        self.n = edges.num_vertices
        self.src = edges.src
        self.dst = edges.dst
        self.alive = np.ones(edges.src.size, bool)
        self.key = (edges.src.astype(np.int64) << 32) | edges.dst.astype(np.int64)  # sorted
        self.rng = np.random.default_rng(seed)
        self.w_min, self.w_max = w_min, w_max

    def _base_index(self, s, d):
        k = (s.astype(np.int64) << 32) | d.astype(np.int64)
        i = np.searchsorted(self.key, k)
        i = np.minimum(i, self.key.size - 1)
        hit = self.key[i] == k
        return i, hit

    def next(self, size: int, insert_fraction=0.75, tree_fraction=0.5, parents=None,
             near_source_hops=None, dist_hops=None) -> Batch:
        """size changes: insert_fraction insertions of uniform pairs; the deletions drawn
        tree_fraction from tree edges parent[v] -> v (v restricted to `near` vertices when
        dist_hops / near_source_hops are given) and the rest uniformly from the live base edges."""
        rng = self.rng
        ni = int(round(size * insert_fraction))
        nd = size - ni
        n_tree = int(round(nd * tree_fraction)) if parents is not None else 0
        del_s, del_d = [], []
        if n_tree:
            cand = np.nonzero(parents >= 0)[0]
            if dist_hops is not None and near_source_hops is not None:
                near = cand[dist_hops[cand] <= near_source_hops]
                if near.size:
                    cand = near
            if cand.size:
                pick = rng.choice(cand, size=min(n_tree, cand.size), replace=False)
                del_s.append(parents[pick].astype(np.int32))
                del_d.append(pick.astype(np.int32))
        n_uni = nd - sum(a.size for a in del_s)
        live = np.nonzero(self.alive)[0] if not self.alive.all() else None
        if n_uni > 0:
            if live is None:
                idx = rng.integers(0, self.src.size, n_uni)
            else:
                idx = live[rng.integers(0, live.size, n_uni)]
            del_s.append(self.src[idx])
            del_d.append(self.dst[idx])
        ds = np.concatenate(del_s) if del_s else np.zeros(0, np.int32)
        dd = np.concatenate(del_d) if del_d else np.zeros(0, np.int32)
        i, hit = self._base_index(ds, dd) if ds.size else (np.zeros(0, np.int64), np.zeros(0, bool))
        self.alive[i[hit]] = False
        is_ = rng.integers(0, self.n, ni).astype(np.int32)
        id_ = rng.integers(0, self.n, ni).astype(np.int32)
        w = rng.integers(self.w_min, self.w_max, ni, endpoint=True).astype(np.int32)
        # re-inserted base pairs come back to life
        j, hit = self._base_index(is_, id_)
        self.alive[j[hit]] = True
        return Batch(is_, id_, w, ds.astype(np.int32), dd.astype(np.int32))


class NearSourceChurn:
    """Batches for a grid around a centre source: half deletions, concentrated within `hops`
    lattice hops of the source (at most a quarter of the live edges there per batch, the rest
    uniform over the live edges), half insertions, which bring back the near edges the previous
    batch deleted (the rest uniform pairs, lognormal weights).  The region around the source
    churns without being cut off from it."""

    def __init__(self, stream: BatchStream, side: int, source: int, hops: int = 64,
                 insert_fraction: float = 0.5):
        self.stream = stream
        self.insert_fraction = insert_fraction
        src = stream.src.astype(np.int64)
        cx, cy = source % side, source // side
        self.near = np.nonzero(np.abs(src % side - cx) + np.abs(src // side - cy) <= hops)[0]
        self.back = np.zeros(0, np.int64)

    def next(self, size: int) -> Batch:
        st = self.stream
        rng = st.rng
        ni = int(round(size * self.insert_fraction))
        nd = size - ni
        live_near = self.near[st.alive[self.near]]
        k = min(nd, live_near.size // 4)
        pick_near = rng.choice(live_near, k, replace=False) if k else np.zeros(0, np.int64)
        live = np.nonzero(st.alive)[0]
        pick = np.concatenate([pick_near, live[rng.integers(0, live.size, nd - k)]])
        st.alive[pick] = False
        reins = self.back[:ni]
        st.alive[reins] = True
        m = ni - reins.size
        is_ = np.concatenate([st.src[reins], rng.integers(0, st.n, m).astype(np.int32)])
        id_ = np.concatenate([st.dst[reins], rng.integers(0, st.n, m).astype(np.int32)])
        iw = np.clip(np.rint(rng.lognormal(3.0, 1.0, ni)), 1, 10000).astype(np.int32)
        self.back = pick_near
        return Batch(is_.astype(np.int32), id_.astype(np.int32), iw,
                     st.src[pick].astype(np.int32), st.dst[pick].astype(np.int32))


def uniform_batch(edges: EdgeList, num_deletions: int, num_insertions: int, seed=7, w_min=1,
                  w_max=100) -> Batch:
    """Deletions sampled uniformly from the edges, insertions of uniform random pairs."""
    rng = np.random.default_rng(seed)
    pick = rng.choice(edges.src.size, size=num_deletions, replace=False)
    s = rng.integers(0, edges.num_vertices, num_insertions).astype(np.int32)
    d = rng.integers(0, edges.num_vertices, num_insertions).astype(np.int32)
    w = rng.integers(w_min, w_max, num_insertions, endpoint=True).astype(np.int32)
    return Batch(s, d, w, edges.src[pick].copy(), edges.dst[pick].copy())
