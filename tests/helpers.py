"""Shared helpers of the test suite: fixture decoding and seeded random cases."""
from __future__ import annotations

import numpy as np

INF = (2**63 - 1) // 4


def fixture_case(z, name):
    """Decode one golden case of tests/golden/mosp_fixtures.npz."""
    k = int(z[f"{name}/k"])
    ins = z[f"{name}/ins"].reshape(-1, 2 + k)
    dele = z[f"{name}/del"].reshape(-1, 2)
    case = {
        "k": k,
        "row_ptr": z[f"{name}/row_ptr"],
        "col": z[f"{name}/col"],
        "w": z[f"{name}/w"].reshape(k, -1),
        "ins_src": ins[:, 0].copy(),
        "ins_dst": ins[:, 1].copy(),
        "ins_w": ins[:, 2:].copy().ravel(),  # insertion-major
        "del_src": dele[:, 0].copy(),
        "del_dst": dele[:, 1].copy(),
        "invalidated": z[f"{name}/invalidated"],
        "init_d": [z[f"{name}/init_d{j}"] for j in range(k)],
        "init_p": [z[f"{name}/init_p{j}"] for j in range(k)],
        "upd_d": [z[f"{name}/upd_d{j}"] for j in range(k)],
        "upd_p": [z[f"{name}/upd_p{j}"] for j in range(k)],
    }
    if f"{name}/applied_row_ptr" in z.files:
        for key in ("row_ptr", "col", "w", "in_row_ptr", "in_col", "in_w", "increase"):
            case["applied_" + key] = z[f"{name}/applied_{key}"]
        case["applied_w"] = case["applied_w"].reshape(k, -1)
        case["applied_in_w"] = case["applied_in_w"].reshape(k, -1)
    return case


def combined_case(z, name):
    """Decode one case of tests/golden/mosp_combined.npz (K objectives of a graph with KG weight
    columns, preferences, the combined tree and the path costs over all KG columns)."""
    k, kg = int(z[f"{name}/k"]), int(z[f"{name}/kg"])
    ins = z[f"{name}/ins"].reshape(-1, 2 + kg)
    dele = z[f"{name}/del"].reshape(-1, 2)
    return {
        "k": k, "kg": kg, "pref": [int(x) for x in z[f"{name}/pref"]],
        "row_ptr": z[f"{name}/row_ptr"], "col": z[f"{name}/col"],
        "w": z[f"{name}/w"].reshape(kg, -1),
        "ins_src": ins[:, 0].copy(), "ins_dst": ins[:, 1].copy(),
        "ins_w": ins[:, 2:].copy().ravel(),  # insertion-major, KG per insertion
        "del_src": dele[:, 0].copy(), "del_dst": dele[:, 1].copy(),
        "init_d": [z[f"{name}/init_d{j}"] for j in range(k)],
        "init_p": [z[f"{name}/init_p{j}"] for j in range(k)],
        "combined_d": z[f"{name}/combined_d"], "combined_p": z[f"{name}/combined_p"],
        "costs": z[f"{name}/costs"].reshape(-1, kg),
    }


# The random shapes of the reference's randomized differential test
# (cpp/tests/algorithms/sssp/sssp_random_test.cpp:467-580): sparse, dense, grid, hub, chain graphs
# with tiny, [1,100] and large weights; chains of batches.
SHAPES = ("sparse", "dense", "grid", "hub", "chain")
WEIGHTS = {"tiny": (1, 3), "small": (1, 100), "huge": (1, 2**31 - 1)}


def random_graph(rng, shape, n, weights="small", multi=False):
    lo, hi = WEIGHTS[weights]
    if shape == "sparse":
        m = 3 * n
        src = rng.integers(0, n, m)
        dst = rng.integers(0, n, m)
    elif shape == "dense":
        m = n * max(4, n // 3)
        src = rng.integers(0, n, m)
        dst = rng.integers(0, n, m)
    elif shape == "grid":
        side = max(2, int(np.sqrt(n)))
        n = side * side
        v = np.arange(n)
        x, y = v % side, v // side
        right = v[x + 1 < side]
        down = v[y + 1 < side]
        src = np.concatenate([right, right + 1, down, down + side])
        dst = np.concatenate([right + 1, right, down + side, down])
    elif shape == "hub":
        m = 4 * n
        src = np.where(rng.random(m) < 0.5, 0, rng.integers(0, n, m))
        dst = np.where(rng.random(m) < 0.3, 1 % n, rng.integers(0, n, m))
    else:  # chain
        src = np.arange(n - 1)
        dst = np.arange(1, n)
        extra = rng.integers(0, n, n // 4)
        src = np.concatenate([src, extra])
        dst = np.concatenate([dst, rng.integers(0, n, n // 4)])
    w = rng.integers(lo, hi, src.size, endpoint=True)
    return n, src.astype(np.int32), dst.astype(np.int32), w.astype(np.int32)


def random_batch(rng, n, src, dst, size, weights="small", tree_parents=None, grow=0):
    """A batch of about `size` changes: half deletions (of existing edges, some of them tree
    edges, some missing), half insertions (new pairs, upserts of existing ones, self-loops)."""
    lo, hi = WEIGHTS[weights]
    nd = size // 2
    ni = size - nd
    del_src, del_dst = [], []
    if src.size:
        pick = rng.integers(0, src.size, nd)
        del_src = list(src[pick])
        del_dst = list(dst[pick])
    if tree_parents is not None:
        v = np.nonzero(tree_parents >= 0)[0]
        if v.size:
            pick = rng.choice(v, min(v.size, max(1, nd // 3)), replace=False)
            del_src += list(tree_parents[pick])
            del_dst += list(pick)
    del_src += list(rng.integers(0, n, 2))
    del_dst += list(rng.integers(0, n, 2))
    top = n + grow
    ins_src = list(rng.integers(0, top, ni))
    ins_dst = list(rng.integers(0, top, ni))
    if src.size:
        pick = rng.integers(0, src.size, max(1, ni // 4))
        ins_src += list(src[pick])
        ins_dst += list(dst[pick])
    if n:
        s = int(rng.integers(0, n))
        ins_src.append(s)
        ins_dst.append(s)
    ins_w = rng.integers(lo, hi, len(ins_src), endpoint=True)
    return {
        "ins_src": np.asarray(ins_src, np.int32),
        "ins_dst": np.asarray(ins_dst, np.int32),
        "ins_w": np.asarray(ins_w, np.int32),
        "del_src": np.asarray(del_src, np.int32),
        "del_dst": np.asarray(del_dst, np.int32),
    }
