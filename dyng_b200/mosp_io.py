"""The MOSP text formats (the reference's io/csr_triplet.hpp, io/batch_io.hpp legacy files and
io/result_io.hpp), read and written byte for byte:

  <prefix>RowPtr.txt, <prefix>ColInd.txt   one integer per line (n + 1 and m lines)
  <prefix>Values.txt                       the K weights of an edge per line, space-separated
  insert.txt                               "u v w_1 .. w_K" per line
  delete.txt                               "u v" per line
  distances*.txt                           "v d" per line, "v INF" for an unreachable vertex
  SSSPTree*.txt                            "v p" per line, p = -1 for none
  mospCosts.txt                            "v c_1 .. c_K" per line, "INF" for an unreachable cost

Every file ends with a newline after its last line; an empty file is empty.
"""
from __future__ import annotations

import os

import numpy as np

INF_DISTANCE = (2**63 - 1) // 4


def _read_ints(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        data = f.read()
    if not data.strip():
        return np.zeros(0, np.int64)
    return np.array(data.split(), dtype=np.int64)


def _read_rows(path: str) -> list:
    with open(path) as f:
        return [ln.split() for ln in f if ln.strip()]


def read_csr(prefix: str):
    """(row_ptr int64 [n+1], col int32 [m], weights int32 [K, m] objective-major)."""
    row_ptr = _read_ints(prefix + "RowPtr.txt")
    col = _read_ints(prefix + "ColInd.txt").astype(np.int32)
    rows = _read_rows(prefix + "Values.txt")
    if len(rows) != col.size:
        raise ValueError(f"{prefix}Values.txt: {len(rows)} lines for {col.size} edges")
    k = len(rows[0]) if rows else 1
    if any(len(r) != k for r in rows):
        raise ValueError(f"{prefix}Values.txt: lines with different numbers of weights")
    w = np.array(rows, dtype=np.int64).reshape(col.size, k).T if rows else np.zeros((k, 0))
    return row_ptr, col, np.ascontiguousarray(w.astype(np.int32))


def write_csr(prefix: str, row_ptr, col, weights) -> None:
    w = np.asarray(weights).reshape(-1, len(col)) if len(col) else np.zeros((1, 0), np.int64)
    _write_lines(prefix + "RowPtr.txt", (str(int(x)) for x in row_ptr))
    _write_lines(prefix + "ColInd.txt", (str(int(x)) for x in col))
    _write_lines(prefix + "Values.txt", (" ".join(str(int(x)) for x in w[:, e])
                                         for e in range(len(col))))


def read_changes(directory: str, k: int):
    """(ins_src, ins_dst, ins_w [n_ins x K] insertion-major, del_src, del_dst)."""
    ins = _read_rows(os.path.join(directory, "insert.txt"))
    dele = _read_rows(os.path.join(directory, "delete.txt"))
    if any(len(r) != 2 + k for r in ins):
        raise ValueError(f"{directory}/insert.txt: lines must hold u v and {k} weights")
    if any(len(r) != 2 for r in dele):
        raise ValueError(f"{directory}/delete.txt: lines must hold u v")
    ia = np.array(ins, dtype=np.int64).reshape(-1, 2 + k)
    da = np.array(dele, dtype=np.int64).reshape(-1, 2)
    return (ia[:, 0].astype(np.int32), ia[:, 1].astype(np.int32),
            np.ascontiguousarray(ia[:, 2:].astype(np.int32)),
            da[:, 0].astype(np.int32), da[:, 1].astype(np.int32))


def write_changes(directory: str, ins_src, ins_dst, ins_w, del_src, del_dst) -> None:
    os.makedirs(directory, exist_ok=True)
    w = np.asarray(ins_w).reshape(len(ins_src), -1) if len(ins_src) else np.zeros((0, 1))
    _write_lines(os.path.join(directory, "insert.txt"),
                 (" ".join([str(int(u)), str(int(v))] + [str(int(x)) for x in w[i]])
                  for i, (u, v) in enumerate(zip(ins_src, ins_dst))))
    _write_lines(os.path.join(directory, "delete.txt"),
                 (f"{int(u)} {int(v)}" for u, v in zip(del_src, del_dst)))


def read_distances(path: str) -> np.ndarray:
    rows = _read_rows(path)
    d = np.zeros(len(rows), np.int64)
    for r in rows:
        v = int(r[0])
        d[v] = INF_DISTANCE if r[1] == "INF" else int(r[1])
    return d


def read_tree(path: str) -> np.ndarray:
    rows = _read_rows(path)
    p = np.zeros(len(rows), np.int32)
    for r in rows:
        p[int(r[0])] = int(r[1])
    return p


def write_distances(path: str, d) -> None:
    """Values >= INF / 2 print as INF (io/result_io.cpp:165-181)."""
    _write_lines(path, (f"{v} INF" if int(x) >= INF_DISTANCE // 2 else f"{v} {int(x)}"
                        for v, x in enumerate(d)))


def write_path_costs(path: str, costs) -> None:
    """n x K costs, one vertex per line (io/result_io.cpp:185-209)."""
    c = np.asarray(costs)
    _write_lines(path, (" ".join([str(v)] + ["INF" if int(x) >= INF_DISTANCE // 2 else str(int(x))
                                             for x in row]) for v, row in enumerate(c)))


def read_path_costs(path: str) -> np.ndarray:
    rows = _read_rows(path)
    k = len(rows[0]) - 1 if rows else 0
    out = np.zeros((len(rows), k), np.int64)
    for r in rows:
        out[int(r[0])] = [INF_DISTANCE if t == "INF" else int(t) for t in r[1:]]
    return out


def write_tree(path: str, p) -> None:
    _write_lines(path, (f"{v} {int(x)}" for v, x in enumerate(p)))


def _write_lines(path: str, lines) -> None:
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w", newline="\n") as f:
        for ln in lines:
            f.write(ln)
            f.write("\n")
