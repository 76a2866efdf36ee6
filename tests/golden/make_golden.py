"""Convert the reference's golden fixtures into tests/golden/mosp_fixtures.npz and
tests/golden/mosp_combined.npz.

Run once, in a checkout where the dynG reference tree is present:

    python tests/golden/make_golden.py /path/to/dyng

It reads (never modifies) three fixture directories of the reference:
  - cpp/tests/data/mosp_sssp/   34 cases (cases.txt): for every objective k the initial tree
    (init/obj<k>/{distancesOriginal,SSSPTreeOriginal}.txt, "v d" / "v INF", "v p"), the tree
    after one update (updated/obj<k>/...) and stats.txt ("obj<k> invalidated <n>");
  - cpp/tests/data/mosp_graph_io/<case>/applied/  the CSR after the batch, its transpose and the
    weight-increase mask (one line per insertion, K flags);
  - cpp/tests/data/mosp_combined/  8 cases (cases.txt: name, input dir, init dir, K, preferences):
    the combined graph after the batch (combined/distancesCsr.txt "v d", SSSPTreeCsr.txt "v p",
    mospCosts.txt "v c_1 .. c_KG" over every weight column of the graph), from the K initial
    trees under init/.
Inputs: graphCsr{RowPtr,ColInd,Values}.txt (one row offset / neighbour per line, K weights per
line), insert.txt ("u v w1 .. wK") and delete.txt ("u v").  Blank lines are skipped.

The npz keys are "<case>/<array>"; INF distances are stored as INT64_MAX // 4.  The consumer is
tests/test_oracle.py (CPU) and tests/test_parity_fixtures.py (GPU), which must run where the
reference tree is absent, hence this committed copy of the data.
"""
from __future__ import annotations

import os
import sys

import numpy as np

INF = (2**63 - 1) // 4


def _rows(path):
    if not os.path.exists(path):
        return []
    out = []
    with open(path) as f:
        for line in f:
            toks = line.split()
            if toks:
                out.append(toks)
    return out


def _ints(path):
    return [int(t[0]) for t in _rows(path)]


def _vertex_values(path, n, inf_ok):
    vals = np.zeros(n, np.int64)
    for toks in _rows(path):
        v = int(toks[0])
        vals[v] = INF if (inf_ok and toks[1] == "INF") else int(toks[1])
    return vals


def _csr(prefix, k):
    rp = np.asarray(_ints(prefix + "RowPtr.txt"), np.int64)
    col = np.asarray(_ints(prefix + "ColInd.txt"), np.int32)
    vals = _rows(prefix + "Values.txt")
    w = np.asarray([[int(x) for x in r[:k]] for r in vals], np.int32).reshape(-1, k)
    return rp, col, np.ascontiguousarray(w.T)  # objective-major


def main(root):
    data = os.path.join(root, "cpp", "tests", "data")
    out = {}
    names = []
    for line in open(os.path.join(data, "mosp_sssp", "cases.txt")):
        toks = line.split()
        if not toks:
            continue
        name, inp, k = toks[0], toks[1], int(toks[2])
        names.append(name)
        ind = os.path.join(data, inp)
        rp, col, w = _csr(os.path.join(ind, "graphCsr"), k)
        n = rp.size - 1
        ins = _rows(os.path.join(ind, "insert.txt"))
        dele = _rows(os.path.join(ind, "delete.txt"))
        out[f"{name}/k"] = np.int64(k)
        out[f"{name}/row_ptr"] = rp
        out[f"{name}/col"] = col
        out[f"{name}/w"] = w
        out[f"{name}/ins"] = np.asarray([[int(x) for x in r[:2 + k]] for r in ins],
                                        np.int32).reshape(-1, 2 + k)
        out[f"{name}/del"] = np.asarray([[int(x) for x in r[:2]] for r in dele],
                                        np.int32).reshape(-1, 2)
        exp = os.path.join(data, "mosp_sssp", name)
        inval = {}
        for toks in _rows(os.path.join(exp, "stats.txt")):
            inval[int(toks[0][3:])] = int(toks[2])
        out[f"{name}/invalidated"] = np.asarray([inval[j] for j in range(k)], np.int64)
        for j in range(k):
            ob = f"obj{j}"
            out[f"{name}/init_d{j}"] = _vertex_values(
                os.path.join(exp, "init", ob, "distancesOriginal.txt"), n, True)
            out[f"{name}/init_p{j}"] = _vertex_values(
                os.path.join(exp, "init", ob, "SSSPTreeOriginal.txt"), n, False).astype(np.int32)
            nu = len(_rows(os.path.join(exp, "updated", ob, "distancesUpdated.txt")))
            out[f"{name}/upd_d{j}"] = _vertex_values(
                os.path.join(exp, "updated", ob, "distancesUpdated.txt"), nu, True)
            out[f"{name}/upd_p{j}"] = _vertex_values(
                os.path.join(exp, "updated", ob, "SSSPTreeUpdated.txt"), nu, False).astype(np.int32)
        app = os.path.join(ind, "applied")
        if os.path.isdir(app):
            arp, acol, aw = _csr(os.path.join(app, "graphCsr"), k)
            trp, tcol, tw = _csr(os.path.join(app, "graphCsrTransposed"), k)
            mask = _rows(os.path.join(app, "graphCsrWeightIncrease.txt"))
            out[f"{name}/applied_row_ptr"] = arp
            out[f"{name}/applied_col"] = acol
            out[f"{name}/applied_w"] = aw
            out[f"{name}/applied_in_row_ptr"] = trp
            out[f"{name}/applied_in_col"] = tcol
            out[f"{name}/applied_in_w"] = tw
            out[f"{name}/applied_increase"] = np.asarray(
                [[int(x) for x in r[:k]] for r in mask], np.uint8).reshape(-1, k)
    out["cases"] = np.asarray(names)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mosp_fixtures.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst}: {len(names)} cases")
    combined(data)


def _columns(prefix):
    rows = _rows(prefix + "Values.txt")
    return len(rows[0]) if rows else 1


def combined(data):
    out = {}
    names = []
    for line in open(os.path.join(data, "mosp_combined", "cases.txt")):
        toks = line.split()
        if not toks:
            continue
        name, inp, init, k, pref = toks[0], toks[1], toks[2], int(toks[3]), toks[4]
        names.append(name)
        ind = os.path.join(data, inp)
        kg = _columns(os.path.join(ind, "graphCsr"))
        rp, col, w = _csr(os.path.join(ind, "graphCsr"), kg)
        n = rp.size - 1
        ins = _rows(os.path.join(ind, "insert.txt"))
        dele = _rows(os.path.join(ind, "delete.txt"))
        out[f"{name}/k"] = np.int64(k)
        out[f"{name}/kg"] = np.int64(kg)
        out[f"{name}/pref"] = np.asarray([int(x) for x in pref.split(",")], np.int32)
        out[f"{name}/row_ptr"] = rp
        out[f"{name}/col"] = col
        out[f"{name}/w"] = w
        out[f"{name}/ins"] = np.asarray([[int(x) for x in r[:2 + kg]] for r in ins],
                                        np.int32).reshape(-1, 2 + kg)
        out[f"{name}/del"] = np.asarray([[int(x) for x in r[:2]] for r in dele],
                                        np.int32).reshape(-1, 2)
        for j in range(k):
            ob = os.path.join(data, init, f"obj{j}")
            out[f"{name}/init_d{j}"] = _vertex_values(
                os.path.join(ob, "distancesOriginal.txt"), n, True)
            out[f"{name}/init_p{j}"] = _vertex_values(
                os.path.join(ob, "SSSPTreeOriginal.txt"), n, False).astype(np.int32)
        cd = os.path.join(data, "mosp_combined", name, "combined")
        nu = len(_rows(os.path.join(cd, "distancesCsr.txt")))
        out[f"{name}/combined_d"] = _vertex_values(os.path.join(cd, "distancesCsr.txt"), nu, True)
        out[f"{name}/combined_p"] = _vertex_values(
            os.path.join(cd, "SSSPTreeCsr.txt"), nu, False).astype(np.int32)
        costs = np.zeros((nu, kg), np.int64)
        for toks in _rows(os.path.join(cd, "mospCosts.txt")):
            costs[int(toks[0])] = [INF if t == "INF" else int(t) for t in toks[1:1 + kg]]
        out[f"{name}/costs"] = costs
    out["cases"] = np.asarray(names)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mosp_combined.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst}: {len(names)} cases")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DYNG_REFERENCE")
    if not root:
        sys.exit("usage: python tests/golden/make_golden.py <dynG source tree> "
                 "(or set DYNG_REFERENCE)")
    main(root)
