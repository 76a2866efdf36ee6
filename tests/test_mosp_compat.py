"""The MOSP text formats and the compat driver (python -m dyng_b200.compat).

CPU: the writers reproduce the reference's fixture files byte for byte (where the reference tree
is present), and every reader/writer pair round-trips.  GPU: the driver, run on each golden case
written out in MOSP's format, writes the golden updated trees byte for byte and reports the
golden `invalidated` per objective (the reference's mosp_compat replay of the 34 cases); with
--mosp it writes the golden combinedGraph/ files of the 8 preference cases byte for byte
(python/tests/test_cli.py:686-723)."""
import os

import numpy as np
import pytest

from dyng_b200 import mosp_io as io
from tests.helpers import combined_case, fixture_case

# the reference's fixture tree, when DYNG_REFERENCE names a dynG source tree (else skipped)
REFERENCE_DATA = os.path.join(os.environ.get("DYNG_REFERENCE", "/nonexistent"),
                              "cpp", "tests", "data")
REFERENCE_FIXTURES = os.path.join(REFERENCE_DATA, "mosp_sssp")


def _cases(z):
    return [str(c) for c in z["cases"]]


def test_round_trips(tmp_path):
    rng = np.random.default_rng(0)
    row_ptr = np.array([0, 2, 2, 5], np.int64)
    col = np.array([1, 2, 0, 1, 2], np.int32)
    w = rng.integers(1, 100, (3, 5)).astype(np.int32)
    io.write_csr(str(tmp_path / "g"), row_ptr, col, w)
    r, c, ww = io.read_csr(str(tmp_path / "g"))
    assert np.array_equal(r, row_ptr) and np.array_equal(c, col) and np.array_equal(ww, w)
    ins_w = rng.integers(1, 9, (2, 3)).astype(np.int32)
    io.write_changes(str(tmp_path / "ch"), [0, 2], [1, 0], ins_w, [1], [2])
    s, t, iw, ds, dd = io.read_changes(str(tmp_path / "ch"), 3)
    assert s.tolist() == [0, 2] and t.tolist() == [1, 0] and np.array_equal(iw, ins_w)
    assert ds.tolist() == [1] and dd.tolist() == [2]
    d = np.array([0, 5, io.INF_DISTANCE], np.int64)
    io.write_distances(str(tmp_path / "o" / "d.txt"), d)
    assert (tmp_path / "o" / "d.txt").read_bytes() == b"0 0\n1 5\n2 INF\n"
    assert np.array_equal(io.read_distances(str(tmp_path / "o" / "d.txt")), d)
    io.write_tree(str(tmp_path / "o" / "p.txt"), [-1, 0, -1])
    assert io.read_tree(str(tmp_path / "o" / "p.txt")).tolist() == [-1, 0, -1]
    io.write_changes(str(tmp_path / "empty"), [], [], np.zeros((0, 1)), [], [])
    assert (tmp_path / "empty" / "delete.txt").read_bytes() == b""


@pytest.mark.skipif(not os.path.isdir(REFERENCE_FIXTURES), reason="reference tree absent")
def test_writers_reproduce_the_reference_files_byte_for_byte(tmp_path):
    done = 0
    for case in sorted(os.listdir(REFERENCE_FIXTURES)):
        base = os.path.join(REFERENCE_FIXTURES, case)
        if not os.path.isdir(os.path.join(base, "input")):
            continue
        for stage, names in (("init", ("distancesOriginal.txt", "SSSPTreeOriginal.txt")),
                             ("updated", ("distancesUpdated.txt", "SSSPTreeUpdated.txt"))):
            for obj in sorted(os.listdir(os.path.join(base, stage))):
                dist, tree = (os.path.join(base, stage, obj, n) for n in names)
                io.write_distances(str(tmp_path / "d.txt"), io.read_distances(dist))
                io.write_tree(str(tmp_path / "p.txt"), io.read_tree(tree))
                assert (tmp_path / "d.txt").read_bytes() == open(dist, "rb").read(), dist
                assert (tmp_path / "p.txt").read_bytes() == open(tree, "rb").read(), tree
                done += 1
        prefix = os.path.join(base, "input", "graphCsr")
        io.write_csr(str(tmp_path / "g"), *io.read_csr(prefix))
        for suffix in ("RowPtr.txt", "ColInd.txt", "Values.txt"):
            assert (tmp_path / ("g" + suffix)).read_bytes() == open(prefix + suffix, "rb").read()
        k = io.read_csr(prefix)[2].shape[0]
        io.write_changes(str(tmp_path / "ch"), *io.read_changes(os.path.join(base, "input"), k))
        for n in ("insert.txt", "delete.txt"):
            assert (tmp_path / "ch" / n).read_bytes() == open(os.path.join(base, "input", n),
                                                              "rb").read()
    assert done >= 10


def _write_case(root, c):
    k = c["k"]
    io.write_csr(os.path.join(root, "input", "graphCsr"), c["row_ptr"], c["col"], c["w"])
    io.write_changes(os.path.join(root, "input"), c["ins_src"], c["ins_dst"],
                     c["ins_w"].reshape(-1, k), c["del_src"], c["del_dst"])
    for j in range(k):
        io.write_distances(os.path.join(root, "init", f"obj{j}", "distancesOriginal.txt"),
                           c["init_d"][j])
        io.write_tree(os.path.join(root, "init", f"obj{j}", "SSSPTreeOriginal.txt"),
                      c["init_p"][j])


def test_cost_files_round_trip(tmp_path):
    costs = np.array([[0, 0, 0], [7, 17, io.INF_DISTANCE], [3, 4, 5]], np.int64)
    io.write_path_costs(str(tmp_path / "c.txt"), costs)
    assert (tmp_path / "c.txt").read_bytes() == b"0 0 0 0\n1 7 17 INF\n2 3 4 5\n"
    assert np.array_equal(io.read_path_costs(str(tmp_path / "c.txt")), costs)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE_DATA, "mosp_combined")),
                    reason="reference tree absent")
def test_combined_writers_reproduce_the_reference_files(tmp_path):
    root = os.path.join(REFERENCE_DATA, "mosp_combined")
    done = 0
    for case in sorted(os.listdir(root)):
        cd = os.path.join(root, case, "combined")
        if not os.path.isdir(cd):
            continue
        d, p, c = (os.path.join(cd, x) for x in ("distancesCsr.txt", "SSSPTreeCsr.txt",
                                                  "mospCosts.txt"))
        io.write_distances(str(tmp_path / "d.txt"), io.read_distances(d))
        io.write_tree(str(tmp_path / "p.txt"), io.read_tree(p))
        io.write_path_costs(str(tmp_path / "c.txt"), io.read_path_costs(c))
        for mine, theirs in (("d.txt", d), ("p.txt", p), ("c.txt", c)):
            assert (tmp_path / mine).read_bytes() == open(theirs, "rb").read(), theirs
        done += 1
    assert done == 8


@pytest.mark.gpu
def test_compat_driver_replays_every_golden_case(fixtures, tmp_path):
    from dyng_b200 import compat
    done = 0
    for name in _cases(fixtures):
        c = fixture_case(fixtures, name)
        root = tmp_path / name
        _write_case(str(root), c)
        lines = []
        compat.run_update(str(root / "input" / "graphCsr"), str(root / "input"), str(root / "init"),
                          str(root / "out"), log=lines.append)
        assert lines == [f"obj{j} invalidated {int(c['invalidated'][j])}" for j in range(c["k"])]
        for j in range(c["k"]):
            io.write_distances(str(root / "want_d.txt"), c["upd_d"][j])
            io.write_tree(str(root / "want_p.txt"), c["upd_p"][j])
            got = root / "out" / f"obj{j}"
            assert (got / "distancesUpdated.txt").read_bytes() == (root / "want_d.txt").read_bytes()
            assert (got / "SSSPTreeUpdated.txt").read_bytes() == (root / "want_p.txt").read_bytes()
        done += 1
    assert done == len(_cases(fixtures)) >= 34


@pytest.mark.gpu
def test_compat_driver_mosp_mode_replays_the_combined_cases(combined_fixtures, tmp_path):
    from dyng_b200 import compat
    names = [str(x) for x in combined_fixtures["cases"]]
    for name in names:
        c = combined_case(combined_fixtures, name)
        root = tmp_path / name
        io.write_csr(str(root / "input" / "graphCsr"), c["row_ptr"], c["col"], c["w"])
        io.write_changes(str(root / "input"), c["ins_src"], c["ins_dst"],
                         c["ins_w"].reshape(-1, c["kg"]), c["del_src"], c["del_dst"])
        for j in range(c["k"]):
            io.write_distances(str(root / "init" / f"obj{j}" / "distancesOriginal.txt"),
                               c["init_d"][j])
            io.write_tree(str(root / "init" / f"obj{j}" / "SSSPTreeOriginal.txt"), c["init_p"][j])
        lines = []
        compat.main(["--graph", str(root / "input" / "graphCsr"), "--changes", str(root / "input"),
                     "--init", str(root / "init"), "--out", str(root / "out"), "-k", str(c["k"]),
                     "--mosp", "--pref", ",".join(str(p) for p in c["pref"])])
        io.write_distances(str(root / "want_d.txt"), c["combined_d"])
        io.write_tree(str(root / "want_p.txt"), c["combined_p"])
        io.write_path_costs(str(root / "want_c.txt"), c["costs"])
        got = root / "out" / "combinedGraph"
        assert (got / "distancesCsr.txt").read_bytes() == (root / "want_d.txt").read_bytes(), name
        assert (got / "SSSPTreeCsr.txt").read_bytes() == (root / "want_p.txt").read_bytes(), name
        assert (got / "mospCosts.txt").read_bytes() == (root / "want_c.txt").read_bytes(), name
        assert sorted(p.name for p in (root / "out").iterdir()) == ["combinedGraph"] + [
            f"obj{j}" for j in range(c["k"])]
    assert len(names) == 8
