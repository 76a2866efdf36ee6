"""A batch wider than the applier's shared-memory pair stages, against the oracle.

The pair step of the batch applier groups a batch's operations by (u, v) pair and lists the new
pairs and touched rows through a stage of 3,072 entries per list in each block's shared memory;
a block whose share of the batch holds more falls back to appending to the global lists
directly.  The persistent grid has 444 blocks, so only a batch of more than about 1.36 M new
pairs reaches that fallback: here R-MAT scale 18 takes a 2M-change batch (about 2 M pairs,
every block's stage overflowing) and then a 100k-change batch, each compared with the oracle
(distances, parents, `invalidated`, `affected` and the apply summary).
"""
import numpy as np
import pytest

import dyng_b200 as D
from dyng_b200 import generators as G
from oracle import oracle as O
from tests.test_gpu_scale_parity import _check, _gpu_batch, _oracle_batch, oracle_threads  # noqa: F401

pytestmark = pytest.mark.gpu

STAGE_ENTRIES = 3072
PERSISTENT_BLOCKS = 444


def test_a_batch_wider_than_every_pair_stage_matches_the_oracle(oracle_threads):  # noqa: F811
    e = G.rmat(18, 16, w_max=1000, seed=5)
    rp, col, w = e.csr()
    og = O.Graph.from_csr(rp, col, w, 1, O.default_props())
    ot, _ = O.compute(og, 0, rule=1)
    g = D.Graph.from_csr(rp, col, w)
    t = D.sssp.compute(g, 0)
    np.testing.assert_array_equal(t.distances, ot.distances)
    np.testing.assert_array_equal(t.parents, ot.parents)
    stream = G.BatchStream(e, seed=9)
    for size in (2_000_000, 100_000):
        b = stream.next(size, 0.75, 0.5, parents=ot.parents)
        ost, osm = O.update(og, _oracle_batch(b), ot)
        st = D.sssp.update(g, _gpu_batch(b), t)
        _check(f"{size} changes", t, st, ot, ost, osm)
        if size == 2_000_000:
            # the batch's pairs exceed what the stages of all blocks hold together
            assert osm["inserted_edges"] + osm["deleted_edges"] > STAGE_ENTRIES * PERSISTENT_BLOCKS
    assert g.num_edges() == og.m
