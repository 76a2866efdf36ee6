"""The update's statistics record on the CPU (dyng_b200/sssp.py, Stats over the C ABI's
dyngb200_stats): the algorithmic-byte accounting behind the bench line's roofline and its
per-phase split, and the reference's profiler stage names (parity/timed_regions/sssp.toml)."""
import numpy as np

from dyng_b200 import _native as N
from dyng_b200 import sssp as S


def _stats(work, phase_ms, affected=0, apply_ms=0.0, sssp_ms=0.0):
    s = N.Stats()
    for i, v in enumerate(work):
        s.work[i] = v
    for i, v in enumerate(phase_ms):
        s.phase_ms[i] = v
    s.affected = affected
    s.apply_ms = apply_ms
    s.sssp_ms = sssp_ms
    return S.Stats(s)


def test_work_tables_cover_the_native_counters():
    n = len(N.Stats().work)
    assert len(S.Stats.WORK_BYTES) == n
    assert len(S.Stats.WORK_NAMES) <= n
    # counters past the named ones carry no bytes
    assert all(b == 0 for b in S.Stats.WORK_BYTES[len(S.Stats.WORK_NAMES):])
    assert len(S.Stats.PHASES) == len(N.Stats().phase_ms)


def test_every_counter_with_bytes_belongs_to_exactly_one_phase():
    owned = [i for units, _ in S.Stats.PHASE_WORK.values() for i in units]
    assert len(owned) == len(set(owned))
    with_bytes = {i for i, b in enumerate(S.Stats.WORK_BYTES) if b > 0}
    assert with_bytes == set(owned)
    timed = sorted(p for _, phases in S.Stats.PHASE_WORK.values() for p in phases)
    assert timed == list(range(len(S.Stats.PHASES)))


def test_phase_bytes_add_up_to_the_total():
    rng = np.random.default_rng(3)
    work = rng.integers(0, 10**6, len(S.Stats.WORK_BYTES)).tolist()
    ms = rng.uniform(0.001, 0.2, len(S.Stats.PHASES)).tolist()
    st = _stats(work, ms, affected=1234)
    split = st.phase_bytes_ms()
    assert set(split) == set(S.Stats.PHASE_WORK)
    total = sum(b for b, _ in split.values())
    assert total == st.algorithmic_bytes + 12 * 1234  # the unpack's result writes
    assert np.isclose(sum(t for _, t in split.values()), sum(ms))


def test_bytes_per_unit():
    names = S.Stats.WORK_NAMES
    per_unit = dict(zip(names, S.Stats.WORK_BYTES))
    # ancestor + flag per visit; list entry, row descriptor and own word per pull candidate and
    # per pushed vertex; column + weight per slot; one packed word per read and per atomicMin
    assert per_unit["round_visits"] == 8 and per_unit["jumps"] == 12
    assert per_unit["pull_candidates"] == 20 and per_unit["pushes"] == 20
    assert per_unit["pull_slots"] == 8 and per_unit["push_slots"] == 8
    assert per_unit["push_words"] == 8 and per_unit["atomics"] == 8
    assert per_unit["unpacked"] == 20 and per_unit["stamps_scanned"] == 4
    assert per_unit["atomic_attempts"] == 0  # a diagnostic, not traffic
    one = [0] * len(S.Stats.WORK_BYTES)
    one[names.index("pushes")] = 10
    one[names.index("push_slots")] = 160
    assert _stats(one, [0.0] * 7).algorithmic_bytes == 10 * 20 + 160 * 8


def test_stages_use_the_reference_profiler_names():
    ms = [0.01, 0.1, 0.002, 0.012, 0.05, 0.2, 0.025]
    st = _stats([0] * len(S.Stats.WORK_BYTES), ms, apply_ms=0.17, sssp_ms=0.45)
    stages = st.stages_ms()
    assert set(stages) == {"sssp.update", "sssp.commit", "graph.apply", "graph.transpose",
                           "sssp.identify_affected", "sssp.seed", "sssp.loop", "sssp.finalize"}
    assert np.isclose(stages["sssp.update"], 0.62)
    assert stages["graph.apply"] == stages["sssp.commit"]
    assert np.isclose(stages["graph.apply"], 0.17)  # the native field is a float
    assert np.isclose(stages["sssp.identify_affected"], 0.01 + 0.1 + 0.002)
    assert np.isclose(stages["sssp.seed"], 0.012 + 0.05)
    assert np.isclose(stages["sssp.loop"], 0.2) and np.isclose(stages["sssp.finalize"], 0.025)
