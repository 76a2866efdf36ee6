"""The C ABI library builds for sm_100a, loads without a GPU and exports every symbol that
include/dyngb200.h declares (no compute calls here)."""
import ctypes
import os

from dyng_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    from dyng_b200 import build
    build.build()
    lib = ctypes.CDLL(N.LIB_PATH)
    headers = [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))
               if h.endswith(".h")]
    declared = sorted({s for h in headers for s in N.declared_symbols(h)})
    assert len(declared) >= 27
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # the ctypes table covers the header exactly
    assert set(declared) == set(N.SIGNATURES)


def test_host_only_entry_points():
    L = N.lib()
    assert L.dyngb200_abi_version() == 1
    assert L.dyngb200_status_name(3) == b"stale_result"
    p = N.Props()
    L.dyngb200_props_default(ctypes.byref(p))
    assert (p.directed, p.sorted, p.allow_multi, p.deletions_first) == (1, 1, 0, 1)
    L.dyngb200_props_mosp_compatible(ctypes.byref(p))
    assert (p.sorted, p.allow_multi) == (0, 1)


def test_generators_are_deterministic():
    import numpy as np
    from dyng_b200 import generators as G
    a = G.rmat(10, 8, seed=5)
    b = G.rmat(10, 8, seed=5)
    assert np.array_equal(a.src, b.src) and np.array_equal(a.weights, b.weights)
    assert np.all(a.src != a.dst)
    key = (a.src.astype(np.int64) << 32) | a.dst
    assert np.all(np.diff(key) > 0)  # sorted, no duplicate pairs
    g = G.grid(16, seed=2)
    assert g.num_vertices == 256 and g.weights.min() >= 1


def test_null_handles_are_argument_errors_on_the_host():
    """A null handle is refused before anything reaches the device (so this runs without a GPU):
    INVALID_ARGUMENT with a message naming the reference's call; destroying null is a no-op."""
    L = N.lib()
    st = N.Stats()
    status = L.dyngb200_sssp_update(None, None, None, None, ctypes.byref(st))
    assert L.dyngb200_status_name(status) == b"invalid_argument"
    assert L.dyngb200_last_error_message().startswith(b"sssp::update")
    assert L.dyngb200_status_name(L.dyngb200_context_synchronize(None)) == b"invalid_argument"
    for destroy in (L.dyngb200_graph_destroy, L.dyngb200_tree_destroy,
                    L.dyngb200_context_destroy):
        assert destroy(None) == 0
