"""The allocation-free compute entry point (dyngb200_sssp_compute_static_scratch).

It exists for callers that must not allocate device memory while they run -- serving processes
that fix their memory budget at start-up, host frameworks that own the allocator -- so its
scratch is a fixed device array inside the library.
This file checks, through the C ABI, that two calls in a row give the same distances and parents
as the regular entry point (dyngb200_sssp_compute), and that graphs beyond the array's limit
are refused.  It is collected last so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

import dyng_b200 as D
from dyng_b200 import _native as N
from dyng_b200 import generators as G

pytestmark = pytest.mark.gpu


def _static_compute(graph, source, n, objective=0, delta=0):
    import torch
    dist = torch.empty(n, dtype=torch.int64, device="cuda")
    par = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    status = N.lib().dyngb200_sssp_compute_static_scratch(
        graph._h, source, objective, delta,
        ctypes.cast(ctypes.c_void_p(dist.data_ptr()), N.c_i64p),
        ctypes.cast(ctypes.c_void_p(par.data_ptr()), N.c_i32p), None)
    return status, dist.cpu().numpy(), par.cpu().numpy()


def test_static_scratch_matches_regular_compute_twice():
    e = G.rmat(14, 8, w_max=1000, seed=21)
    rp, col, w = e.csr()
    g = D.Graph.from_csr(rp, col, w)
    n = g.num_vertices()
    for source in (0, 17):  # two calls in a row share (and must reset) the static array
        ref = D.sssp.compute(g, source)
        status, d, p = _static_compute(g, source, n)
        assert status == 0, N.lib().dyngb200_last_error_message().decode()
        np.testing.assert_array_equal(d, ref.distances)
        np.testing.assert_array_equal(p, ref.parents)


def test_static_scratch_call_allocates_nothing():
    # after a warm-up call, a call on a fresh source leaves the library's allocation count, torch's
    # allocator and the device's free memory exactly where they were
    import gc

    import torch
    from dyng_b200.graph import device_allocations
    e = G.rmat(12, 8, w_max=100, seed=5)
    rp, col, w = e.csr()
    g = D.Graph.from_csr(rp, col, w)
    n = g.num_vertices()
    D.sssp.compute(g, 0)  # column statistics current
    dist = torch.empty(n, dtype=torch.int64, device="cuda")
    par = torch.empty(n, dtype=torch.int32, device="cuda")
    lib = N.lib()

    def call(source):
        return lib.dyngb200_sssp_compute_static_scratch(
            g._h, source, 0, 0, ctypes.cast(ctypes.c_void_p(dist.data_ptr()), N.c_i64p),
            ctypes.cast(ctypes.c_void_p(par.data_ptr()), N.c_i32p), None)

    assert call(1) == 0, lib.dyngb200_last_error_message().decode()
    gc.collect()
    torch.cuda.synchronize()
    before = (device_allocations(), torch.cuda.memory_allocated(), torch.cuda.mem_get_info()[0])
    assert call(2) == 0, lib.dyngb200_last_error_message().decode()
    torch.cuda.synchronize()
    after = (device_allocations(), torch.cuda.memory_allocated(), torch.cuda.mem_get_info()[0])
    assert after == before
    ref = D.sssp.compute(g, 2)
    np.testing.assert_array_equal(dist.cpu().numpy(), ref.distances)
    np.testing.assert_array_equal(par.cpu().numpy(), ref.parents)


def test_static_scratch_refuses_large_graphs():
    n = (1 << 16) + 5
    src = np.arange(n - 1, dtype=np.int32)
    g = D.Graph.from_edges(src, src + 1, np.ones(n - 1, np.int32), n)
    status, _, _ = _static_compute(g, 0, n)
    assert status == 1  # DYNGB200_INVALID_ARGUMENT
    assert b"65536" in N.lib().dyngb200_last_error_message()
