"""Failure detection of the staged kernels, tested without a GPU fault.

Every wait of a kernel that stages its planes with bulk-tensor copies is
bounded: if a plane's copies do not arrive within about a second, the block
stops, sets CLOVER_STATUS_TIMEOUT in the chunk's status word and returns. Here
the same bounded wait is made to run out on a barrier phase that nothing
completes (clover_gpu_wait_selftest, with a limit of a few milliseconds); the
status comes back and the device keeps working: a run right after it matches
the oracle bit for bit.
"""
import ctypes
import time

import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks
import oracle_lib as O

pytestmark = pytest.mark.gpu

STATUS_TIMEOUT = 0x20


def test_bounded_wait_runs_out_and_reports_timeout():
    L = C.lib()
    L.clover_gpu_wait_selftest.argtypes = [ctypes.c_longlong]
    L.clover_gpu_wait_selftest.restype = ctypes.c_int
    t0 = time.perf_counter()
    assert L.clover_gpu_wait_selftest(10_000_000) == STATUS_TIMEOUT  # ~5 ms of SM clocks
    assert time.perf_counter() - t0 < 30.0
    # the context is intact: a chunk runs after it and matches the oracle
    d = decks.shock(12, 10, 8, 12, states=decks.MIXED_STATES)
    r = O.run(d, want_fields=True)
    ch = C.Chunk(decks.to_deck(d))
    try:
        assert ch.run() == r["steps"]
        assert ch.status == 0
        assert np.array_equal(ch.dt_history(), r["dt"])
        assert np.array_equal(ch.field("density0"), r["fields"]["density0"])
    finally:
        ch.close()
