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


def test_abi_reports_a_staged_wait_that_ran_out():
    """The drop-in ABI's staged kernels report a bounded wait that gave up
    through the library's device status word, read back at the next
    synchronisation: CLOVER_STATUS_TIMEOUT with a message, and the calls that
    follow (status cleared) still match the oracle bit for bit."""
    L = C.lib()
    L.clover_gpu_wait_selftest_queued.argtypes = [ctypes.c_longlong]
    L.clover_gpu_wait_selftest_queued.restype = ctypes.c_int
    L.clover_gpu_release()
    L.clover_gpu_clear_status()
    d = decks.shock(12, 10, 8, 6, states=decks.MIXED_STATES)
    r = O.run(d, max_steps=6, want_fields=True)
    di = C.DropIn(decks.to_deck(d))
    try:
        assert di.run(2) == 2
        assert L.clover_gpu_status() == 0
        assert L.clover_gpu_wait_selftest_queued(10_000_000) == 0  # ~5 ms of SM clocks
        L.clover_gpu_synchronize()
        assert L.clover_gpu_status() & STATUS_TIMEOUT
        assert b"gave up" in L.clover_gpu_error_string()
        L.clover_gpu_clear_status()
        assert di.run(6) == r["steps"]
        assert L.clover_gpu_status() == 0
        assert np.array_equal(di.dt_history(), r["dt"])
        assert np.array_equal(di.field("density0"), r["fields"]["density0"])
    finally:
        di.close()
        L.clover_gpu_release()
        L.clover_gpu_clear_status()
