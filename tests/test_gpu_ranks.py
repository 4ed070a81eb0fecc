"""GPU: the decomposed run with one brick per rank (RankBricks over
torch.distributed), against the decomposed oracle run.

The ranks are processes sharing one GPU with the gloo backend: their halo
messages are staged through host memory by the transport and no kernel waits
on another rank's, so the ranks' kernels run independently. Each rank's brick
(halos included), the dt sequence and the field summaries (every rank holds
the whole deck's) must equal the oracle's decomposed run: arrays and dt bit for
bit, summaries to 1e-12 (the all-reduce adds in its own order).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import decks
from brick_harness import BrickOracle

pytestmark = pytest.mark.gpu

FIELDS = ("density0", "energy0", "pressure", "viscosity", "soundspeed", "density1", "energy1",
          "xvel0", "yvel0", "zvel0", "xvel1", "yvel1", "zvel1", "vol_flux_x", "vol_flux_y",
          "vol_flux_z", "mass_flux_x", "mass_flux_y", "mass_flux_z")


def deck_dict():
    return decks.shock(14, 11, 9, 20, states=decks.MIXED_STATES)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    import cloverleaf3d_ref_b200 as C
    from cloverleaf3d_ref_b200.ranks import RankBricks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    out = {"rank": rank}
    try:
        rb = RankBricks(decks.to_deck(deck_dict()), dist)
        out["steps"] = rb.run()
        out["dt"] = rb.dt_history()
        out["sums"], out["sum_steps"] = rb.summaries()
        out["extent"] = rb.extent
        out["fields"] = {f: rb.field(f) for f in FIELDS}
        rb.close()
        C.lib().clover_gpu_release()
    except Exception as e:  # reported to the parent
        out["error"] = repr(e)
    finally:
        q.put(out)
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_rank_bricks_match_decomposed_oracle(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got = sorted((q.get(timeout=300) for _ in range(world)), key=lambda o: o["rank"])
    finally:
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():
                p.kill()
    for o in got:
        assert "error" not in o, o.get("error")
    ref = BrickOracle(deck_dict(), world)
    steps = ref.run()
    for o in got:
        r = o["rank"]
        assert o["steps"] == steps
        assert tuple(int(v) for v in ref.ext[r]) == o["extent"]
        assert np.array_equal(o["dt"], np.array(ref.dts))
        assert np.array_equal(o["sum_steps"], np.array(ref.sum_steps))
        np.testing.assert_allclose(o["sums"], np.array(ref.sums), rtol=1e-12, atol=1e-300)
        for f in FIELDS:
            assert np.array_equal(o["fields"][f], ref.h[r].a[f]), (r, f)


def test_transport_failure_ends_the_run_with_an_error():
    """A transport that reports a failure (a peer that is gone, a closed
    channel) ends the brick driver with an error: the start fails when the
    first exchange fails, and a run fails at the first reduction that fails.
    One process, no peer: the callbacks are fakes."""
    import ctypes
    import cloverleaf3d_ref_b200 as C
    from cloverleaf3d_ref_b200.ranks import TransportStruct, _EXCHANGE, _MIN, _SUM
    L = C.lib()
    deck = decks.to_deck(deck_dict())
    calls = {"exchange": 0, "min": 0}

    def exchange_ok(ctx, axis, lo, s_lo, r_lo, n_lo, hi, s_hi, r_hi, n_hi):
        calls["exchange"] += 1
        return 0  # leaves the received halo as it was

    def exchange_fail(*a):
        calls["exchange"] += 1
        return 1

    def min_fail(ctx, p):
        calls["min"] += 1
        return 1

    def ok_sum(ctx, p, n):
        return 0

    cbs = [_EXCHANGE(exchange_fail), _MIN(min_fail), _SUM(ok_sum)]
    t = TransportStruct(None, 1, cbs[0], cbs[1], cbs[2])
    L.clover_gpu_clear_status()
    h = L.clover_bricks_create_rank(ctypes.byref(deck.s), 2, 0, ctypes.byref(t))
    assert not h and calls["exchange"] == 1
    cbs = [_EXCHANGE(exchange_ok), _MIN(min_fail), _SUM(ok_sum)]
    t = TransportStruct(None, 1, cbs[0], cbs[1], cbs[2])
    h = L.clover_bricks_create_rank(ctypes.byref(deck.s), 2, 0, ctypes.byref(t))
    assert h
    assert L.clover_bricks_run(h, 5) == -1 and calls["min"] == 1
    L.clover_bricks_destroy(h)
    L.clover_gpu_clear_status()
