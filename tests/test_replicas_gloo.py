"""CPU: the multi-rank host logic of the replica / ensemble-partition path,
run as two gloo ranks on 127.0.0.1 (world size 2).

Each rank draws the same seeded ensemble decks, takes its share with
deck_share, and the shares are gathered: every deck is taken by exactly one
rank and the cells are balanced. max_over_ranks gives every rank the
largest of the ranks' values."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from cloverleaf3d_ref_b200.replicas import deck_share, max_over_ranks


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    import cloverleaf3d_ref_b200 as C
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        decks = C.draw_decks(64, 2024, cells=(24, 128), end_step=150)
        cells = [d.cells for d in decks]
        mine = deck_share(cells, rank, world)
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        # a timing that differs per rank: the max must reach every rank
        t = max_over_ranks(10.0 + 7.5 * rank, dist, "cpu")
        dist.barrier()
        q.put((rank, cells, shares, t))
    finally:
        dist.destroy_process_group()


def test_deck_share_single_rank_takes_all():
    assert deck_share([5, 1, 3], 0, 1) == [0, 1, 2]
    assert deck_share([], 0, 3) == []
    with pytest.raises(ValueError):
        deck_share([1], 2, 2)


def test_deck_share_balances_cells():
    cells = [100, 90, 80, 10, 10, 10]
    shares = [deck_share(cells, r, 3) for r in range(3)]
    assert sorted(i for s in shares for i in s) == list(range(6))
    loads = [sum(cells[i] for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(cells)


def test_max_over_ranks_without_group():
    assert max_over_ranks(3.25) == 3.25


def test_two_gloo_ranks_partition_decks_and_take_max_time():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got = [q.get(timeout=180) for _ in range(world)]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    got.sort()
    cells = got[0][1]
    for rank, c, shares, t in got:
        assert c == cells  # every rank drew the same decks
        assert shares == got[0][2]  # and computed the same partition
        assert t == 17.5
    shares = got[0][2]
    taken = sorted(i for s in shares for i in s)
    assert taken == list(range(len(cells)))
    loads = [sum(cells[i] for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(cells)
    assert all(len(s) > 0 for s in shares)


# ---- the transport of the one-brick-per-rank decomposed run ----

def transport_main(rank, world, port, q):
    import ctypes
    import datetime
    import numpy as np
    import torch.distributed as dist
    from cloverleaf3d_ref_b200.ranks import DistTransport
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t = DistTransport(dist)
        chunk = rank + 1
        lo = chunk - 1 if chunk > 1 else -1
        hi = chunk + 1 if chunk < world else -1
        n = 5 + rank  # each pair's messages share a length: the lower rank's
        n_lo = 5 + (rank - 1) if lo > 0 else 0
        n_hi = n if hi > 0 else 0
        bufs = [np.full(max(n_lo, 1), 100.0 * chunk + 1), np.zeros(max(n_lo, 1)),
                np.full(max(n_hi, 1), 100.0 * chunk + 2), np.zeros(max(n_hi, 1))]
        P = [b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for b in bufs]
        rc = t.s.exchange(None, 0, lo, P[0], P[1], n_lo, hi, P[2], P[3], n_hi)
        v = (ctypes.c_double * 1)(10.0 - rank)
        rc_min = t.s.min(None, v)
        s = (ctypes.c_double * 5)(*[float(rank + i) for i in range(5)])
        rc_sum = t.s.sum(None, s, 5)
        dist.barrier()
        q.put((rank, rc, rc_min, rc_sum, bufs[1][:n_lo].tolist(), bufs[3][:n_hi].tolist(),
               v[0], list(s), t.failures))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_transport_moves_messages_between_neighbours(world):
    """Ranks in a line exchange their lo/hi messages with their neighbours
    (chunk ids rank+1) in one phase; min and sum are all-reduces."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=transport_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=180) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    for rank, rc, rc_min, rc_sum, r_lo, r_hi, vmin, s, failures in got:
        assert (rc, rc_min, rc_sum) == (0, 0, 0), failures
        chunk = rank + 1
        # from the lower neighbour: its hi message; from the upper: its lo message
        assert r_lo == [100.0 * (chunk - 1) + 2] * len(r_lo)
        assert r_hi == [100.0 * (chunk + 1) + 1] * len(r_hi)
        assert len(r_lo) == (5 + rank - 1 if rank > 0 else 0)
        assert len(r_hi) == (5 + rank if rank < world - 1 else 0)
        assert vmin == 10.0 - (world - 1)
        assert s == [float(sum(r + i for r in range(world))) for i in range(5)]
