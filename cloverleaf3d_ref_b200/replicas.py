"""Replicas over GPUs, one process per GPU.

A deck is one chunk on one GPU (the single-chunk step does not shard), and the
decks of an ensemble are independent: N ranks take disjoint shares of the
decks and exchange nothing but their timings. These helpers are the host side
of that: which decks a rank takes, and the job's time as its slowest rank's.
"""


def deck_share(cells, rank, world):
    """Indices of the decks rank takes out of decks with the given cell counts.

    Decks go largest first, each to the rank with the fewest cells so far (the
    lower rank on a tie), which every rank computes alike; the returned indices
    are in deck order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of %d" % (rank, world))
    order = sorted(range(len(cells)), key=lambda i: (-cells[i], i))
    load = [0] * world
    owner = [0] * len(cells)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += cells[i]
    return [i for i in range(len(cells)) if owner[i] == rank]


def max_over_ranks(value, dist=None, device="cpu"):
    """The largest value over the ranks of the default process group (the
    value itself without one). device: where the reduction runs ("cuda" for
    NCCL, "cpu" for gloo)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    if dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
