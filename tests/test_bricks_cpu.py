"""CPU: the decomposition of one deck into bricks (clover.f90:108-256,
clover_decompose) as the library exports it.

The reference picks the chunk grid with the smallest surface-to-volume metric
among the factorisations of the chunk count (strictly smaller wins, starting
from 1 x 1 x n, the metric in default REAL), then gives the first mod(cells,
chunks) chunks of each axis one cell more. Checked here: the grid is the one
an independent restatement of that search picks, the bricks tile the deck
exactly, neighbours are mutual and adjacent, and the chunk ids run x fastest.
"""
import itertools

import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C


def metric32(x, y, z, cx, cy, cz):
    """clover.f90:131-135 / :155-159 in single precision (1.0*x_cells is REAL)."""
    f = np.float32
    ax, ay, az = f(f(1.0) * f(x)) / f(cx), f(f(1.0) * f(y)) / f(cy), f(f(1.0) * f(z)) / f(cz)
    surface = f(f(f(ax * ay) * f(2)) + f(f(ax * az) * f(2))) + f(f(ay * az) * f(2))
    volume = f(f(ax * ay) * az)
    return float(surface) / float(volume)


def expected_grid(x, y, z, n):
    best = (1, 1, n)
    bm = metric32(x, y, z, 1, 1, n)
    for c in range(1, n + 1):
        if n % c:
            continue
        d1 = n // c
        for j in range(1, d1 + 1):
            if d1 % j or n % (c * j):
                continue
            m = metric32(x, y, z, c, j, n // (c * j))
            if m < bm:
                best, bm = (c, j, n // (c * j)), m
    return best


CASES = [(64, 48, 40, n) for n in (1, 2, 3, 4, 5, 6, 8, 12, 16, 27)] + [
    (32, 32, 32, 2), (32, 32, 32, 8), (17, 9, 5, 6), (7, 7, 7, 7), (100, 10, 10, 4),
    (10, 100, 10, 4), (10, 10, 100, 4), (33, 35, 37, 12)]


@pytest.mark.parametrize("x,y,z,n", CASES)
def test_decomposition_tiles_the_deck(x, y, z, n):
    grid, ext, nbr = C.decompose(x, y, z, n)
    assert tuple(grid) == expected_grid(x, y, z, n)
    gx, gy, gz = (int(v) for v in grid)
    assert gx * gy * gz == n
    cover = np.zeros((x, y, z), dtype=np.int32)
    for e in ext:
        cover[e[0] - 1:e[1], e[2] - 1:e[3], e[4] - 1:e[5]] += 1
    assert np.all(cover == 1)
    # chunk id (1-based) = cx + (cy-1) gx + (cz-1) gx gy; the first mod(cells, g)
    # chunks of an axis take one cell more
    for (cx, cy, cz) in itertools.product(range(1, gx + 1), range(1, gy + 1), range(1, gz + 1)):
        i = cx - 1 + (cy - 1) * gx + (cz - 1) * gx * gy
        e = ext[i]
        for a, (c, g, cells) in enumerate(((cx, gx, x), (cy, gy, y), (cz, gz, z))):
            size = e[2 * a + 1] - e[2 * a] + 1
            assert size == cells // g + (1 if c <= cells % g else 0)
        want = [i if cx > 1 else -1, i + 2 if cx < gx else -1,
                i + 1 - gx if cy > 1 else -1, i + 1 + gx if cy < gy else -1,
                i + 1 - gx * gy if cz > 1 else -1, i + 1 + gx * gy if cz < gz else -1]
        assert list(nbr[i]) == want
        for f in range(6):  # neighbours are mutual and share the face
            o = nbr[i][f]
            if o < 0:
                continue
            assert nbr[o - 1][f ^ 1] == i + 1
            a = f // 2
            if f % 2:
                assert ext[o - 1][2 * a] == e[2 * a + 1] + 1
            else:
                assert ext[o - 1][2 * a + 1] == e[2 * a] - 1


def test_equal_metrics_keep_the_first_grid():
    """A cube split in two: every split has the same metric, and the strict
    comparison keeps the initial 1 x 1 x 2."""
    grid, _, _ = C.decompose(32, 32, 32, 2)
    assert tuple(grid) == (1, 1, 2)


def test_more_chunks_than_cells_is_refused():
    with pytest.raises(C.CloverError):
        C.decompose(2, 2, 2, 27)


# ---- the decomposed run of the oracle (the checker of the brick driver) ----
import decks  # noqa: E402
import oracle_lib as O  # noqa: E402
from brick_harness import BrickOracle  # noqa: E402


def _owned(d, f, g):
    nx, ny, nz = d["x_cells"], d["y_cells"], d["z_cells"]
    return g[tuple(slice(2, 2 + m + (g.shape[a] - (m + 4))) for a, m in enumerate((nx, ny, nz)))]


def test_brick_oracle_one_brick_is_the_single_chunk():
    d = decks.shock(10, 8, 7, 12, states=decks.MIXED_STATES)
    ref = O.run(d, want_fields=True)
    b = BrickOracle(d, 1)
    assert b.run() == ref["steps"]
    assert np.array_equal(np.array(b.dts), ref["dt"])
    assert np.array_equal(np.array(b.sums), ref["summaries"])
    for f in ("density0", "energy0", "xvel0", "zvel1", "mass_flux_y", "vol_flux_z"):
        assert np.array_equal(b.h[0].a[f], ref["fields"][f]), f


@pytest.mark.parametrize("n", [2, 3])
def test_decomposed_1d_flow_equals_the_single_chunk(n):
    """test_problem 1 moves along x only: the decomposed run equals the
    single-chunk run bit for bit (summaries to rounding)."""
    d = dict(decks.test_problem_1(), x_cells=24, y_cells=6, z_cells=6, end_step=20)
    ref = O.run(d, want_fields=True)
    b = BrickOracle(d, n)
    assert b.run() == ref["steps"]
    assert np.array_equal(np.array(b.dts), ref["dt"])
    np.testing.assert_allclose(np.array(b.sums), ref["summaries"], rtol=1e-13)
    for f in ("density0", "energy0", "xvel0", "mass_flux_x"):
        assert np.array_equal(_owned(d, f, b.field(f)), _owned(d, f, ref["fields"][f])), f


def test_decomposed_3d_flow_differs_from_the_single_chunk_in_the_last_bits():
    """With flow across a brick face the reference's halo extents leave a few
    corner values one update old (update_halo_kernel.f90 reflects x-face data
    on z faces to n+d, one short of the exchanged n+1+d): the decomposed run
    departs from the single-chunk run at rounding level, not beyond."""
    d = decks.shock(14, 11, 9, 24, states=decks.MIXED_STATES)
    ref = O.run(d, want_fields=True)
    b = BrickOracle(d, 2)
    assert b.run() == ref["steps"]
    assert np.array_equal(np.array(b.dts), ref["dt"])
    g, r = _owned(d, "density0", b.field("density0")), _owned(d, "density0", ref["fields"]["density0"])
    rel = np.max(np.abs(g - r) / np.abs(r))
    assert 0 < rel < 1e-11
