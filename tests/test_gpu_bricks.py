"""GPU: the brick decomposition of one deck and the halo messages it moves.

1. The twelve pack_kernel.f90 entry points (clover_pack_message_* /
   clover_unpack_message_*) against the oracle's restatement, every side,
   field type and depth, with buffer and tile offsets: buffers and fields
   equal bit for bit.
2. Decomposed runs (Bricks: clover_decompose's bricks in one process, halo
   messages exchanged on the device before each update_halo's reflective
   faces, dt the minimum over the bricks, summaries their sum) against the
   decomposed run of the oracle (tests/brick_harness.py): the dt sequence and
   every field bit for bit, each brick's arrays halos included, the summaries
   to 1e-12 (a different summation order inside each brick). The decomposed
   reference is not the single-chunk one bit for bit: update_halo_kernel.f90
   reflects some fields over extents one short of a brick's exchanged halo
   (x-face data on z faces to n+d), so such corners keep the neighbour's value
   of the previous update; tests/test_bricks_cpu.py shows the size of that.
"""
import ctypes

import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks
import oracle_lib as O
from brick_harness import BrickOracle

pytestmark = pytest.mark.gpu

SIDES = ["left", "right", "bottom", "top", "back", "front"]
FIELD_EXTRA = {1: (0, 0, 0), 2: (1, 1, 1), 3: (1, 0, 0), 4: (0, 1, 0), 5: (0, 0, 1)}


@pytest.fixture(autouse=True)
def fresh_abi():
    L = C.lib()
    L.clover_gpu_release()
    L.clover_gpu_clear_status()
    yield
    L.clover_gpu_release()
    L.clover_gpu_clear_status()


def iref(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def msg_args(bounds, field, buf, depth, ftype, boff, oa, ob, g, kinds=True):
    """The argument list of pack_kernel.f90's routines (the oracle's omits the
    five *_DATA constants)."""
    k = [iref(v) for v in (1, 2, 3, 4, 5)] if kinds else []
    return ([iref(v) for v in bounds] + [field.ctypes.data_as(ctypes.c_void_p),
                                          buf.ctypes.data_as(ctypes.c_void_p)] + k +
            [iref(depth), iref(ftype), iref(boff), iref(oa), iref(ob)] + [iref(v) for v in g])


@pytest.mark.parametrize("side", range(6))
@pytest.mark.parametrize("ftype", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("depth", [1, 2])
def test_messages_match_oracle(side, ftype, depth):
    L = C.lib()
    lo = O.load()
    lo.oracle_pack_message.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 16
    nx, ny, nz = 6, 5, 4
    bounds = (1, nx, 1, ny, 1, nz)
    ex = FIELD_EXTRA[ftype]
    shape = (nx + 4 + ex[0], ny + 4 + ex[1], nz + 4 + ex[2])
    rng = np.random.default_rng(100 * side + 10 * ftype + depth)
    field = np.asfortranarray(rng.standard_normal(shape))
    # a tile offset of 1 in both offset axes and a chunk one cell larger than the
    # tile in each (g_*_max), and a message that starts at buffer index 7
    boff, oa, ob, g = 6, 1, 1, (nx + 1, ny + 1, nz + 1)
    buf_ref = np.full(20000, -7.0)
    buf = buf_ref.copy()
    lo.oracle_pack_message(side, 1, *msg_args(bounds, field, buf_ref, depth, ftype, boff, oa, ob,
                                              g, kinds=False))
    getattr(L, "clover_pack_message_" + SIDES[side])(*msg_args(bounds, field, buf, depth, ftype,
                                                               boff, oa, ob, g))
    assert L.clover_gpu_status() == 0, L.clover_gpu_error_string()
    assert np.array_equal(buf, buf_ref)
    assert np.count_nonzero(buf != -7.0) > 0
    # unpack a random message into a fresh field
    msg = rng.standard_normal(20000)
    f_ref = np.asfortranarray(rng.standard_normal(shape))
    f_dev = f_ref.copy(order="F")
    lo.oracle_pack_message(side, 0, *msg_args(bounds, f_ref, msg, depth, ftype, boff, oa, ob, g,
                                              kinds=False))
    getattr(L, "clover_unpack_message_" + SIDES[side])(*msg_args(bounds, f_dev, msg, depth, ftype,
                                                                 boff, oa, ob, g))
    L.clover_gpu_sync_to_host()
    assert L.clover_gpu_status() == 0, L.clover_gpu_error_string()
    assert np.array_equal(f_dev, f_ref)


DECKS = {
    "shock": lambda: decks.shock(14, 11, 9, 24, states=decks.MIXED_STATES),
    "tp1": lambda: dict(decks.test_problem_1(), x_cells=24, y_cells=6, z_cells=6, end_step=30),
}
ALL_FIELDS = ("density0", "energy0", "pressure", "viscosity", "soundspeed", "density1",
              "energy1", "xvel0", "yvel0", "zvel0", "xvel1", "yvel1", "zvel1", "vol_flux_x",
              "vol_flux_y", "vol_flux_z", "mass_flux_x", "mass_flux_y", "mass_flux_z")


@pytest.mark.parametrize("name", sorted(DECKS))
@pytest.mark.parametrize("n", [2, 3, 4, 6, 8])
def test_bricks_match_decomposed_oracle(name, n):
    d = DECKS[name]()
    ref = BrickOracle(d, n)
    ref_steps = ref.run()
    w = C.Bricks(decks.to_deck(d), n)
    assert w.n == n
    assert [tuple(int(v) for v in e) for e in ref.ext] == w.extents
    steps = w.run()
    assert steps == ref_steps
    assert np.array_equal(w.dt_history(), np.array(ref.dts))
    s, st = w.summaries()
    assert np.array_equal(st, np.array(ref.sum_steps))
    np.testing.assert_allclose(s, np.array(ref.sums), rtol=1e-12, atol=1e-300)
    nx, ny, nz = d["x_cells"], d["y_cells"], d["z_cells"]
    for f in ALL_FIELDS:
        g = w.field(f)
        r = ref.field(f)
        sl = tuple(slice(2, 2 + m + (r.shape[a] - (m + 4))) for a, m in enumerate((nx, ny, nz)))
        assert np.array_equal(g[sl], r[sl]), (f, np.argwhere(g[sl] != r[sl])[:5])
    # every brick's own arrays, halos included, as the decomposed oracle has them
    for i in range(n):
        for f in ("density1", "energy1", "xvel1", "mass_flux_z", "vol_flux_x"):
            assert np.array_equal(w.brick_field(i, f), ref.h[i].a[f]), (i, f)
    w.close()


def test_one_brick_is_the_single_chunk():
    d = DECKS["shock"]()
    ref = O.run(d, want_fields=True)
    w = C.Bricks(decks.to_deck(d), 1)
    assert w.run() == ref["steps"]
    assert np.array_equal(w.dt_history(), ref["dt"])
    for f in ALL_FIELDS:
        assert np.array_equal(w.brick_field(0, f), ref["fields"][f]), f
    w.close()
