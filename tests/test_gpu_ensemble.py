"""Ensembles: many decks of different sizes advanced by one batched launch per
kernel, each deck with its own dt.

Every deck of an ensemble must give what the same deck gives alone: the
oracle's dt sequence and final arrays bit for bit (summaries to 1e-12, their
sums run in another fixed order), whatever schedule the autotuner picks and
with or without graph replay. The mixed-precision ensemble must equal the
mixed-precision single chunks bit for bit and stay within 1e-5 of FP64.
"""
import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks
import oracle_lib as O

pytestmark = pytest.mark.gpu

SUMMARY_RTOL = 1e-12
STEPS = 12


def compare(r, dts, sums, sum_steps, field):
    assert np.array_equal(dts, r["dt"]), "dt sequence differs"
    assert np.array_equal(sum_steps, r["summary_steps"])
    np.testing.assert_allclose(sums, r["summaries"], rtol=SUMMARY_RTOL, atol=0)
    for n in O.FIELD_NAMES:
        f = field(n)
        if not np.array_equal(f, r["fields"][n]):
            bad = np.argwhere(f != r["fields"][n])
            raise AssertionError("%s differs at %d elements, first %s" % (n, len(bad), bad[0]))


def oracle_decks():
    """Uneven sizes, a one-cell-thick deck, every geometry kind, moving states
    and different timestep controls."""
    kw = dict(end_step=STEPS, summary_frequency=5)
    return [
        decks.shock(13, 9, 11, STEPS, states=decks.MIXED_STATES, **kw),
        decks.shock(16, 16, 16, STEPS, **kw),
        decks.shock(7, 1, 5, STEPS, states=decks.MIXED_STATES, **kw),
        decks.shock(33, 6, 9, STEPS, initial_timestep=0.01, timestep_rise=1.2, **kw),
        decks.shock(5, 21, 14, STEPS, states=decks.MIXED_STATES, max_timestep=0.02, **kw),
    ]


@pytest.mark.parametrize("graphs", [True, False])
def test_ensemble_decks_match_oracle(graphs):
    ds = oracle_decks()
    ens = C.Ensemble([decks.to_deck(d) for d in ds])
    ens.use_graphs(graphs)
    assert ens.run() == STEPS
    for i, d in enumerate(ds):
        assert ens.deck_status(i) == 0
        r = O.run(d, want_fields=True)
        assert r["steps"] == STEPS
        sums, sst = ens.deck_summaries(i)
        compare(r, ens.deck_dt_history(i), sums, sst, lambda n, i=i: ens.deck_field(i, n))
    # decks with different controls take different dt sequences
    assert not np.array_equal(ens.deck_dt_history(1), ens.deck_dt_history(3))
    ens.close()


def test_decks_of_three_cells_or_more_match_oracle():
    """Without a thin deck the batched step leaves out the halo updates that
    repeat a no-op and the shell copies a depth-2 update overwrites; every
    field, halos included, still equals the oracle's."""
    kw = dict(end_step=STEPS, summary_frequency=5)
    ds = [decks.shock(13, 9, 11, STEPS, states=decks.MIXED_STATES, **kw),
          decks.shock(16, 16, 16, STEPS, **kw),
          decks.shock(33, 6, 9, STEPS, initial_timestep=0.01, timestep_rise=1.2, **kw)]
    ens = C.Ensemble([decks.to_deck(d) for d in ds])
    assert ens.run() == STEPS
    for i, d in enumerate(ds):
        r = O.run(d, want_fields=True)
        sums, sst = ens.deck_summaries(i)
        compare(r, ens.deck_dt_history(i), sums, sst, lambda n, i=i: ens.deck_field(i, n))
    ens.close()


def test_one_deck_ensemble_matches_chunk():
    d = decks.to_deck(decks.shock(19, 11, 8, 9, states=decks.MIXED_STATES))
    ens = C.Ensemble([d])
    ch = C.Chunk(d)
    ens.step(9)
    ch.step(9)
    assert np.array_equal(ens.deck_dt_history(0), ch.dt_history())
    for n in O.FIELD_NAMES:
        assert np.array_equal(ens.deck_field(0, n), ch.field(n)), n
    ens.close()
    ch.close()


def test_autotuned_schedule_is_bitwise_neutral():
    ds = C.draw_decks(10, seed=5, cells=(4, 40), end_step=16, summary_frequency=8)
    plain = C.Ensemble(ds)
    plain.use_graphs(False)
    plain.step(16)
    tuned = C.Ensemble(ds)
    assert tuned.autotune(1) > 10
    assert tuned.steps == 0 and tuned.deck_time(0) == 0.0
    sched = tuned.schedule()
    assert sched and all(s["items"] > 0 and s["blocks"] > 0 for s in sched)
    assert any(s["seg"] > 0 for s in sched)
    tuned.step(16)
    tuned.sync()
    for i in range(len(ds)):
        assert np.array_equal(tuned.deck_dt_history(i), plain.deck_dt_history(i))
        for n in ("density0", "energy0", "xvel0", "zvel1", "mass_flux_y", "vol_flux_z"):
            assert np.array_equal(tuned.deck_field(i, n), plain.deck_field(i, n)), (i, n)
        a, _ = tuned.deck_summaries(i)
        b, _ = plain.deck_summaries(i)
        assert np.array_equal(a, b)
    plain.close()
    tuned.close()


def test_mixed_ensemble_matches_mixed_chunks_and_fp64():
    ds = C.draw_decks(6, seed=9, cells=(6, 30), end_step=20, summary_frequency=10)
    mixed = C.Ensemble(ds, C.PRECISION_MIXED)
    fp64 = C.Ensemble(ds, C.PRECISION_FP64)
    mixed.run()
    fp64.run()
    for i, d in enumerate(ds):
        ch = C.Chunk(d, C.PRECISION_MIXED)
        ch.run()
        assert np.array_equal(mixed.deck_dt_history(i), ch.dt_history())
        for n in ("density0", "energy0", "pressure", "xvel0", "yvel0", "zvel0"):
            assert np.array_equal(mixed.deck_field(i, n), ch.field(n)), (i, n)
        sm, _ = mixed.deck_summaries(i)
        sf, _ = fp64.deck_summaries(i)
        scale = np.maximum(np.abs(sf), np.abs(sf).max(axis=0) * 1e-3)
        err = np.abs(sm - sf) / scale
        assert err.max() <= 1e-5, err.max(axis=0)
        # mass is carried in FP64 (density, mass and volume fluxes), far below
        # the FP32 rounding of the stored fields; FP64 itself drifts ~1e-4 on
        # these 3D decks (the reference's z volume flux in flux_calc is not
        # the PdV one), and the mixed run follows that drift to ~1e-11
        assert np.max(np.abs(sm[:, 1] - sf[:, 1]) / sf[:, 1]) <= 1e-9
        ch.close()
    mixed.close()
    fp64.close()


@pytest.mark.parametrize("sched", [(0, 0, 0), (0, 1, 0), (2, 2, 16), (1, 4, 8)])
def test_large_decks_every_schedule_bitwise(sched):
    """Decks large enough that every block of a persistent grid walks many
    items (and item lists take a while to upload), under one block per item,
    full and partial persistent grids, every item order and several segment
    lengths: each deck equals the same deck run alone."""
    ds = C.draw_decks(4, seed=31, cells=(56, 96), end_step=4, summary_frequency=2)
    ens = C.Ensemble(ds)
    ens.set_schedule(*sched)
    ens.step(4)
    ens.sync()
    for i, d in enumerate(ds):
        ch = C.Chunk(d)
        ch.step(4)
        assert np.array_equal(ens.deck_dt_history(i), ch.dt_history())
        for n in O.FIELD_NAMES:
            assert np.array_equal(ens.deck_field(i, n), ch.field(n)), (i, n)
        a, _ = ens.deck_summaries(i)
        b, _ = ch.summaries()
        np.testing.assert_allclose(a, b, rtol=SUMMARY_RTOL, atol=0)
        ch.close()
    ens.close()


def test_deck_status_is_per_deck():
    """A deck whose dtmin lies above its dt is flagged; the others are not."""
    ds = C.draw_decks(3, seed=2, cells=(6, 12), end_step=4, summary_frequency=2)
    ds[1] = ds[1].replace(dtmin=1.0)
    ens = C.Ensemble(ds)
    ens.step(4)
    ens.sync()
    assert ens.deck_status(1) & 0x4
    assert ens.deck_status(0) == 0 and ens.deck_status(2) == 0
    ens.close()


def test_ensemble_rejects_inconsistent_decks():
    ds = C.draw_decks(2, seed=3, cells=(4, 8), end_step=4)
    ds[1] = ds[1].replace(end_step=5)
    with pytest.raises(C.CloverError):
        C.Ensemble(ds)
