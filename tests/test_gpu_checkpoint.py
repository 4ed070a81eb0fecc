"""Checkpoint / restart of resident chunks and ensembles.

A run that stops, writes a checkpoint and is restored into a fresh chunk
must continue bit for bit like the run that never stopped: dt sequence,
summaries and every array, across the sweep-order alternation and the
velocity buffer pairs of the fused step (the checkpoint is taken after an
odd number of steps)."""
import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks
import oracle_lib as O

pytestmark = pytest.mark.gpu


def _same(a, b, fields, deck=None):
    get_a = (lambda n: a.deck_field(deck, n)) if deck is not None else a.field
    get_b = (lambda n: b.deck_field(deck, n)) if deck is not None else b.field
    for n in fields:
        assert np.array_equal(get_a(n), get_b(n)), n


@pytest.mark.parametrize("precision", [C.PRECISION_FP64, C.PRECISION_MIXED])
def test_chunk_restart_is_bitwise(tmp_path, precision):
    d = decks.to_deck(decks.shock(17, 12, 9, 40, states=decks.MIXED_STATES,
                                  summary_frequency=4))
    full = C.Chunk(d, precision)
    full.step(7)
    path = str(tmp_path / "chunk.ckpt")
    full.checkpoint(path)
    full.step(13)
    full.sync()
    resumed = C.Chunk(d, precision)
    resumed.restore(path)
    assert resumed.steps == 7
    resumed.step(13)
    resumed.sync()
    assert resumed.steps == full.steps == 20
    assert np.array_equal(resumed.dt_history(), full.dt_history())
    a, sa = resumed.summaries()
    b, sb = full.summaries()
    assert np.array_equal(sa, sb) and np.array_equal(a, b)
    _same(resumed, full, O.FIELD_NAMES)
    # the field dump and summary log of the resumed chunk
    resumed.dump_fields(str(tmp_path / "fields.npz"))
    z = np.load(str(tmp_path / "fields.npz"))
    assert np.array_equal(z["density0"], full.field("density0"))
    resumed.write_summary_log(str(tmp_path / "summary.txt"))
    rows = open(str(tmp_path / "summary.txt")).read().splitlines()[1:]
    assert [int(r.split()[0]) for r in rows] == list(sb)
    assert float(rows[-1].split()[2]) == b[-1][1]
    full.close()
    resumed.close()


def test_ensemble_restart_is_bitwise(tmp_path):
    ds = C.draw_decks(5, seed=17, cells=(6, 20), end_step=30, summary_frequency=5)
    full = C.Ensemble(ds)
    full.step(5)
    path = str(tmp_path / "ens.ckpt")
    full.checkpoint(path)
    full.step(6)
    full.sync()
    resumed = C.Ensemble(ds)
    resumed.restore(path)
    resumed.step(6)
    resumed.sync()
    for i in range(len(ds)):
        assert np.array_equal(resumed.deck_dt_history(i), full.deck_dt_history(i))
        assert np.array_equal(resumed.deck_summaries(i)[0], full.deck_summaries(i)[0])
        _same(resumed, full, ("density0", "energy1", "xvel1", "zvel0", "mass_flux_z"), deck=i)
    full.close()
    resumed.close()


def test_restore_rejects_other_decks(tmp_path):
    a = C.Chunk(decks.to_deck(decks.shock(8, 8, 8, 10)))
    path = str(tmp_path / "a.ckpt")
    a.checkpoint(path)
    b = C.Chunk(decks.to_deck(decks.shock(9, 8, 8, 10)))
    with pytest.raises(C.CloverError):
        b.restore(path)
    c = C.Chunk(decks.to_deck(decks.shock(8, 8, 8, 10)), C.PRECISION_MIXED)
    with pytest.raises(C.CloverError):
        c.restore(path)
    a.close()
    b.close()
    c.close()
