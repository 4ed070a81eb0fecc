"""GPU: the benchmark problem at the sizes of its parity configurations,
through the native fused FP64 step, against the oracle.

Config 1: the two-state shock at 32^3 for 100 steps (dt pinned at 0.04).
Config 2: the same at 96^3 for 300 steps, end_time far enough (the default
end_time of 10 would stop it at step 250). Bar: the dt sequence and every
field bit for bit, the field summaries to 1e-12 (a different summation
order; the stated bar is 1e-10).
"""
import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks
import oracle_lib as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,steps", [(32, 100), (96, 300)])
def test_config_matches_oracle(n, steps):
    d = decks.shock(n, n, n, steps, end_time=1000.0)
    ref = O.run(d, want_fields=True)
    assert ref["steps"] == steps
    ch = C.Chunk(decks.to_deck(d), C.PRECISION_FP64)
    assert ch.run() == steps
    assert np.array_equal(ch.dt_history(), ref["dt"])
    s, st = ch.summaries()
    assert np.array_equal(st, ref["summary_steps"])
    np.testing.assert_allclose(s, ref["summaries"], rtol=1e-12, atol=0)
    for f in O.FIELD_NAMES:
        assert np.array_equal(ch.field(f), ref["fields"][f]), f
    ch.close()
