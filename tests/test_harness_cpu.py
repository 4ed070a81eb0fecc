"""The Python restatement of the drivers (hydro_harness) over the oracle
kernels reproduces the oracle's own C driver bit for bit. The GPU parity
tests drive the ABI through the same harness."""
import numpy as np

import decks
import hydro_harness as H
import oracle_lib as O


def run_harness(d, steps):
    nx, ny, nz = d["x_cells"], d["y_cells"], d["z_cells"]
    a = H.new_chunk(nx, ny, nz)
    h = H.Hydro(H.Backend(O.load(), "oracle_"), a, nx, ny, nz, d)
    h.start()
    dts = []
    for _ in range(steps):
        h.step()
        dts.append(h.dt)
    h.field_summary()  # the oracle driver ends with one (hydro.f90:87)
    return a, np.array(dts), h


def test_harness_matches_oracle_driver():
    d = decks.shock(11, 7, 6, 6)
    a, dts, _ = run_harness(d, 6)
    r = O.run(d, max_steps=6, want_fields=True)
    assert np.array_equal(dts, r["dt"])
    for n in O.FIELD_NAMES:
        assert np.array_equal(a[n], r["fields"][n]), n


def test_harness_mixed_states_match_oracle_driver():
    d = decks.shock(9, 8, 10, 4, states=decks.MIXED_STATES)
    a, dts, _ = run_harness(d, 4)
    r = O.run(d, max_steps=4, want_fields=True)
    assert np.array_equal(dts, r["dt"])
    for n in O.FIELD_NAMES:
        assert np.array_equal(a[n], r["fields"][n]), n
