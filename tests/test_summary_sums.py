"""CPU pin of the summary-term restatement (tests/summary_exact.py) that the
compensated-sum GPU tests measure against: summed in the oracle's order, the
numpy terms give the oracle's field_summary bit for bit, and the oracle's
plain running sums sit measurably away from the exactly rounded sums on a
grid of a few hundred thousand cells."""
import numpy as np

import decks
import oracle_lib as O
import summary_exact as X


def _final_terms(d):
    r = O.run(d, want_fields=True)
    f = r["fields"]
    nx, ny, nz = d["x_cells"], d["y_cells"], d["z_cells"]
    terms = X.cell_terms(nx, ny, nz, X.cell_volume(d), f["density0"], f["energy0"], f["pressure"],
                         f["xvel0"], f["yvel0"], f["zvel0"])
    return r, terms


def test_terms_in_oracle_order_equal_the_oracle_summary():
    d = decks.shock(14, 11, 9, 12, states=decks.MIXED_STATES)
    r, terms = _final_terms(d)
    assert np.array_equal(X.oracle_order_sums(terms), r["summaries"][-1])


def test_plain_sums_are_off_the_exactly_rounded_sums():
    """The discriminating case of the GPU compensated-sum tests: on 72x64x56
    cells after 20 steps, the oracle's plain running sums of mass, internal and
    kinetic energy and pressure*volume are several ulps away from the exactly
    rounded sums (a compensated sum is within one)."""
    d = decks.shock(72, 64, 56, 20)
    r, terms = _final_terms(d)
    plain = r["summaries"][-1]
    exact = X.exact_sums(terms)
    err = X.ulps(plain, exact)
    assert err[1:].max() >= 4, err
