"""Compensated field_summary sums on the GPU (field_summary_kernel.f90:57-77).

Every summary path -- one chunk (FP64 and mixed storage), an ensemble's
per-deck sums, and the drop-in entry point on caller arrays -- carries a
Neumaier compensation term through its thread loop, block tree and second
stage, so each quantity comes back within one ulp of the exactly rounded sum
of the per-cell terms (math.fsum over tests/summary_exact.py's terms, pinned
to the oracle bit for bit on the CPU). The same grids' plain running sums (the
oracle's order) are several ulps away, which the tests check too, so that
the one-ulp bound is not met by accident.
"""
import ctypes

import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks
import summary_exact as X

pytestmark = pytest.mark.gpu

MAX_ULPS = 1.0
SUMMED = ("density0", "energy0", "pressure", "xvel0", "yvel0", "zvel0")


def _check(got, terms):
    exact = X.exact_sums(terms)
    assert X.ulps(got, exact).max() <= MAX_ULPS, (got, exact, X.ulps(got, exact))
    return X.ulps(X.oracle_order_sums(terms), exact).max()


@pytest.mark.parametrize("precision", [C.PRECISION_FP64, C.PRECISION_MIXED])
def test_chunk_summary_within_one_ulp_of_exact(precision):
    d = decks.shock(72, 64, 56, 20)
    ch = C.Chunk(decks.to_deck(d), precision=precision)
    try:
        assert ch.run() == 20
        sums, _ = ch.summaries()
        f = {n: ch.field(n) for n in SUMMED}
    finally:
        ch.close()
    terms = X.cell_terms(72, 64, 56, X.cell_volume(d), *[f[n] for n in SUMMED])
    assert _check(sums[-1], terms) >= 4


def test_ensemble_deck_summaries_within_one_ulp_of_exact():
    ds = [decks.shock(40, 33, 29, 20), decks.shock(24, 50, 31, 20), decks.shock(61, 20, 22, 20)]
    en = C.Ensemble([decks.to_deck(d) for d in ds])
    try:
        assert en.run() == 20
        worst_plain = 0.0
        for i, d in enumerate(ds):
            sums, _ = en.deck_summaries(i)
            f = {n: en.deck_field(i, n) for n in SUMMED}
            terms = X.cell_terms(d["x_cells"], d["y_cells"], d["z_cells"], X.cell_volume(d),
                                 *[f[n] for n in SUMMED])
            worst_plain = max(worst_plain, _check(sums[-1], terms))
    finally:
        en.close()
    assert worst_plain >= 2


def test_dropin_summary_of_caller_arrays_within_one_ulp_of_exact():
    """clover_field_summary_kernel on host arrays of a two-state field (the
    benchmark problem's piecewise-constant states, random velocities): long
    runs of equal terms are where plain running sums drift furthest."""
    L = C.lib()
    L.clover_gpu_release()
    L.clover_gpu_clear_status()
    nx, ny, nz = 45, 38, 33
    rng = np.random.default_rng(11)
    cell, vert = (nx + 4, ny + 4, nz + 4), (nx + 5, ny + 5, nz + 5)
    rho = np.full(cell, 0.2, order="F")
    rho[:20, :15, :10] = 1.0
    e = np.full(cell, 1.0, order="F")
    e[:20, :15, :10] = 2.5
    a = {
        "volume": np.full(cell, 0.0123, order="F"), "density0": rho, "energy0": e,
        "pressure": np.asfortranarray(0.4 * rho * e),
        "xvel0": np.asfortranarray(0.3 * rng.uniform(-1, 1, vert)),
        "yvel0": np.asfortranarray(0.3 * rng.uniform(-1, 1, vert)),
        "zvel0": np.asfortranarray(0.3 * rng.uniform(-1, 1, vert)),
    }
    names = ("volume",) + SUMMED
    b = [ctypes.byref(ctypes.c_int(v)) for v in (1, nx, 1, ny, 1, nz)]
    out = [ctypes.c_double(0.0) for _ in range(5)]
    try:
        L.clover_field_summary_kernel(*b, *[ctypes.c_void_p(a[n].ctypes.data) for n in names],
                                      *[ctypes.byref(o) for o in out])
        assert L.clover_gpu_status() == 0, L.clover_gpu_error_string()
    finally:
        L.clover_gpu_release()
    terms = X.cell_terms(nx, ny, nz, a["volume"], *[a[n] for n in SUMMED])
    assert _check([o.value for o in out], terms) >= 4
