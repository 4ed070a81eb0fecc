"""test_problem_1 with its flow along y and along z on the GPU.

The oracle's y and z forms are pinned on the CPU (tests/test_oracle.py: the
rotated runs meet the reference's known-answer criterion, and with the
reference's two direction-dependent halo extents made symmetric all three
rotations agree to 1e-14). Here the native chunk (fused and unfused step,
graph replay) and the drop-in driver run the same rotated decks and must
match the oracle bit for bit: dt and every array of the 19 fields, the
summaries to 1e-12.
"""
import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks
import oracle_lib as O

pytestmark = pytest.mark.gpu

SUMMARY_RTOL = 1e-12


@pytest.fixture(autouse=True)
def fresh_abi():
    L = C.lib()
    L.clover_gpu_release()
    L.clover_gpu_clear_status()
    yield
    L.clover_gpu_release()
    L.clover_gpu_clear_status()


def _deck(case, axis):
    tp1 = decks.test_problem_1()
    if case == "tp1":
        return decks.rotated(tp1, axis)
    # the same problem on a finer cross-section (40 x 8 x 8 cells, 60 steps)
    big = dict(tp1, x_cells=40, y_cells=8, z_cells=8, end_step=60)
    return decks.rotated(big, axis)


def _compare(r, dts, sums, sum_steps, field):
    assert np.array_equal(dts, r["dt"]), "dt sequence differs"
    assert np.array_equal(sum_steps, r["summary_steps"])
    np.testing.assert_allclose(sums, r["summaries"], rtol=SUMMARY_RTOL, atol=0)
    for n in O.FIELD_NAMES:
        f = field(n)
        if not np.array_equal(f, r["fields"][n]):
            bad = np.argwhere(f != r["fields"][n])
            raise AssertionError("%s differs at %d elements, first %s" % (n, len(bad), bad[0]))


@pytest.mark.parametrize("form", ["staged", "register", "unfused"])
@pytest.mark.parametrize("axis", [1, 2])
@pytest.mark.parametrize("case", ["tp1", "tp1_40x8x8"])
def test_native_rotated_bitwise(case, axis, form):
    """The fused step with its stencils staged by bulk-tensor copies or in
    their register-marching forms, and the unfused step."""
    d = _deck(case, axis)
    r = O.run(d, want_fields=True)
    ch = C.Chunk(decks.to_deck(d))
    ch.use_fused(form != "unfused")
    if form != "unfused":
        assert ch.use_tma(form == "staged") == (form == "staged")
    try:
        assert ch.run() == r["steps"]
        assert ch.status == 0
        sums, sst = ch.summaries()
        _compare(r, ch.dt_history(), sums, sst, ch.field)
    finally:
        ch.close()


@pytest.mark.parametrize("axis", [1, 2])
@pytest.mark.parametrize("case", ["tp1", "tp1_40x8x8"])
def test_dropin_rotated_bitwise(case, axis):
    d = _deck(case, axis)
    r = O.run(d, max_steps=d["end_step"], want_fields=True)
    di = C.DropIn(decks.to_deck(d))
    try:
        assert di.run(d["end_step"]) == r["steps"]
        sums, sst = di.summaries()
        _compare(r, di.dt_history(), sums, sst, di.field)
        if case == "tp1":
            ke = sums[-1][3]
            assert abs(100.0 * (ke / 3.64560737191257) - 100.0) < 0.001
    finally:
        di.close()
