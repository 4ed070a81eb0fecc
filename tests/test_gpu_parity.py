"""GPU parity: the CUDA kernels against the oracle, through the drop-in C ABI.

FP64 kernels are built without multiply-add contraction and keep the
reference's operation order, so every array must match the oracle BIT FOR
BIT after every kernel call; only the field_summary sums (a different
reduction order) are compared with a tolerance (1e-12 relative).
"""
import ctypes

import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks
import hydro_harness as H
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


def oracle_trace(d, steps):
    """Run the oracle kernel by kernel, snapshotting every array after each call."""
    nx, ny, nz = d["x_cells"], d["y_cells"], d["z_cells"]
    a = H.new_chunk(nx, ny, nz)
    snaps = []
    b = H.Backend(O.load(), "oracle_", after=lambda name: snaps.append((name, H.clone(a))))
    h = H.Hydro(b, a, nx, ny, nz, d)
    h.start()
    scal = []
    for _ in range(steps):
        h.step()
        scal.append(h.calc_dt_out)
    scal.append(tuple(h.field_summary()))
    return snaps, scal


def gpu_lockstep(d, steps, snaps):
    """Run the same calls through the ABI and compare after each one."""
    L = C.lib()
    nx, ny, nz = d["x_cells"], d["y_cells"], d["z_cells"]
    a = H.new_chunk(nx, ny, nz)
    idx = [0]
    mism = []

    def after(name):
        L.clover_gpu_sync_to_host()
        assert L.clover_gpu_status() in (0, 4), L.clover_gpu_error_string()
        ref_name, ref = snaps[idx[0]]
        assert ref_name == name
        for k in ref:
            if not np.array_equal(a[k], ref[k]):
                bad = np.argwhere(a[k] != ref[k])
                mism.append((idx[0], name, k, len(bad), tuple(bad[0])))
        idx[0] += 1
        if mism:
            raise AssertionError("first mismatch (call, kernel, array, count, index): %s" % (mism[0],))

    h = H.Hydro(H.Backend(L, "clover_", after=after), a, nx, ny, nz, d)
    h.start()
    scal = []
    for _ in range(steps):
        h.step()
        scal.append(h.calc_dt_out)
    scal.append(tuple(h.field_summary()))
    return scal


@pytest.mark.parametrize("staging", [True, False])
@pytest.mark.parametrize("case", ["shock_11x7x6", "mixed_9x8x10", "thin_5x1x3", "tp1_10x2x2"])
def test_kernel_by_kernel_bitwise(case, staging):
    """Every array after every call, with the staged drop-in forms (planes
    copied into shared memory by bulk-tensor copies) allowed and forbidden."""
    C.lib().clover_gpu_use_staging(1 if staging else 0)
    try:
        _kernel_by_kernel(case)
    finally:
        C.lib().clover_gpu_use_staging(1)


def _kernel_by_kernel(case):
    d = {
        "shock_11x7x6": decks.shock(11, 7, 6, 3),
        "mixed_9x8x10": decks.shock(9, 8, 10, 2, states=decks.MIXED_STATES),
        "thin_5x1x3": decks.shock(5, 1, 3, 2, states=decks.MIXED_STATES),
        "tp1_10x2x2": decks.test_problem_1(),
    }[case]
    steps = 3 if case != "tp1_10x2x2" else 2
    snaps, ref_scal = oracle_trace(d, steps)
    got = gpu_lockstep(d, steps, snaps)
    for r, g in zip(ref_scal[:-1], got[:-1]):
        assert r == g  # calc_dt outputs, dt_min_val bitwise
    np.testing.assert_allclose(got[-1], ref_scal[-1], rtol=SUMMARY_RTOL, atol=0)


def run_both(d, steps):
    r = O.run(d, max_steps=steps, want_fields=True)
    return r


def compare_run(r, dts, sums, sum_steps, fields):
    assert np.array_equal(dts, r["dt"]), "dt sequence differs"
    assert np.array_equal(sum_steps, r["summary_steps"])
    np.testing.assert_allclose(sums, r["summaries"], rtol=SUMMARY_RTOL, atol=0)
    for n in O.FIELD_NAMES:
        f = fields(n)
        if not np.array_equal(f, r["fields"][n]):
            bad = np.argwhere(f != r["fields"][n])
            raise AssertionError("%s differs at %d elements, first %s" % (n, len(bad), bad[0]))


@pytest.mark.parametrize("case", ["tp1", "shock16", "mixed"])
def test_dropin_driver_run_bitwise(case):
    d = {"tp1": decks.test_problem_1(), "shock16": decks.shock(16, 16, 16, 30),
         "mixed": decks.shock(13, 9, 11, 20, states=decks.MIXED_STATES)}[case]
    steps = d["end_step"]
    r = O.run(d, max_steps=steps, want_fields=True)
    di = C.DropIn(decks.to_deck(d))
    n = di.run(steps)
    assert n == r["steps"]
    sums, sst = di.summaries()
    compare_run(r, di.dt_history(), sums, sst, di.field)
    if case == "tp1":
        ke = sums[-1][3]
        assert abs(100.0 * (ke / 3.64560737191257) - 100.0) < 0.001
    di.close()


def test_dropin_state_restored_from_host_arrays():
    """Copying the state back, marking every mirror stale and carrying on
    (each array uploaded again from its host copy at its next use) gives the
    uninterrupted run bit for bit."""
    d = decks.shock(13, 9, 11, 20, states=decks.MIXED_STATES)
    r = O.run(d, max_steps=20, want_fields=True)
    L = C.lib()
    di = C.DropIn(decks.to_deck(d))
    assert di.run(7) == 7  # the driver's step count is cumulative
    L.clover_gpu_sync_to_host()
    L.clover_gpu_invalidate_all()
    assert di.run(20) == r["steps"]
    sums, sst = di.summaries()
    keep = np.isin(sst, r["summary_steps"])  # drop the summary the first call ended with
    compare_run(r, di.dt_history(), sums[keep], sst[keep], di.field)
    di.close()


@pytest.mark.parametrize("case", ["tp1", "shock16", "mixed", "thin", "uneven"])
def test_native_staged_and_register_forms_bitwise(case):
    """The fused step with its stencils staged in shared memory by bulk-tensor
    copies and with their register-marching forms: both equal the oracle bit
    for bit (tiles that run past the grid on every axis, one-cell and
    two-cell axes, segments of the march split mid-grid)."""
    d = {"tp1": decks.test_problem_1(), "shock16": decks.shock(16, 16, 16, 30),
         "mixed": decks.shock(13, 9, 11, 20, states=decks.MIXED_STATES),
         "thin": decks.shock(7, 1, 5, 9, states=decks.MIXED_STATES),
         "uneven": decks.shock(70, 17, 45, 12, states=decks.MIXED_STATES)}[case]
    r = O.run(d, want_fields=True)
    for tma in (True, False):
        ch = C.Chunk(decks.to_deck(d))
        assert ch.use_tma(tma) == tma
        n = ch.run()
        assert n == r["steps"]
        assert ch.status == 0
        sums, sst = ch.summaries()
        compare_run(r, ch.dt_history(), sums, sst, ch.field)
        ch.close()


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("case", ["tp1", "shock16", "mixed", "thin"])
def test_native_chunk_run_bitwise(case, graphs, fused):
    """The native step (fused kernels or one kernel per reference pass, graph
    replay or direct launches) against the oracle: dt and every array of the
    19 fields bit for bit, summaries to 1e-12."""
    d = {"tp1": decks.test_problem_1(), "shock16": decks.shock(16, 16, 16, 30),
         "mixed": decks.shock(13, 9, 11, 20, states=decks.MIXED_STATES),
         "thin": decks.shock(7, 1, 5, 9, states=decks.MIXED_STATES)}[case]
    r = O.run(d, want_fields=True)
    ch = C.Chunk(decks.to_deck(d))
    ch.use_fused(fused)
    ch.use_graphs(graphs)
    n = ch.run()
    assert n == r["steps"]
    assert ch.status == 0
    sums, sst = ch.summaries()
    compare_run(r, ch.dt_history(), sums, sst, ch.field)
    ch.close()


def test_native_end_time_stop():
    """hydro.f90:84: the run stops at the first step with time+g_small > end_time."""
    d = decks.shock(12, 10, 8, 1000, end_time=1.0)
    r = O.run(d, want_fields=True)
    ch = C.Chunk(decks.to_deck(d))
    n = ch.run()
    assert n == r["steps"]
    sums, sst = ch.summaries()
    compare_run(r, ch.dt_history(), sums, sst, ch.field)
    ch.close()


def test_native_known_answer():
    ch = C.Chunk(decks.to_deck(decks.test_problem_1()))
    assert ch.run() == 75
    sums, _ = ch.summaries()
    ke = sums[-1][3]
    assert abs(ke / 3.64560737191257 - 1.0) < 1e-13
    ch.close()


def test_native_fused_long_run_bitwise():
    """A longer fused run on an uneven grid (several segments of the marching
    kernels along every axis) stays bit-identical."""
    d = decks.shock(40, 37, 70, 40, states=decks.MIXED_STATES)
    r = O.run(d, want_fields=True)
    ch = C.Chunk(decks.to_deck(d))
    n = ch.run()
    assert n == r["steps"]
    sums, sst = ch.summaries()
    compare_run(r, ch.dt_history(), sums, sst, ch.field)
    ch.close()


def test_mom_volumes_formed_again_after_host_change_or_other_call():
    """advec_mom reuses the pre/post volumes of the previous velocity call of
    a sweep only while nothing else happened: after the host changes an input
    (clover_gpu_invalidate) or another library call (here flux_calc, which
    rewrites the volume fluxes), they are formed again, as the reference
    forms them in every call."""
    d = decks.shock(9, 8, 10, 2, states=decks.MIXED_STATES)
    nx, ny, nz = d["x_cells"], d["y_cells"], d["z_cells"]
    L = C.lib()
    a_ref, a_gpu = H.new_chunk(nx, ny, nz), H.new_chunk(nx, ny, nz)
    hs = [H.Hydro(H.Backend(O.load(), "oracle_"), a_ref, nx, ny, nz, d),
          H.Hydro(H.Backend(L, "clover_"), a_gpu, nx, ny, nz, d)]

    def check(names):
        L.clover_gpu_sync_to_host()
        assert L.clover_gpu_status() in (0, 4), L.clover_gpu_error_string()
        for k in names:
            assert np.array_equal(a_gpu[k], a_ref[k]), k

    for h in hs:
        h.start()
        h.timestep()
        h.pdv(True)
        h.accelerate()
        h.pdv(False)
        h.flux_calc()
        h.halo([4, 2, 14, 15, 16], 2)
        h.advec_cell(1, 1)
        h.halo([2, 4, 9, 11, 13, 17, 18, 19], 2)
        h.advec_mom(1, 1, 1)
    check(["wa6", "wa7", "xvel1"])
    for a in (a_ref, a_gpu):  # the host changes an input between two velocity calls
        a["vol_flux_y"] *= 1.25
    L.clover_gpu_invalidate(ctypes.c_void_p(a_gpu["vol_flux_y"].ctypes.data))
    for h in hs:
        h.advec_mom(2, 1, 1)
    check(["wa6", "wa7", "yvel1"])
    for h in hs:  # another library call rewrites the volume fluxes
        h.flux_calc()
        h.advec_mom(3, 1, 1)
    check(["vol_flux_x", "vol_flux_y", "vol_flux_z", "wa6", "wa7", "zvel1"])


def test_array_passed_with_another_chunks_bounds_is_refused():
    """An array is the chunk's whose bounds it was first passed with. Passed
    with other bounds, the call sets CLOVER_STATUS_BOUNDS and runs on a zeroed
    stand-in (no access outside any allocation); the array keeps its values."""
    L = C.lib()
    names = ("density0", "energy0", "pressure", "soundspeed")
    a = {n: np.zeros(O.shape("cell", 6, 5, 4), order="F") for n in names}
    a["density0"][:] = 1.0
    a["energy0"][:] = 2.0

    def call(bounds):
        L.clover_ideal_gas_kernel(*[ctypes.byref(ctypes.c_int(v)) for v in bounds],
                                  *[a[n].ctypes.data_as(ctypes.c_void_p) for n in names])
        L.clover_gpu_synchronize()

    call((1, 6, 1, 5, 1, 4))
    assert L.clover_gpu_status() == 0
    call((1, 8, 1, 8, 1, 8))
    assert L.clover_gpu_status() & 0x2
    L.clover_gpu_clear_status()
    L.clover_gpu_sync_to_host()
    assert np.all(a["pressure"][2:8, 2:7, 2:6] == (1.4 - 1.0) * 1.0 * 2.0)


def test_mixed_staged_and_register_forms_identical():
    """The mixed-precision step gives the same bits with its stencils staged
    by bulk-tensor copies or in their register-marching forms."""
    d = decks.shock(70, 17, 45, 12, states=decks.MIXED_STATES)
    out = []
    for tma in (True, False):
        ch = C.Chunk(decks.to_deck(d), precision=C.PRECISION_MIXED)
        assert ch.use_tma(tma) == tma
        assert ch.run() == 12
        assert ch.status == 0
        out.append((ch.dt_history(), ch.summaries()[0], {n: ch.field(n) for n in O.FIELD_NAMES}))
        ch.close()
    (dt_a, s_a, f_a), (dt_b, s_b, f_b) = out
    assert np.array_equal(dt_a, dt_b)
    assert np.array_equal(s_a, s_b)
    for n in O.FIELD_NAMES:
        assert np.array_equal(f_a[n], f_b[n]), n
