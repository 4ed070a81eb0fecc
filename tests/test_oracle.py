"""CPU tests of the oracle: pinned against the reference's known answer and
checked for the invariants of the scheme (no GPU needed)."""
import json
import os

import numpy as np

import oracle_lib as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_known_answer_test_problem_1():
    """field_summary.f90:119-136: final KE within 0.001% of 3.64560737191257.
    The restatement reproduces it to ~1e-15 relative."""
    g = json.load(open(os.path.join(GOLDEN, "test_problem_1.json")))
    r = O.run(g["deck"])
    assert r["steps"] == 75
    ke = r["summaries"][-1][3]
    qa_diff = abs(100.0 * (ke / g["final_kinetic_energy"]) - 100.0)
    assert qa_diff < g["tolerance_percent"]
    assert abs(ke / g["final_kinetic_energy"] - 1.0) < 1e-13


def test_mass_and_volume_conserved_reflective_box():
    g = json.load(open(os.path.join(GOLDEN, "test_problem_1.json")))
    d = dict(g["deck"], x_cells=12, y_cells=7, z_cells=5, end_step=30, summary_frequency=5)
    r = O.run(d)
    s = r["summaries"]
    vol, mass = s[:, 0], s[:, 1]
    assert np.allclose(vol, vol[0], rtol=1e-14, atol=0)
    assert np.allclose(mass, mass[0], rtol=1e-12, atol=0)


def test_threads_do_not_change_results():
    """Every oracle loop writes disjoint elements, and the summary reduces
    plane partials in a fixed order, so results are independent of threads."""
    g = json.load(open(os.path.join(GOLDEN, "test_problem_1.json")))
    d = dict(g["deck"], x_cells=9, y_cells=6, z_cells=5, end_step=12)
    a = O.run(d, want_fields=True)
    b = O.run(d, want_fields=True, fast=True)
    assert np.array_equal(a["dt"], b["dt"])
    assert np.array_equal(a["summaries"], b["summaries"])
    for n in O.FIELD_NAMES:
        assert np.array_equal(a["fields"][n], b["fields"][n]), n


def test_reference_index_ranges_in_bounds_on_edge_grids():
    """ASan/UBSan build of the oracle on 1-cell-thick, 2-cell and odd grids
    with every state geometry: no out-of-bounds access in any kernel."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", O.ORACLE_DIR, "asan"],
                          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    r = subprocess.run([os.path.join(O.ORACLE_DIR, "_build", "oracle_asan")],
                       capture_output=True, text=True, env=dict(os.environ, ASAN_OPTIONS="detect_leaks=0"))
    assert r.returncode == 0, r.stderr[-2000:]
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr
    assert r.stdout.count("steps 6") == 9
