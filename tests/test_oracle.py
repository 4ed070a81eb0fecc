"""CPU tests of the oracle: pinned against the reference's known answer and
checked for the invariants of the scheme (no GPU needed)."""
import json
import os

import numpy as np

import decks
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


def test_halo_update_repeat_is_a_no_op_for_cell_vertex_and_z_face_fields():
    """update_halo_kernel.f90 applied twice equals applying it once for the
    cell fields, the vertex velocities and the z-face fluxes, at depth 1 and
    2, when each axis has at least three cells: the sources of every halo copy
    then lie inside the chunk along the face normal, and a corner cell that a
    face pass reads stale is rewritten by a later pass. The native step relies
    on this to leave out repeats of an update whose fields are unchanged since
    their last one (density1, energy1 and vol_flux_z in the second pre-sweep
    update of advection.f90, mass_flux_z after the x and y sweeps). The x- and
    y-face fluxes are not repeat-safe: the z faces do not reach their far
    halo columns (j = x_max+2.. for x faces), whose corners keep values a face
    pass read before a later pass wrote them. On thinner axes a face's high
    side reads cells its low side writes."""
    import hydro_harness as H
    rng = np.random.default_rng(11)
    lib = O.load()
    deck = {"initial_timestep": 0.04}
    safe = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity",
            "soundspeed", "xvel0", "xvel1", "yvel0", "yvel1", "zvel0", "zvel1", "vol_flux_z",
            "mass_flux_z"]
    unsafe = ["vol_flux_x", "mass_flux_x", "vol_flux_y", "mass_flux_y"]
    for nx, ny, nz in [(3, 3, 3), (5, 4, 6), (7, 3, 9), (4, 8, 3)]:
        for depth in (1, 2):
            a = H.new_chunk(nx, ny, nz)
            for k in H.ARRAYS_3D:
                a[k][...] = rng.standard_normal(a[k].shape)
            h = H.Hydro(H.Backend(lib, "oracle_"), a, nx, ny, nz, deck)
            h.halo(list(range(1, 20)), depth)
            once = H.clone(a)
            h.halo(list(range(1, 20)), depth)
            for k in safe:
                assert np.array_equal(a[k].view(np.uint64), once[k].view(np.uint64)), \
                    (nx, ny, nz, depth, k)
            for k in unsafe:
                assert not np.array_equal(a[k], once[k]), (nx, ny, nz, depth, k)
    # a one-cell axis: the repeat changes the far halo layer of a cell field
    a = H.new_chunk(4, 1, 4)
    for k in H.ARRAYS_3D:
        a[k][...] = rng.standard_normal(a[k].shape)
    h = H.Hydro(H.Backend(lib, "oracle_"), a, 4, 1, 4, deck)
    h.halo([1], 2)
    once = H.clone(a)
    h.halo([1], 2)
    assert not np.array_equal(a["density0"], once["density0"])


def test_depth_two_halo_update_rewrites_every_halo_cell_of_cell_and_vertex_fields():
    """A depth-2 update_halo_kernel.f90 call leaves the halo of every cell
    field and vertex velocity (and of vol_flux_z, mass_flux_z) a function of
    the interior alone, on grids with three or more cells per axis: two
    states with the same interior and different halos agree after it. The
    native step's out-of-place sweeps therefore copy no halo shell into their
    output buffers when such an update of those fields follows before the
    shell is read."""
    import hydro_harness as H
    rng = np.random.default_rng(5)
    lib = O.load()
    deck = {"initial_timestep": 0.04}
    extra = {"cell": (0, 0, 0), "vert": (1, 1, 1), "work": (1, 1, 1), "xface": (1, 0, 0),
             "yface": (0, 1, 0), "zface": (0, 0, 1)}
    fields = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity",
              "soundspeed", "xvel0", "xvel1", "yvel0", "yvel1", "zvel0", "zvel1", "vol_flux_z",
              "mass_flux_z"]
    for nx, ny, nz in [(3, 3, 3), (5, 4, 6), (7, 3, 9)]:
        base = H.new_chunk(nx, ny, nz)
        for k in H.ARRAYS_3D:
            base[k][...] = rng.standard_normal(base[k].shape)
        a, b = H.clone(base), H.clone(base)
        for k, kind in H.ARRAYS_3D.items():
            ex = extra[kind]
            halo = np.ones(b[k].shape, bool)
            halo[2:2 + nx + ex[0], 2:2 + ny + ex[1], 2:2 + nz + ex[2]] = False
            b[k][halo] = rng.standard_normal(int(halo.sum()))
        for arr in (a, b):
            H.Hydro(H.Backend(lib, "oracle_"), arr, nx, ny, nz, deck).halo(list(range(1, 20)), 2)
        for k in fields:
            assert np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64)), (nx, ny, nz, k)


# test_problem_1 turned onto y and z: the x axis and each axis it is exchanged
# with swap places, so arrays of the rotated run transpose onto the x run's.
_PERM = {1: (1, 0, 2), 2: (2, 1, 0)}


def _x_name(n, axis):
    """The rotated run's name for the x run's array n (velocity and face-flux
    components move with their axis)."""
    a = "xyz"[axis]
    swap = {"x": a, a: "x"}
    for c in "xyz":
        for suffix in ("vel0", "vel1"):
            if n == c + suffix:
                return swap.get(c, c) + suffix
        for prefix in ("vol_flux_", "mass_flux_"):
            if n == prefix + c:
                return prefix + swap.get(c, c)
    return n


def test_known_answer_with_the_flow_along_y_and_z():
    """The test_problem_1 shock run along y and along z meets the reference's
    own criterion (final KE within 0.001% of 3.64560737191257,
    field_summary.f90:119-136), so the y and z forms of the cell and momentum
    sweeps, their limiters, the y- and z-face halo rules and flux_calc's z
    form carry the known answer, not only the x forms."""
    g = json.load(open(os.path.join(GOLDEN, "test_problem_1.json")))
    for axis in (1, 2):
        r = O.run(decks.rotated(g["deck"], axis))
        assert r["steps"] == 75
        ke = r["summaries"][-1][3]
        assert abs(100.0 * (ke / g["final_kinetic_energy"]) - 100.0) < g["tolerance_percent"]


def test_rotations_differ_only_by_the_reference_halo_extents():
    """What separates the x, y and z runs of test_problem_1 is two
    direction-dependent extents of the reference, nothing in the restated
    arithmetic:
    - update_halo_kernel.f90 reflects the x and y face fluxes on the z faces
      over their face axis up to max+d (:1018-1142, :1156-1280), one node short
      of the z face fluxes' max+1+d (:1294-1417), so mass_flux_x(x_max+3) and
      mass_flux_y(y_max+3) in the z halo planes stay stale (the x and y
      momentum sweeps read them);
    - the y cell sweep forms fluxes up to z_max+2 (advec_cell_kernel.f90:220),
      into the z halo planes.
    The oracle built with both made symmetric (ORACLE_SYMMETRIC_HALO) gives
    the three rotations' summaries equal to 1e-14 at every step and dt equal
    bit for bit: the x, y and z forms of every kernel are the same arithmetic.
    The reference build's x run, with the stale corner, reproduces the known
    answer to 1e-15, while the symmetric build misses it by 7e-9: the known
    answer pins the stale corner too."""
    g = json.load(open(os.path.join(GOLDEN, "test_problem_1.json")))
    d = dict(g["deck"], summary_frequency=5)
    sym = [O.run(decks.rotated(d, a), symmetric=True) for a in range(3)]
    for a in (0, 1):
        assert np.array_equal(sym[a]["dt"], sym[2]["dt"])
        np.testing.assert_allclose(sym[a]["summaries"], sym[2]["summaries"], rtol=1e-14, atol=0)
    ke_ref = O.run(d)["summaries"][-1][3]
    ke_sym = sym[0]["summaries"][-1][3]
    assert abs(ke_ref / g["final_kinetic_energy"] - 1.0) < 1e-14
    assert abs(ke_sym / g["final_kinetic_energy"] - 1.0) > 1e-9


def test_rotated_runs_equal_the_x_run_to_rounding():
    """Before the stale corners reach the flow, every field of the y and z
    runs, transposed, equals the x run's to a few ulps and the transverse
    velocities are exactly zero (20 steps). Bit for bit they differ by an ulp
    from the first step: the cross-direction sweeps of a 1-D flow round
    (advec_cell's energy update e*m/m, advec_cell_kernel.f90:173-185, and
    advec_mom's velocity update v*m/m, advec_mom_kernel.f90:244-250, with zero
    fluxes), and the sweep order alternates (advection.f90:43-179)."""
    d = dict(decks.test_problem_1(), end_step=20, summary_frequency=5)
    rx = O.run(d, want_fields=True)
    for axis in (1, 2):
        rr = O.run(decks.rotated(d, axis), want_fields=True)
        assert np.array_equal(rr["dt"], rx["dt"])
        np.testing.assert_allclose(rr["summaries"], rx["summaries"], rtol=1e-14, atol=0)
        for c in (c for c in "xyz" if c != "xyz"[axis]):
            assert not np.any(rr["fields"][c + "vel0"]), (axis, c)
        for n in O.FIELD_NAMES:
            a = rx["fields"][n][2:-2, 2:-2, 2:-2]
            b = rr["fields"][_x_name(n, axis)].transpose(_PERM[axis])[2:-2, 2:-2, 2:-2]
            assert np.abs(a - b).max() <= 8 * np.spacing(np.abs(a).max()), (axis, n)


def test_fp64_mass_drift_is_the_flux_calc_z_sum():
    """On the benchmark's two-state problem the reference (FP64) does not
    conserve mass: 1e-4 relative over 40 steps at 24^3. flux_calc_kernel.f90:86
    sums zvel0 over nodes (j,k), (j+1,k), (j+1,k), (j+1,k+1) where the PdV
    kernel sums (j,k), (j+1,k), (j,k+1), (j+1,k+1), so the advection's z volume
    fluxes do not cancel the PdV volume change. A test-only build of the oracle
    whose z sum takes PdV's four nodes (ORACLE_FLUX_Z_PDV) conserves mass to
    rounding on the same deck: the drift is that sum's alone."""
    d = decks.shock(24, 24, 24, 40)
    ref = np.array(O.run(d)["summaries"])[:, 1]
    pdv = np.array(O.run(d, fluxz=True)["summaries"])[:, 1]
    assert np.abs(ref / ref[0] - 1).max() > 1e-5
    assert np.abs(pdv / pdv[0] - 1).max() < 1e-14


def _deck_of(struct, region_energy_scale=1.0):
    """A drawn ensemble deck (cloverleaf3d_ref_b200.draw_decks) as the oracle's
    mapping, the region's energy scaled."""
    s = struct
    d = {k: getattr(s, k) for k in ("x_cells", "y_cells", "z_cells", "xmin", "ymin", "zmin",
                                     "xmax", "ymax", "zmax", "initial_timestep", "max_timestep",
                                     "timestep_rise", "end_time", "end_step", "summary_frequency")}
    states = [dict(density=s.state_density[0], energy=s.state_energy[0])]
    states.append(dict(density=s.state_density[1], energy=s.state_energy[1] * region_energy_scale,
                       geometry="cuboid", xmin=s.state_xmin[1], xmax=s.state_xmax[1],
                       ymin=s.state_ymin[1], ymax=s.state_ymax[1], zmin=s.state_zmin[1],
                       zmax=s.state_zmax[1]))
    d["states"] = states
    return d


def test_drawn_ensemble_deck_is_ill_conditioned_in_fp64():
    """Deck 20 of the 64-deck ensemble (seed 2024; 35x111x96 cells on the
    [0,10]^3 cube): a 1e-7 relative change of the region's energy, FP64 alone,
    moves the internal energy by 4.9e-5 and the kinetic energy by 6.0e-5 (more
    than 1e-5 and 3e-5) within the configuration's 150 steps. A storage precision that
    rounds at 1e-7 every step cannot meet 1e-5 against FP64 on such decks."""
    import cloverleaf3d_ref_b200 as C
    s = C.draw_decks(64, 2024)[20].s
    assert (s.x_cells, s.y_cells, s.z_cells, s.end_step) == (35, 111, 96, 150)
    a = np.array(O.run(_deck_of(s), fast=True)["summaries"])
    b = np.array(O.run(_deck_of(s, 1.0 + 1e-7), fast=True)["summaries"])
    moving = a[:, 3] > 0
    assert np.abs(b[:, 2] / a[:, 2] - 1).max() > 1e-5
    assert np.abs(b[moving, 3] / a[moving, 3] - 1).max() > 3e-5
