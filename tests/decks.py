"""Decks used by the tests (values only; the problem is the reference's
two-state shock of clover.in and of the default deck of initialise.f90:77-93)."""

TWO_STATE = [
    dict(density=0.2, energy=1.0),
    dict(density=1.0, energy=2.5, geometry="cuboid", xmin=0.0, xmax=5.0, ymin=0.0,
         ymax=2.0, zmin=0.0, zmax=2.0),
]


def shock(nx, ny, nz, steps, states=None, **kw):
    """The two-state shock on [0,10]^3 (the benchmark problem's geometry)."""
    d = dict(x_cells=nx, y_cells=ny, z_cells=nz, xmin=0.0, ymin=0.0, zmin=0.0,
             xmax=10.0, ymax=10.0, zmax=10.0, initial_timestep=0.04, max_timestep=0.04,
             timestep_rise=1.5, end_step=steps, end_time=1000.0, summary_frequency=10,
             states=states or TWO_STATE)
    d.update(kw)
    return d


def test_problem_1():
    """Default deck of initialise.f90:77-93 (pins the known answer)."""
    return dict(x_cells=10, y_cells=2, z_cells=2, xmin=0.0, ymin=0.0, zmin=0.0,
                xmax=10.0, ymax=2.0, zmax=2.0, initial_timestep=0.04, max_timestep=0.04,
                end_step=75, states=TWO_STATE)


def rotated(d, axis):
    """The deck with its x axis exchanged for axis 1 (y) or 2 (z): cell
    counts, domain bounds, and each state's bounds and velocity move with the
    axis, so a flow along x becomes the same flow along y or z."""
    if axis == 0:
        return dict(d, states=[dict(s) for s in d["states"]])
    a = "xyz"[axis]
    r = dict(d)
    for kx, ka in (("x_cells", a + "_cells"), ("xmin", a + "min"), ("xmax", a + "max")):
        if kx in d or ka in d:
            r[kx], r[ka] = d.get(ka), d.get(kx)
    states = []
    for s in d["states"]:
        t = {k: v for k, v in s.items() if k not in ("xmin", "xmax", "xvel", a + "min", a + "max", a + "vel")}
        for kx, ka in (("xmin", a + "min"), ("xmax", a + "max"), ("xvel", a + "vel")):
            if ka in s:
                t[kx] = s[ka]
            if kx in s:
                t[ka] = s[kx]
        states.append(t)
    r["states"] = states
    return r


def test_problem_1_along(axis):
    """test_problem_1 with its flow along x (0), y (1) or z (2)."""
    return rotated(test_problem_1(), axis)


# A deck with every geometry kind and moving states, on an uneven grid.
MIXED_STATES = [
    dict(density=0.2, energy=1.0, xvel=0.1),
    dict(density=1.0, energy=2.5, geometry="cuboid", xmin=0.0, xmax=4.0, ymin=1.0,
         ymax=6.0, zmin=0.0, zmax=3.0, yvel=-0.2),
    dict(density=2.0, energy=0.5, geometry="sphere", xmin=7.0, ymin=3.0, zmin=6.0,
         radius=2.2, zvel=0.3),
    dict(density=3.0, energy=4.0, geometry="point", xmin=0.0, ymin=0.0, zmin=0.0),
]


def to_deck(d):
    """A cloverleaf3d_ref_b200.Deck from a dict deck."""
    import cloverleaf3d_ref_b200 as C
    kw = {k: v for k, v in d.items() if k != "states"}
    return C.Deck.from_values(states=d["states"], **kw)
