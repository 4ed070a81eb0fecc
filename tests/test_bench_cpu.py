"""CPU: the bench's conversion of library decks to the oracle's deck mapping
(used by its CPU legs) keeps every value the oracle reads."""
import os
import sys

import oracle_lib as O

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
import cloverleaf3d_ref_b200 as C  # noqa: E402


def test_drawn_deck_converts_to_the_oracle_deck():
    for dk in C.draw_decks(3, 77, cells=(16, 48), end_step=40, summary_frequency=5):
        d = bench.deck_dict(dk)
        od = O.make_deck(d)
        s = dk.s
        assert (od.x_cells, od.y_cells, od.z_cells) == (s.x_cells, s.y_cells, s.z_cells)
        assert (od.end_step, od.summary_frequency) == (40, 5)
        assert (od.dtinit, od.dtmax, od.dtrise) == (s.initial_timestep, s.max_timestep,
                                                     s.timestep_rise)
        assert od.number_of_states == s.number_of_states == 2
        for i in range(2):
            for f in ("density", "energy", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax"):
                assert getattr(od, "state_" + f)[i] == getattr(s, "state_" + f)[i], f
        assert od.state_geometry[1] == s.state_geometry[1] == 1  # cuboid


def test_benchmark_deck_values():
    d = bench.deck_values(512, 23)
    assert (d["x_cells"], d["end_step"], d["summary_frequency"]) == (512, 23, 10)
    assert (d["initial_timestep"], d["max_timestep"], d["timestep_rise"]) == (0.04, 0.04, 1.5)
    assert (d["xmax"], d["ymax"], d["zmax"]) == (10.0, 10.0, 10.0)
