"""The library's deck reader: read_input.f90 keys and defaults, parse.f90
lexing (comments, '=' and ',' as blanks, case folding)."""
import pytest

import cloverleaf3d_ref_b200 as C

DECK = """
*clover
 state 1 density=0.2 energy=1.0
 state 2 density=1.0 energy=2.5 geometry=cuboid xmin=0.0 xmax=5.0 ymin=0.0 ymax=2.0 zmin=0.0 zmax=2.0
 x_cells=96
 Y_CELLS=48 ! trailing comment
 z_cells 32
 xmin=0.0
 xmax=10.0 ; another comment
 ymax=10.0
 zmax=10.0
 initial_timestep=0.04
 max_timestep=0.04
 timestep_rise=1.5
 end_step=300
 end_time=12.5
 test_problem 1
*endclover
 x_cells=7
"""


def test_parse_keys():
    d = C.Deck.parse(DECK)
    assert (d.x_cells, d.y_cells, d.z_cells) == (96, 48, 32)
    assert (d.xmax, d.ymax, d.zmax) == (10.0, 10.0, 10.0)
    assert (d.initial_timestep, d.max_timestep, d.timestep_rise) == (0.04, 0.04, 1.5)
    assert (d.end_step, d.end_time, d.test_problem) == (300, 12.5, 1)
    assert d.number_of_states == 2
    assert d.state_density[1] == 1.0 and d.state_energy[1] == 2.5
    assert d.state_geometry[1] == 1
    assert (d.state_xmax[1], d.state_ymax[1], d.state_zmax[1]) == (5.0, 2.0, 2.0)


def test_defaults_read_input():
    d = C.Deck.parse("*clover\n state 1 density=1 energy=1\n*endclover\n")
    assert (d.x_cells, d.y_cells, d.z_cells) == (10, 10, 10)
    assert (d.xmin, d.xmax) == (0.0, 100.0)
    assert d.end_time == 10.0 and d.end_step == 640000
    assert d.summary_frequency == 10 and d.visit_frequency == 0
    assert (d.initial_timestep, d.max_timestep, d.timestep_rise) == (0.1, 1.0, 1.05)
    assert d.dtmin == 1e-7 and d.dtc_safe == 0.75 and d.dtu_safe == 0.5
    # an integer word is read as a real ("1" -> 1.0)
    assert d.state_density[0] == 1.0


def test_errors():
    with pytest.raises(C.CloverError, match="No states"):
        C.Deck.parse("*clover\n x_cells=4\n*endclover\n")
    with pytest.raises(C.CloverError, match="twice"):
        C.Deck.parse("*clover\n state 1 density=1\n state 1 density=2\n*endclover\n")


def test_geometry_kinds_and_value_on_next_line():
    d = C.Deck.parse("*clover\n state 1 density=1 energy=1\n"
                     " state 2 density=2 energy=1 geometry=sphere xmin=1 ymin=2 zmin=3 radius=0.5\n"
                     " state 3 geometry=point xmin=0 ymin=0 zmin=0 density=3 energy=3\n"
                     " end_step\n 17\n*endclover\n")
    assert list(d.state_geometry[:3])[1:] == [2, 3]
    assert d.state_radius[1] == 0.5
    assert d.end_step == 17
