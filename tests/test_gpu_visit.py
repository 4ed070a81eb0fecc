"""VTK output (visit.f90): a run with visit_frequency writes clover.visit and
one legacy ASCII VTK file per visit (at step 0, every visit_frequency steps
and after the final step), with the rectilinear grid of the vertex
coordinates, the cell fields density/energy/pressure/viscosity and the node
velocities in E12.4, viscosity at or below 1e-8 and velocities within 1e-8
of zero written as zero."""
import os

import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C
import decks

pytestmark = pytest.mark.gpu


def read_vtk(path):
    lines = open(path).read().splitlines()
    assert lines[:4] == ["# vtk DataFile Version 3.0", "vtk output", "ASCII",
                         "DATASET RECTILINEAR_GRID"]
    out, i = {}, 4
    dims = [int(x) for x in lines[i].split()[1:]]
    i += 1
    while i < len(lines):
        w = lines[i].split()
        if w[0] in ("X_COORDINATES", "Y_COORDINATES", "Z_COORDINATES"):
            n = int(w[1])
            out[w[0]] = np.array([float(x) for x in lines[i + 1:i + 1 + n]])
            i += 1 + n
        elif w[0] in ("CELL_DATA", "POINT_DATA") or w[0] == "FIELD":
            i += 1
        else:
            n = int(w[2])
            assert all(len(x) == 12 for x in lines[i + 1:i + 1 + n])
            out[w[0]] = np.array([float(x.replace("+1", "E+1") if "E" not in x else x)
                                  for x in lines[i + 1:i + 1 + n]])
            i += 1 + n
    return dims, out


def test_visit_files(tmp_path):
    nx, ny, nz = 11, 7, 6
    d = decks.to_deck(decks.shock(nx, ny, nz, 10, states=decks.MIXED_STATES,
                                  visit_frequency=5, summary_frequency=5))
    ch = C.Chunk(d)
    ch.set_visit_dir(str(tmp_path))
    assert ch.run() == 10
    index = open(os.path.join(str(tmp_path), "clover.visit")).read().splitlines()
    assert index[0] == "!NBLOCKS     0"
    assert index[1:] == ["clover.00001.00000.vtk", "clover.00001.00005.vtk",
                         "clover.00001.00010.vtk", "clover.00001.00010.vtk"]
    dims, v = read_vtk(os.path.join(str(tmp_path), "clover.00001.00010.vtk"))
    assert dims == [nx + 1, ny + 1, nz + 1]
    np.testing.assert_allclose(v["X_COORDINATES"], np.linspace(0, 10, nx + 1), rtol=5e-4, atol=1e-12)
    rho = ch.field("density0")[2:2 + nx, 2:2 + ny, 2:2 + nz]
    np.testing.assert_allclose(v["density"], rho.flatten(order="F"), rtol=5e-4)
    e = ch.field("energy0")[2:2 + nx, 2:2 + ny, 2:2 + nz]
    np.testing.assert_allclose(v["energy"], e.flatten(order="F"), rtol=5e-4)
    q = ch.field("viscosity")[2:2 + nx, 2:2 + ny, 2:2 + nz].flatten(order="F")
    np.testing.assert_allclose(v["viscosity"], np.where(q > 1e-8, q, 0.0), rtol=5e-4, atol=0)
    u = ch.field("xvel0")[2:3 + nx, 2:3 + ny, 2:3 + nz].flatten(order="F")
    np.testing.assert_allclose(v["x_vel"], np.where(np.abs(u) > 1e-8, u, 0.0), rtol=5e-4, atol=0)
    assert np.any(v["x_vel"] != 0.0) and np.any(v["viscosity"] != 0.0)
    ch.close()
