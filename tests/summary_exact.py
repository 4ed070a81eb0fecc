"""Per-cell terms of field_summary_kernel.f90:60-75 in numpy, and their sums.

The terms are formed with the kernel's operations in its order (numpy
evaluates elementwise IEEE double operations left to right, without
contraction), so summing them in the oracle's order gives the oracle's
summary bit for bit (pinned by tests/test_summary_sums.py), and math.fsum of
them gives the exactly rounded sum the compensated GPU sums are held to.
Arrays are reference-layout (Fortran order, lower bound min-2).
"""
import math

import numpy as np


def cell_volume(deck):
    """initialise_chunk_kernel.f90:113-175: dx = (xmax-xmin)/float(x_cells)
    (the count is exact in a default REAL), volume = dx*dy*dz."""
    dx = (deck["xmax"] - deck["xmin"]) / float(deck["x_cells"])
    dy = (deck["ymax"] - deck["ymin"]) / float(deck["y_cells"])
    dz = (deck["zmax"] - deck["zmin"]) / float(deck["z_cells"])
    return dx * dy * dz


def cell_terms(nx, ny, nz, volume, density0, energy0, pressure, xvel0, yvel0, zvel0):
    """The five per-cell terms (vol, mass, ie, ke, press) of the interior,
    each an (nx, ny, nz) Fortran-order array. volume: a scalar or a cell array."""
    I = (slice(2, nx + 2), slice(2, ny + 2), slice(2, nz + 2))

    def vert(a, dj, dk, dl):
        return a[2 + dj:nx + 2 + dj, 2 + dk:ny + 2 + dk, 2 + dl:nz + 2 + dl]

    vsqrd = np.zeros((nx, ny, nz), order="F")
    for dl in (0, 1):
        for dk in (0, 1):
            for dj in (0, 1):
                u, v, w = vert(xvel0, dj, dk, dl), vert(yvel0, dj, dk, dl), vert(zvel0, dj, dk, dl)
                vsqrd = vsqrd + 0.125 * (u * u + v * v + w * w)
    vol = np.broadcast_to(np.float64(volume), (nx, ny, nz)) if np.ndim(volume) == 0 else volume[I]
    mass = vol * density0[I]
    return [np.asfortranarray(vol), mass, mass * energy0[I], mass * 0.5 * vsqrd, vol * pressure[I]]


def oracle_order_sums(terms):
    """The oracle's order: each z plane summed in loop order (j fastest), then
    the plane sums added in z order."""
    out = []
    for t in terms:
        planes = [np.cumsum(t[:, :, l].ravel(order="F"))[-1] for l in range(t.shape[2])]
        s = 0.0
        for p in planes:
            s = s + p
        out.append(s)
    return np.array(out)


def exact_sums(terms):
    """Each quantity's sum of terms, exactly rounded (math.fsum)."""
    return np.array([math.fsum(t.ravel(order="F")) for t in terms])


def ulps(got, exact):
    """|got - exact| in units of the last place of exact, per quantity."""
    got, exact = np.asarray(got, dtype=np.float64), np.asarray(exact, dtype=np.float64)
    return np.abs(got - exact) / np.spacing(np.abs(exact))
