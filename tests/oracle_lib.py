"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure only: the oracle is the checker, never the thing measured.
Arrays follow the reference layout (column major, lower bound min-2):
cell (nx+4, ny+4, nz+4), vertex/work (nx+5, ny+5, nz+5), x-face (nx+5, ny+4,
nz+4), y-face (nx+4, ny+5, nz+4), z-face (nx+4, ny+4, nz+5).
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
FAST_LIB_PATH = os.path.join(ORACLE_DIR, "_build", "liboracle_fast.so")
# parity build with two direction-dependent extents of the reference made
# symmetric (ORACLE_SYMMETRIC_HALO): only the rotation tests load it
SYMMETRIC_LIB_PATH = os.path.join(ORACLE_DIR, "_build", "liboracle_symmetric.so")
# parity build whose flux_calc z sum takes PdV's four nodes (ORACLE_FLUX_Z_PDV):
# only the mass-drift test loads it
FLUXZ_LIB_PATH = os.path.join(ORACLE_DIR, "_build", "liboracle_fluxz.so")

# Reference field ids (data.f90:55-74), 1-based, in order.
FIELD_NAMES = [
    "density0", "density1", "energy0", "energy1", "pressure", "viscosity",
    "soundspeed", "xvel0", "xvel1", "yvel0", "yvel1", "zvel0", "zvel1",
    "vol_flux_x", "vol_flux_y", "vol_flux_z", "mass_flux_x", "mass_flux_y",
    "mass_flux_z",
]
FIELD_KIND = {
    "density0": "cell", "density1": "cell", "energy0": "cell", "energy1": "cell",
    "pressure": "cell", "viscosity": "cell", "soundspeed": "cell",
    "xvel0": "vert", "xvel1": "vert", "yvel0": "vert", "yvel1": "vert",
    "zvel0": "vert", "zvel1": "vert",
    "vol_flux_x": "xface", "vol_flux_y": "yface", "vol_flux_z": "zface",
    "mass_flux_x": "xface", "mass_flux_y": "yface", "mass_flux_z": "zface",
}


def shape(kind, nx, ny, nz):
    """Fortran-order shape of a reference array of the given kind."""
    return {
        "cell": (nx + 4, ny + 4, nz + 4),
        "vert": (nx + 5, ny + 5, nz + 5),
        "work": (nx + 5, ny + 5, nz + 5),
        "xface": (nx + 5, ny + 4, nz + 4),
        "yface": (nx + 4, ny + 5, nz + 4),
        "zface": (nx + 4, ny + 4, nz + 5),
        "cx": (nx + 4,), "cy": (ny + 4,), "cz": (nz + 4,),
        "vx": (nx + 5,), "vy": (ny + 5,), "vz": (nz + 5,),
    }[kind]


class OracleDeck(ctypes.Structure):
    _fields_ = [
        ("x_cells", ctypes.c_int), ("y_cells", ctypes.c_int), ("z_cells", ctypes.c_int),
        ("xmin", ctypes.c_double), ("ymin", ctypes.c_double), ("zmin", ctypes.c_double),
        ("xmax", ctypes.c_double), ("ymax", ctypes.c_double), ("zmax", ctypes.c_double),
        ("dtinit", ctypes.c_double), ("dtmax", ctypes.c_double),
        ("dtrise", ctypes.c_double), ("dtmin", ctypes.c_double),
        ("end_time", ctypes.c_double), ("end_step", ctypes.c_int),
        ("summary_frequency", ctypes.c_int), ("number_of_states", ctypes.c_int),
        ("state_density", ctypes.c_double * 16), ("state_energy", ctypes.c_double * 16),
        ("state_xvel", ctypes.c_double * 16), ("state_yvel", ctypes.c_double * 16),
        ("state_zvel", ctypes.c_double * 16), ("state_xmin", ctypes.c_double * 16),
        ("state_xmax", ctypes.c_double * 16), ("state_ymin", ctypes.c_double * 16),
        ("state_ymax", ctypes.c_double * 16), ("state_zmin", ctypes.c_double * 16),
        ("state_zmax", ctypes.c_double * 16), ("state_radius", ctypes.c_double * 16),
        ("state_geometry", ctypes.c_int * 16),
    ]


def build():
    subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])


_LIBS = {}


def load(fast=False, symmetric=False, fluxz=False):
    path = (FLUXZ_LIB_PATH if fluxz else SYMMETRIC_LIB_PATH if symmetric
            else FAST_LIB_PATH if fast else LIB_PATH)
    if path not in _LIBS:
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        lib.oracle_run.restype = ctypes.c_int
        _LIBS[path] = lib
    return _LIBS[path]


def make_deck(d):
    """Fill an OracleDeck from a mapping with the deck keys (defaults of
    read_input.f90:38-86 for anything missing)."""
    od = OracleDeck()
    od.x_cells = d.get("x_cells", 10)
    od.y_cells = d.get("y_cells", 10)
    od.z_cells = d.get("z_cells", 10)
    od.xmin, od.ymin, od.zmin = d.get("xmin", 0.0), d.get("ymin", 0.0), d.get("zmin", 0.0)
    od.xmax, od.ymax, od.zmax = d.get("xmax", 100.0), d.get("ymax", 100.0), d.get("zmax", 100.0)
    od.dtinit = d.get("initial_timestep", 0.1)
    od.dtmax = d.get("max_timestep", 1.0)
    od.dtrise = d.get("timestep_rise", 1.05)
    od.dtmin = 0.0000001
    od.end_time = d.get("end_time", 10.0)
    od.end_step = d.get("end_step", 640000)
    od.summary_frequency = d.get("summary_frequency", 10)
    states = d["states"]
    od.number_of_states = len(states)
    for i, s in enumerate(states):
        od.state_density[i] = s.get("density", 0.0)
        od.state_energy[i] = s.get("energy", 0.0)
        od.state_xvel[i] = s.get("xvel", 0.0)
        od.state_yvel[i] = s.get("yvel", 0.0)
        od.state_zvel[i] = s.get("zvel", 0.0)
        od.state_xmin[i] = s.get("xmin", 0.0)
        od.state_xmax[i] = s.get("xmax", 0.0)
        od.state_ymin[i] = s.get("ymin", 0.0)
        od.state_ymax[i] = s.get("ymax", 0.0)
        od.state_zmin[i] = s.get("zmin", 0.0)
        od.state_zmax[i] = s.get("zmax", 0.0)
        od.state_radius[i] = s.get("radius", 0.0)
        od.state_geometry[i] = {"cuboid": 1, "sphere": 2, "point": 3}[s.get("geometry", "cuboid")]
    return od


def run(deck, max_steps=None, want_fields=False, fast=False, symmetric=False, fluxz=False):
    """Run the oracle hydro loop. Returns dict(dt, summaries, summary_steps, steps, fields)."""
    lib = load(fast, symmetric, fluxz)
    od = make_deck(deck)
    if max_steps is None:
        max_steps = od.end_step
    nsum_cap = max_steps // max(od.summary_frequency, 1) + 4
    dts = np.zeros(max_steps, dtype=np.float64)
    sums = np.zeros((nsum_cap, 5), dtype=np.float64)
    steps = np.zeros(nsum_cap, dtype=np.int32)
    nsum = ctypes.c_int(0)
    nx, ny, nz = od.x_cells, od.y_cells, od.z_cells
    fields = None
    fptr = None
    if want_fields:
        fields = {n: np.zeros(shape(FIELD_KIND[n], nx, ny, nz), order="F") for n in FIELD_NAMES}
        fptr = (ctypes.POINTER(ctypes.c_double) * 19)(
            *[fields[n].ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for n in FIELD_NAMES])
    nsteps = lib.oracle_run(
        ctypes.byref(od), ctypes.c_int(max_steps), dts.ctypes.data_as(ctypes.c_void_p),
        ctypes.c_int(nsum_cap), sums.ctypes.data_as(ctypes.c_void_p),
        steps.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nsum), fptr)
    n = min(nsum.value, nsum_cap)
    taken = abs(nsteps)
    return {
        "steps": nsteps, "dt": dts[:taken], "summaries": sums[:n],
        "summary_steps": steps[:n], "fields": fields,
    }


class KeptRun:
    """An oracle run whose chunk stays in host memory: dt, summaries and steps
    as run() gives them, and each field fetched on demand (for runs too large
    to hold every field twice)."""

    def __init__(self, deck, max_steps=None):
        lib = load()
        lib.oracle_run_keep.restype = ctypes.c_void_p
        lib.oracle_kept_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.oracle_kept_free.argtypes = [ctypes.c_void_p]
        self.lib = lib
        od = make_deck(deck)
        if max_steps is None:
            max_steps = od.end_step
        nsum_cap = max_steps // max(od.summary_frequency, 1) + 4
        dts = np.zeros(max_steps, dtype=np.float64)
        sums = np.zeros((nsum_cap, 5), dtype=np.float64)
        steps = np.zeros(nsum_cap, dtype=np.int32)
        nsum, nsteps = ctypes.c_int(0), ctypes.c_int(0)
        self.h = lib.oracle_run_keep(
            ctypes.byref(od), ctypes.c_int(max_steps), dts.ctypes.data_as(ctypes.c_void_p),
            ctypes.c_int(nsum_cap), sums.ctypes.data_as(ctypes.c_void_p),
            steps.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nsum), ctypes.byref(nsteps))
        if not self.h:
            raise MemoryError("oracle chunk allocation failed")
        n = min(nsum.value, nsum_cap)
        self.steps = nsteps.value
        self.dt = dts[:abs(nsteps.value)]
        self.summaries = sums[:n]
        self.summary_steps = steps[:n]
        self.dims = (od.x_cells, od.y_cells, od.z_cells)

    def field(self, name):
        a = np.zeros(shape(FIELD_KIND[name], *self.dims), order="F")
        assert self.lib.oracle_kept_field(self.h, FIELD_NAMES.index(name) + 1,
                                          a.ctypes.data_as(ctypes.c_void_p)) == 0
        return a

    def close(self):
        if self.h:
            self.lib.oracle_kept_free(self.h)
            self.h = None


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def iref(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def dref(v):
    return ctypes.byref(ctypes.c_double(float(v)))
