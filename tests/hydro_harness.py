"""One CloverLeaf3D hydro step driven kernel by kernel through either backend.

The oracle (oracle/_build/liboracle.so, prefix ``oracle_``) and the drop-in
ABI (libclover_b200.so, prefix ``clover_``) export the same argument lists,
so the same Python restatement of the reference drivers (timestep.f90,
PdV.f90, advection.f90, ...) runs on both. ``Backend.after`` is called after
every kernel so a test can compare all arrays call by call.
"""
import ctypes

import numpy as np

import oracle_lib as O

G_SMALL = float(np.float32(1.0e-16))  # data.f90:30 (a default REAL literal)
G_BIG = float(np.float32(1.0e21))     # data.f90:31

ARRAYS_3D = {
    "density0": "cell", "density1": "cell", "energy0": "cell", "energy1": "cell",
    "pressure": "cell", "viscosity": "cell", "soundspeed": "cell", "volume": "cell",
    "xvel0": "vert", "xvel1": "vert", "yvel0": "vert", "yvel1": "vert",
    "zvel0": "vert", "zvel1": "vert",
    "vol_flux_x": "xface", "mass_flux_x": "xface", "xarea": "xface",
    "vol_flux_y": "yface", "mass_flux_y": "yface", "yarea": "yface",
    "vol_flux_z": "zface", "mass_flux_z": "zface", "zarea": "zface",
    "wa1": "work", "wa2": "work", "wa3": "work", "wa4": "work", "wa5": "work",
    "wa6": "work", "wa7": "work",
}
ARRAYS_1D = {
    "cellx": "cx", "celly": "cy", "cellz": "cz", "celldx": "cx", "celldy": "cy",
    "celldz": "cz", "vertexx": "vx", "vertexy": "vy", "vertexz": "vz",
    "vertexdx": "vx", "vertexdy": "vy", "vertexdz": "vz",
}


def new_chunk(nx, ny, nz):
    """build_field.f90: every array zeroed."""
    a = {}
    for n, k in ARRAYS_3D.items():
        a[n] = np.zeros(O.shape(k, nx, ny, nz), order="F")
    for n, k in ARRAYS_1D.items():
        a[n] = np.zeros(O.shape(k, nx, ny, nz))
    return a


def clone(a):
    return {k: v.copy(order="K") for k, v in a.items()}


def p(x):
    return x.ctypes.data_as(ctypes.c_void_p)


def I(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def D(v):
    return ctypes.byref(ctypes.c_double(float(v)))


class Backend:
    def __init__(self, lib, prefix, after=None):
        self.lib = lib
        self.prefix = prefix
        self.after_hook = after

    def call(self, name, *args):
        getattr(self.lib, self.prefix + name)(*args)
        if self.after_hook:
            self.after_hook(name)


class Hydro:
    """The reference drivers over one chunk's arrays and one backend."""

    def __init__(self, backend, arrays, nx, ny, nz, deck):
        self.b = backend
        self.a = arrays
        self.nx, self.ny, self.nz = nx, ny, nz
        self.deck = deck
        self.bounds = [ctypes.c_int(v) for v in (1, nx, 1, ny, 1, nz)]
        self.dt = deck["initial_timestep"]
        self.dtold = deck["initial_timestep"]
        self.advect_x = True

    def B(self):
        return [ctypes.byref(v) for v in self.bounds]

    def A(self, *names):
        return [p(self.a[n]) for n in names]

    # initialise_chunk.f90 + generate_chunk.f90 + start.f90:99-136
    def start(self):
        d = self.deck
        dx = (d["xmax"] - d["xmin"]) / float(np.float32(self.nx))
        dy = (d["ymax"] - d["ymin"]) / float(np.float32(self.ny))
        dz = (d["zmax"] - d["zmin"]) / float(np.float32(self.nz))
        self.b.call("initialise_chunk_kernel", *self.B(), D(d["xmin"]), D(d["ymin"]),
                    D(d["zmin"]), D(dx), D(dy), D(dz),
                    *self.A("vertexx", "vertexdx", "vertexy", "vertexdy", "vertexz",
                            "vertexdz", "cellx", "celldx", "celly", "celldy", "cellz",
                            "celldz", "volume", "xarea", "yarea", "zarea"))
        st = d["states"]
        n = len(st)
        arr = {k: (ctypes.c_double * n)(*[s.get(k, 0.0) for s in st])
               for k in ("density", "energy", "xvel", "yvel", "zvel", "xmin", "xmax",
                         "ymin", "ymax", "zmin", "zmax", "radius")}
        for i in range(1, n):  # read_input.f90:293-303
            arr["xmin"][i] += dx / 100.0
            arr["ymin"][i] += dy / 100.0
            arr["zmin"][i] += dz / 100.0
            arr["xmax"][i] -= dx / 100.0
            arr["ymax"][i] -= dy / 100.0
            arr["zmax"][i] -= dz / 100.0
        geo = (ctypes.c_int * n)(*[{"cuboid": 1, "sphere": 2, "point": 3}[s.get("geometry", "cuboid")]
                                   for s in st])
        self.b.call("generate_chunk_kernel", *self.B(),
                    *self.A("vertexx", "vertexy", "vertexz", "cellx", "celly", "cellz",
                            "density0", "energy0", "xvel0", "yvel0", "zvel0"),
                    I(n), arr["density"], arr["energy"], arr["xvel"], arr["yvel"], arr["zvel"],
                    arr["xmin"], arr["xmax"], arr["ymin"], arr["ymax"], arr["zmin"], arr["zmax"],
                    arr["radius"], geo, I(1), I(2), I(3))
        self.ideal_gas(False)
        self.halo([1, 3, 5, 6, 2, 4, 8, 10, 12, 9, 11, 13], 2)

    def halo(self, ids, depth):
        fields = (ctypes.c_int * 19)(*[1 if i + 1 in ids else 0 for i in range(19)])
        nb = (ctypes.c_int * 6)(-1, -1, -1, -1, -1, -1)
        self.b.call("update_halo_kernel", *self.B(), nb, nb,
                    *self.A("density0", "energy0", "pressure", "viscosity", "soundspeed",
                            "density1", "energy1", "xvel0", "yvel0", "zvel0", "xvel1",
                            "yvel1", "zvel1", "vol_flux_x", "vol_flux_y", "vol_flux_z",
                            "mass_flux_x", "mass_flux_y", "mass_flux_z"),
                    fields, I(depth))

    def ideal_gas(self, predict):
        if predict:
            self.b.call("ideal_gas_kernel", *self.B(),
                        *self.A("density1", "energy1", "pressure", "soundspeed"))
        else:
            self.b.call("ideal_gas_kernel", *self.B(),
                        *self.A("density0", "energy0", "pressure", "soundspeed"))

    def timestep(self):
        self.ideal_gas(False)
        self.halo([5, 3, 1, 8, 10], 1)
        self.b.call("viscosity_kernel", *self.B(),
                    *self.A("xarea", "yarea", "zarea", "celldx", "celldy", "celldz",
                            "density0", "pressure", "viscosity", "xvel0", "yvel0", "zvel0"))
        self.halo([6], 1)
        dtlp = ctypes.c_double(0)
        xl, yl, zl = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
        ctl, jl, kl, ll, small = (ctypes.c_int(0) for _ in range(5))
        self.b.call("calc_dt_kernel", *self.B(), D(G_SMALL), D(G_BIG), D(1e-7), D(0.75),
                    D(0.5), D(0.5), D(0.5), D(0.5),
                    *self.A("xarea", "yarea", "zarea", "cellx", "celly", "cellz", "celldx",
                            "celldy", "celldz", "volume", "density0", "energy0", "pressure",
                            "viscosity", "soundspeed", "xvel0", "yvel0", "zvel0", "wa1"),
                    ctypes.byref(dtlp), ctypes.byref(ctl), ctypes.byref(xl), ctypes.byref(yl),
                    ctypes.byref(zl), ctypes.byref(jl), ctypes.byref(kl), ctypes.byref(ll),
                    ctypes.byref(small))
        self.calc_dt_out = (dtlp.value, ctl.value, xl.value, yl.value, zl.value, jl.value,
                            kl.value, ll.value, small.value)
        dt = G_BIG
        if dtlp.value <= dt:
            dt = dtlp.value
        dt = min(dt, self.dtold * self.deck.get("timestep_rise", 1.05),
                 self.deck["max_timestep"])
        self.dt = dt
        self.dtold = dt

    def pdv(self, predict):
        self.b.call("pdv_kernel", I(1 if predict else 0), *self.B(), D(self.dt),
                    *self.A("xarea", "yarea", "zarea", "volume", "density0", "density1",
                            "energy0", "energy1", "pressure", "viscosity", "xvel0", "xvel1",
                            "yvel0", "yvel1", "zvel0", "zvel1"))
        if predict:
            self.ideal_gas(True)
            self.halo([5], 1)
            self.b.call("revert_kernel", *self.B(),
                        *self.A("density0", "density1", "energy0", "energy1"))

    def accelerate(self):
        self.b.call("accelerate_kernel", *self.B(), D(self.dt),
                    *self.A("xarea", "yarea", "zarea", "volume", "density0", "pressure",
                            "viscosity", "xvel0", "yvel0", "zvel0", "xvel1", "yvel1", "zvel1"))

    def flux_calc(self):
        self.b.call("flux_calc_kernel", *self.B(), D(self.dt),
                    *self.A("xarea", "yarea", "zarea", "xvel0", "yvel0", "zvel0", "xvel1",
                            "yvel1", "zvel1", "vol_flux_x", "vol_flux_y", "vol_flux_z"))

    def advec_cell(self, sweep, direction):
        self.b.call("advec_cell_kernel", *self.B(), I(1 if self.advect_x else 0), I(direction),
                    I(sweep),
                    *self.A("vertexdx", "vertexdy", "vertexdz", "volume", "density1",
                            "energy1", "mass_flux_x", "vol_flux_x", "mass_flux_y",
                            "vol_flux_y", "mass_flux_z", "vol_flux_z", "wa1", "wa2", "wa3",
                            "wa4", "wa5", "wa6", "wa7"))

    def advec_mom(self, which, direction, sweep):
        vel = ["xvel1", "yvel1", "zvel1"][which - 1]
        self.b.call("advec_mom_kernel", *self.B(),
                    *self.A(vel, "mass_flux_x", "vol_flux_x", "mass_flux_y", "vol_flux_y",
                            "mass_flux_z", "vol_flux_z", "volume", "density1", "wa1", "wa2",
                            "wa3", "wa4", "wa5", "wa6", "wa7", "celldx", "celldy", "celldz"),
                    I(1 if self.advect_x else 0), I(which), I(sweep), I(direction))

    def advection(self):
        pre = [4, 2, 14, 15, 16]
        post = [2, 4, 9, 11, 13, 17, 18, 19]
        d = 1 if self.advect_x else 3
        self.halo(pre, 2)
        self.advec_cell(1, d)
        self.halo(post, 2)
        for v in (1, 2, 3):
            self.advec_mom(v, d, 1)
        self.halo(pre, 2)
        self.advec_cell(2, 2)
        self.halo(post, 2)
        for v in (1, 2, 3):
            self.advec_mom(v, 2, 2)
        d = 3 if self.advect_x else 1
        self.advec_cell(3, d)
        self.halo(post, 2)
        for v in (1, 2, 3):
            self.advec_mom(v, d, 3)

    def reset_field(self):
        self.b.call("reset_field_kernel", *self.B(),
                    *self.A("density0", "density1", "energy0", "energy1", "xvel0", "xvel1",
                            "yvel0", "yvel1", "zvel0", "zvel1"))

    def field_summary(self):
        self.ideal_gas(False)
        out = [ctypes.c_double(0) for _ in range(5)]
        self.b.call("field_summary_kernel", *self.B(),
                    *self.A("volume", "density0", "energy0", "pressure", "xvel0", "yvel0",
                            "zvel0"), *[ctypes.byref(o) for o in out])
        return [o.value for o in out]

    def step(self):
        self.timestep()
        self.pdv(True)
        self.accelerate()
        self.pdv(False)
        self.flux_calc()
        self.advection()
        self.reset_field()
        self.advect_x = not self.advect_x
