"""The reference's decomposed run on the CPU oracle: the checker of the
library's brick driver (cloverleaf3d_ref_b200.Bricks).

Each brick is one chunk of clover_decompose's grid with its own arrays
(build_field.f90), set up with its mesh origin at its first cell
(initialise_chunk.f90:38-46); the drivers of hydro.f90 make every kernel call
on each brick in turn; every update_halo first exchanges the bricks' halo
messages (clover.f90:474-713: x, then y, then z; oracle_pack_message packs the
sender's side and unpacks the receiver's opposite side) and then applies the
reflective rules on each brick's external faces (update_halo.f90:38-86);
timestep.f90 takes the minimum of the bricks' dt (clover_min) and
field_summary.f90 adds the bricks' sums in brick order (clover_sum).
"""
import ctypes

import numpy as np

import cloverleaf3d_ref_b200 as C
import hydro_harness as H
import oracle_lib as O

# field ids 1..19 (data.f90:55-74) and the arrays they name
FIELDS = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed",
          "xvel0", "xvel1", "yvel0", "yvel1", "zvel0", "zvel1", "vol_flux_x", "vol_flux_y",
          "vol_flux_z", "mass_flux_x", "mass_flux_y", "mass_flux_z"]


def field_type(fid):
    """pack_kernel.f90's CELL/VERTEX/X_FACE/Y_FACE/Z_FACE_DATA as 1..5."""
    if fid <= 7:
        return 1
    if fid <= 13:
        return 2
    return {14: 3, 17: 3, 15: 4, 18: 4}.get(fid, 5)


class BrickOracle:
    def __init__(self, d, n):
        self.lib = O.load()
        self.lib.oracle_pack_message.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 16
        self.d = d
        _, self.ext, self.nbr = C.decompose(d["x_cells"], d["y_cells"], d["z_cells"], n)
        self.h = []
        for e in self.ext:
            nx, ny, nz = e[1] - e[0] + 1, e[3] - e[2] + 1, e[5] - e[4] + 1
            self.h.append(H.Hydro(H.Backend(self.lib, "oracle_"), H.new_chunk(nx, ny, nz),
                                  nx, ny, nz, d))
        self.dt = self.dtold = d["initial_timestep"]
        self.time = 0.0
        self.step_no = 0
        self.advect_x = True
        self.dts, self.sums, self.sum_steps = [], [], []

    # ---- halo: messages between the bricks, then the reflective faces ----
    def message(self, i, side, fid, depth, buf, pack):
        h = self.h[i]
        iv = H.I
        a = h.a[FIELDS[fid - 1]]
        self.lib.oracle_pack_message(side, 1 if pack else 0, *h.B(), H.p(a), H.p(buf), iv(depth),
                                     iv(field_type(fid)), iv(0), iv(0), iv(0),
                                     iv(h.nx), iv(h.ny), iv(h.nz))

    def halo(self, ids, depth):
        for axis in range(3):
            for i in range(len(self.h)):
                hi = int(self.nbr[i][2 * axis + 1])
                if hi < 0:
                    continue
                for fid in ids:
                    buf = np.zeros(4 * (max(hh.nx for hh in self.h) + 8) ** 2 * 8)
                    self.message(i, 2 * axis + 1, fid, depth, buf, True)
                    self.message(hi - 1, 2 * axis, fid, depth, buf, False)
                    buf[:] = 0
                    self.message(hi - 1, 2 * axis, fid, depth, buf, True)
                    self.message(i, 2 * axis + 1, fid, depth, buf, False)
        for i, h in enumerate(self.h):
            fields = (ctypes.c_int * 19)(*[1 if k + 1 in ids else 0 for k in range(19)])
            cn = (ctypes.c_int * 6)(*[int(v) for v in self.nbr[i]])
            tn = (ctypes.c_int * 6)(-1, -1, -1, -1, -1, -1)
            h.b.call("update_halo_kernel", *h.B(), cn, tn,
                     *h.A("density0", "energy0", "pressure", "viscosity", "soundspeed",
                          "density1", "energy1", "xvel0", "yvel0", "zvel0", "xvel1",
                          "yvel1", "zvel1", "vol_flux_x", "vol_flux_y", "vol_flux_z",
                          "mass_flux_x", "mass_flux_y", "mass_flux_z"),
                     fields, H.I(depth))

    # ---- start.f90 per brick ----
    def start(self):
        d = self.d
        dx = (d["xmax"] - d["xmin"]) / float(np.float32(d["x_cells"]))
        dy = (d["ymax"] - d["ymin"]) / float(np.float32(d["y_cells"]))
        dz = (d["zmax"] - d["zmin"]) / float(np.float32(d["z_cells"]))
        st = d["states"]
        n = len(st)
        for h, e in zip(self.h, self.ext):
            xmin = d["xmin"] + dx * float(np.float32(e[0] - 1))
            ymin = d["ymin"] + dy * float(np.float32(e[2] - 1))
            zmin = d["zmin"] + dz * float(np.float32(e[4] - 1))
            h.b.call("initialise_chunk_kernel", *h.B(), H.D(xmin), H.D(ymin), H.D(zmin), H.D(dx),
                     H.D(dy), H.D(dz),
                     *h.A("vertexx", "vertexdx", "vertexy", "vertexdy", "vertexz", "vertexdz",
                          "cellx", "celldx", "celly", "celldy", "cellz", "celldz", "volume",
                          "xarea", "yarea", "zarea"))
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
            h.b.call("generate_chunk_kernel", *h.B(),
                     *h.A("vertexx", "vertexy", "vertexz", "cellx", "celly", "cellz",
                          "density0", "energy0", "xvel0", "yvel0", "zvel0"),
                     H.I(n), arr["density"], arr["energy"], arr["xvel"], arr["yvel"],
                     arr["zvel"], arr["xmin"], arr["xmax"], arr["ymin"], arr["ymax"],
                     arr["zmin"], arr["zmax"], arr["radius"], geo, H.I(1), H.I(2), H.I(3))
            h.ideal_gas(False)
        self.halo([1, 3, 5, 6, 2, 4, 8, 10, 12, 9, 11, 13], 2)
        self.summary()

    def summary(self):
        t = np.zeros(5)
        for h in self.h:
            t += np.array(h.field_summary())  # ideal_gas then the kernel, brick by brick
        self.sums.append(t)
        self.sum_steps.append(self.step_no)

    def timestep(self):
        dt = H.G_BIG
        for h in self.h:
            h.ideal_gas(False)
        self.halo([5, 3, 1, 8, 10], 1)
        for h in self.h:
            h.b.call("viscosity_kernel", *h.B(),
                     *h.A("xarea", "yarea", "zarea", "celldx", "celldy", "celldz", "density0",
                          "pressure", "viscosity", "xvel0", "yvel0", "zvel0"))
        self.halo([6], 1)
        for h in self.h:
            dtlp = ctypes.c_double(0)
            xl, yl, zl = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
            ctl, jl, kl, ll, small = (ctypes.c_int(0) for _ in range(5))
            h.b.call("calc_dt_kernel", *h.B(), H.D(H.G_SMALL), H.D(H.G_BIG), H.D(1e-7), H.D(0.75),
                     H.D(0.5), H.D(0.5), H.D(0.5), H.D(0.5),
                     *h.A("xarea", "yarea", "zarea", "cellx", "celly", "cellz", "celldx",
                          "celldy", "celldz", "volume", "density0", "energy0", "pressure",
                          "viscosity", "soundspeed", "xvel0", "yvel0", "zvel0", "wa1"),
                     ctypes.byref(dtlp), ctypes.byref(ctl), ctypes.byref(xl), ctypes.byref(yl),
                     ctypes.byref(zl), ctypes.byref(jl), ctypes.byref(kl), ctypes.byref(ll),
                     ctypes.byref(small))
            if dtlp.value <= dt:
                dt = dtlp.value
        dt = min(dt, self.dtold * self.d.get("timestep_rise", 1.05), self.d["max_timestep"])
        self.dt = self.dtold = dt
        for h in self.h:
            h.dt = dt

    def pdv(self, predict):
        for h in self.h:
            h.b.call("pdv_kernel", H.I(1 if predict else 0), *h.B(), H.D(self.dt),
                     *h.A("xarea", "yarea", "zarea", "volume", "density0", "density1",
                          "energy0", "energy1", "pressure", "viscosity", "xvel0", "xvel1",
                          "yvel0", "yvel1", "zvel0", "zvel1"))
        if predict:
            for h in self.h:
                h.ideal_gas(True)
            self.halo([5], 1)
            for h in self.h:
                h.b.call("revert_kernel", *h.B(),
                         *h.A("density0", "density1", "energy0", "energy1"))

    def advection(self):
        pre = [4, 2, 14, 15, 16]
        post = [2, 4, 9, 11, 13, 17, 18, 19]
        for h in self.h:
            h.advect_x = self.advect_x
        d = 1 if self.advect_x else 3
        self.halo(pre, 2)
        for h in self.h:
            h.advec_cell(1, d)
        self.halo(post, 2)
        for v in (1, 2, 3):
            for h in self.h:
                h.advec_mom(v, d, 1)
        self.halo(pre, 2)
        for h in self.h:
            h.advec_cell(2, 2)
        self.halo(post, 2)
        for v in (1, 2, 3):
            for h in self.h:
                h.advec_mom(v, 2, 2)
        d = 3 if self.advect_x else 1
        for h in self.h:
            h.advec_cell(3, d)
        self.halo(post, 2)
        for v in (1, 2, 3):
            for h in self.h:
                h.advec_mom(v, d, 3)

    def run(self):
        d = self.d
        self.start()
        while True:
            self.step_no += 1
            self.timestep()
            self.dts.append(self.dt)
            self.pdv(True)
            for h in self.h:
                h.accelerate()
            self.pdv(False)
            for h in self.h:
                h.flux_calc()
            self.advection()
            for h in self.h:
                h.reset_field()
            self.advect_x = not self.advect_x
            self.time += self.dt
            # read_input.f90 defaults: summary_frequency 10, end_time 10.0
            freq = d.get("summary_frequency", 10)
            if freq and self.step_no % freq == 0:
                self.summary()
            if (self.time + H.G_SMALL > d.get("end_time", 10.0)
                    or self.step_no >= d.get("end_step", 2 ** 31 - 1)):
                self.summary()
                return self.step_no

    def field(self, name):
        """The field on the bricks' own cells / nodes / faces in the deck's
        reference layout (the deck's halo left zero)."""
        d = self.d
        shape = O.shape(O.FIELD_KIND[name], d["x_cells"], d["y_cells"], d["z_cells"])
        g = np.zeros(shape, order="F")
        extra = [shape[a] - (m + 4) for a, m in enumerate((d["x_cells"], d["y_cells"], d["z_cells"]))]
        for h, e in zip(self.h, self.ext):
            b = h.a[name]
            src, dst = [], []
            for a in range(3):
                nb = e[2 * a + 1] - e[2 * a] + 1 + extra[a]
                src.append(slice(2, 2 + nb))
                dst.append(slice(e[2 * a] + 1, e[2 * a] + 1 + nb))
            g[tuple(dst)] = b[tuple(src)]
        return g
