"""B200-native CloverLeaf3D hydro cycle.

Python bindings (ctypes) of libclover_b200.so:

* ``Deck``      -- the *clover input deck (parse.f90 / read_input.f90 keys and
                   defaults), parsed by the library's own reader.
* ``Chunk``     -- a chunk resident in HBM, stepped on the device from CUDA
                   graphs (FP64, or FP32 storage with FP64 where conservation
                   needs it).
* ``Ensemble``  -- many independent decks of any sizes advanced together,
                   each with its own dt, every kernel of the step launched
                   once over all decks (autotuned schedules, CUDA graphs).
* ``draw_decks`` -- seeded ensemble decks: the two-state shock problem with
                   drawn sizes, region and densities/energies.
* ``DropIn``    -- the reference's control flow driving the drop-in C ABI
                   (include/clover_kernels.h) with host arrays.
* ``abi``       -- the raw ctypes handle of the drop-in entry points.

The library is built in-tree (``cloverleaf3d_ref_b200/libclover_b200.so``,
``build()``); importing this package never builds or falls back: a missing
library raises.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclover_b200.so")
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)

MAX_STATES = 16
PRECISION_FP64 = 0
PRECISION_MIXED = 1

# reference field ids, data.f90:55-74
FIELD_IDS = {
    "density0": 1, "density1": 2, "energy0": 3, "energy1": 4, "pressure": 5,
    "viscosity": 6, "soundspeed": 7, "xvel0": 8, "xvel1": 9, "yvel0": 10,
    "yvel1": 11, "zvel0": 12, "zvel1": 13, "vol_flux_x": 14, "vol_flux_y": 15,
    "vol_flux_z": 16, "mass_flux_x": 17, "mass_flux_y": 18, "mass_flux_z": 19,
}
FIELD_NAMES = sorted(FIELD_IDS, key=FIELD_IDS.get)

STATUS_BITS = {
    0x1: "cuda_error", 0x2: "bounds", 0x4: "small_dt", 0x8: "no_device",
    0x10: "bad_arg", 0x20: "timeout",
}


def field_shape(name, nx, ny, nz):
    """Fortran-order shape of a reference array (build_field.f90:41-146)."""
    fid = FIELD_IDS[name]
    if fid <= 7:
        return (nx + 4, ny + 4, nz + 4)
    if fid <= 13:
        return (nx + 5, ny + 5, nz + 5)
    if fid in (14, 17):
        return (nx + 5, ny + 4, nz + 4)
    if fid in (15, 18):
        return (nx + 4, ny + 5, nz + 4)
    return (nx + 4, ny + 4, nz + 5)


def build(verbose=False):
    """Compile the CUDA library for sm_100a in-tree."""
    out = None if verbose else subprocess.DEVNULL
    subprocess.check_call(["make", "-s", "-C", CSRC, "-j4"], stdout=out)


class CloverError(RuntimeError):
    pass


_LIB = None


def lib():
    """The loaded libclover_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise CloverError(
                "libclover_b200.so is not built; run cloverleaf3d_ref_b200.build()")
        _LIB = ctypes.CDLL(LIB_PATH)
        _declare(_LIB)
    return _LIB


abi = None  # set by _declare


class DeckStruct(ctypes.Structure):
    _fields_ = [
        ("x_cells", ctypes.c_int), ("y_cells", ctypes.c_int), ("z_cells", ctypes.c_int),
        ("xmin", ctypes.c_double), ("ymin", ctypes.c_double), ("zmin", ctypes.c_double),
        ("xmax", ctypes.c_double), ("ymax", ctypes.c_double), ("zmax", ctypes.c_double),
        ("initial_timestep", ctypes.c_double), ("max_timestep", ctypes.c_double),
        ("timestep_rise", ctypes.c_double), ("end_time", ctypes.c_double),
        ("dtmin", ctypes.c_double), ("dtc_safe", ctypes.c_double),
        ("dtu_safe", ctypes.c_double), ("dtv_safe", ctypes.c_double),
        ("dtw_safe", ctypes.c_double), ("dtdiv_safe", ctypes.c_double),
        ("end_step", ctypes.c_int), ("summary_frequency", ctypes.c_int),
        ("visit_frequency", ctypes.c_int), ("tiles_per_chunk", ctypes.c_int),
        ("test_problem", ctypes.c_int), ("profiler_on", ctypes.c_int),
        ("number_of_states", ctypes.c_int),
        ("state_defined", ctypes.c_int * MAX_STATES),
        ("state_density", ctypes.c_double * MAX_STATES),
        ("state_energy", ctypes.c_double * MAX_STATES),
        ("state_xvel", ctypes.c_double * MAX_STATES),
        ("state_yvel", ctypes.c_double * MAX_STATES),
        ("state_zvel", ctypes.c_double * MAX_STATES),
        ("state_xmin", ctypes.c_double * MAX_STATES),
        ("state_xmax", ctypes.c_double * MAX_STATES),
        ("state_ymin", ctypes.c_double * MAX_STATES),
        ("state_ymax", ctypes.c_double * MAX_STATES),
        ("state_zmin", ctypes.c_double * MAX_STATES),
        ("state_zmax", ctypes.c_double * MAX_STATES),
        ("state_radius", ctypes.c_double * MAX_STATES),
        ("state_geometry", ctypes.c_int * MAX_STATES),
    ]


def _declare(L):
    global abi
    P = ctypes.c_void_p
    L.clover_deck_parse.argtypes = [ctypes.c_char_p, P, ctypes.c_char_p, ctypes.c_int]
    L.clover_deck_parse.restype = ctypes.c_int
    L.clover_deck_defaults.argtypes = [P]
    L.clover_chunk_create.argtypes = [P, ctypes.c_int]
    L.clover_chunk_create.restype = P
    L.clover_last_error.restype = ctypes.c_char_p
    L.clover_chunk_destroy.argtypes = [P]
    for n in ("clover_chunk_step",):
        getattr(L, n).argtypes = [P, ctypes.c_int]
        getattr(L, n).restype = ctypes.c_int
    for n in ("clover_chunk_run", "clover_chunk_sync", "clover_chunk_steps",
              "clover_chunk_status", "clover_chunk_launches_per_step"):
        getattr(L, n).argtypes = [P]
        getattr(L, n).restype = ctypes.c_int
    L.clover_chunk_use_graphs.argtypes = [P, ctypes.c_int]
    L.clover_chunk_use_fused.argtypes = [P, ctypes.c_int]
    L.clover_chunk_use_tma.argtypes = [P, ctypes.c_int]
    L.clover_chunk_use_tma.restype = ctypes.c_int
    L.clover_chunk_time.argtypes = [P]
    L.clover_chunk_time.restype = ctypes.c_double
    L.clover_chunk_dt_history.argtypes = [P, P, ctypes.c_int]
    L.clover_chunk_dt_history.restype = ctypes.c_int
    L.clover_chunk_summaries.argtypes = [P, P, P, ctypes.c_int]
    L.clover_chunk_summaries.restype = ctypes.c_int
    L.clover_chunk_read_field.argtypes = [P, ctypes.c_int, P]
    L.clover_chunk_read_field.restype = ctypes.c_int
    L.clover_chunk_write_field.argtypes = [P, ctypes.c_int, P]
    L.clover_chunk_write_field.restype = ctypes.c_int
    L.clover_chunk_stream.argtypes = [P]
    L.clover_chunk_stream.restype = ctypes.c_size_t
    L.clover_chunk_device_bytes.argtypes = [P]
    L.clover_chunk_device_bytes.restype = ctypes.c_longlong
    L.clover_chunk_set_visit_dir.argtypes = [P, ctypes.c_char_p]
    L.clover_chunk_set_visit_dir.restype = ctypes.c_int
    L.clover_chunk_visit.argtypes = [P]
    L.clover_chunk_visit.restype = ctypes.c_int
    L.clover_format_e12_4.argtypes = [ctypes.c_double, ctypes.c_char_p]
    L.clover_chunk_checkpoint.argtypes = [P, ctypes.c_char_p]
    L.clover_chunk_checkpoint.restype = ctypes.c_int
    L.clover_chunk_restore.argtypes = [P, ctypes.c_char_p]
    L.clover_chunk_restore.restype = ctypes.c_int
    L.clover_chunk_profile.argtypes = [P, ctypes.c_int]
    L.clover_chunk_profile_report.argtypes = [P, P, ctypes.c_int, P, P, P, ctypes.c_int]
    L.clover_chunk_profile_report.restype = ctypes.c_int
    L.clover_ensemble_create.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.clover_ensemble_create.restype = P
    for n in ("clover_ensemble_decks", "clover_ensemble_reset"):
        getattr(L, n).argtypes = [P]
        getattr(L, n).restype = ctypes.c_int
    L.clover_ensemble_autotune.argtypes = [P, ctypes.c_int]
    L.clover_ensemble_autotune.restype = ctypes.c_int
    L.clover_ensemble_set_schedule.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.clover_ensemble_set_schedule.restype = ctypes.c_int
    L.clover_ensemble_schedule.argtypes = [P, ctypes.c_char_p, ctypes.c_int]
    L.clover_ensemble_schedule.restype = ctypes.c_int
    L.clover_ensemble_status.argtypes = [P, ctypes.c_int]
    L.clover_ensemble_status.restype = ctypes.c_int
    L.clover_ensemble_time.argtypes = [P, ctypes.c_int]
    L.clover_ensemble_time.restype = ctypes.c_double
    L.clover_ensemble_dt_history.argtypes = [P, ctypes.c_int, P, ctypes.c_int]
    L.clover_ensemble_dt_history.restype = ctypes.c_int
    L.clover_ensemble_summaries.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int]
    L.clover_ensemble_summaries.restype = ctypes.c_int
    L.clover_ensemble_read_field.argtypes = [P, ctypes.c_int, ctypes.c_int, P]
    L.clover_ensemble_read_field.restype = ctypes.c_int
    L.clover_dropin_create.argtypes = [P]
    L.clover_dropin_create.restype = P
    L.clover_dropin_run.argtypes = [P, ctypes.c_int]
    L.clover_dropin_run.restype = ctypes.c_int
    L.clover_dropin_dt_history.argtypes = [P, P, ctypes.c_int]
    L.clover_dropin_dt_history.restype = ctypes.c_int
    L.clover_dropin_summaries.argtypes = [P, P, P, ctypes.c_int]
    L.clover_dropin_summaries.restype = ctypes.c_int
    L.clover_dropin_read_field.argtypes = [P, ctypes.c_int, P, ctypes.c_longlong]
    L.clover_dropin_read_field.restype = ctypes.c_int
    L.clover_dropin_destroy.argtypes = [P]
    I = ctypes.c_int
    L.clover_decompose.argtypes = [I, I, I, I, P, P, P]
    L.clover_decompose.restype = I
    L.clover_bricks_create.argtypes = [P, I]
    L.clover_bricks_create.restype = P
    L.clover_bricks_run.argtypes = [P, I]
    L.clover_bricks_run.restype = I
    L.clover_bricks_count.argtypes = [P, P]
    L.clover_bricks_count.restype = I
    L.clover_bricks_extent.argtypes = [P, I, P, P]
    L.clover_bricks_extent.restype = I
    L.clover_bricks_dt_history.argtypes = [P, P, I]
    L.clover_bricks_dt_history.restype = I
    L.clover_bricks_summaries.argtypes = [P, P, P, I]
    L.clover_bricks_summaries.restype = I
    L.clover_bricks_read_field.argtypes = [P, I, I, P, ctypes.c_longlong]
    L.clover_bricks_read_field.restype = I
    L.clover_bricks_destroy.argtypes = [P]
    L.clover_gpu_face_copy.argtypes = [P, P, P, P, I, I, I]
    L.clover_bricks_create_rank.argtypes = [P, I, I, P]
    L.clover_bricks_create_rank.restype = P
    L.clover_gpu_message_len.argtypes = [P, I, I, I]
    L.clover_gpu_message_len.restype = ctypes.c_longlong
    L.clover_gpu_pack_device.argtypes = [P, P, I, I, I, P, I]
    L.clover_gpu_pack_device.restype = I
    L.clover_gpu_status.restype = ctypes.c_int
    L.clover_gpu_error_string.restype = ctypes.c_char_p
    L.clover_gpu_invalidate.argtypes = [P]
    L.clover_gpu_invalidate_all.argtypes = []
    L.clover_gpu_use_staging.argtypes = [ctypes.c_int]
    abi = L


class Deck:
    """A parsed *clover deck. Construct from text, a file, or keyword values
    (``Deck.from_values(x_cells=32, ...,
    states=[dict(density=0.2, energy=1.0), dict(...)])``)."""

    def __init__(self, struct):
        self.s = struct

    @classmethod
    def parse(cls, text):
        s = DeckStruct()
        err = ctypes.create_string_buffer(256)
        rc = lib().clover_deck_parse(text.encode(), ctypes.byref(s), err, 256)
        if rc != 0:
            raise CloverError("deck: " + err.value.decode())
        return cls(s)

    @classmethod
    def from_file(cls, path):
        with open(path) as f:
            return cls.parse(f.read())

    @classmethod
    def from_values(cls, states, **kw):
        s = DeckStruct()
        lib().clover_deck_defaults(ctypes.byref(s))
        for k, v in kw.items():
            if not hasattr(s, k):
                raise CloverError("deck: unknown key %s" % k)
            setattr(s, k, v)
        if not 1 <= len(states) <= MAX_STATES:
            raise CloverError("deck: 1..16 states")
        s.number_of_states = len(states)
        geo = {"cuboid": 1, "sphere": 2, "point": 3}
        for i, st in enumerate(states):
            s.state_defined[i] = 1
            for k, v in st.items():
                if k == "geometry":
                    s.state_geometry[i] = geo[v]
                else:
                    getattr(s, "state_" + k)[i] = v
        return cls(s)

    def __getattr__(self, k):
        return getattr(self.s, k)

    def replace(self, **kw):
        s = DeckStruct.from_buffer_copy(self.s)
        for k, v in kw.items():
            setattr(s, k, v)
        return Deck(s)

    @property
    def cells(self):
        return self.s.x_cells * self.s.y_cells * self.s.z_cells


class Chunk:
    """A chunk resident on the current CUDA device (native API)."""

    def __init__(self, deck, precision=PRECISION_FP64):
        L = lib()
        self.deck = deck
        self.precision = precision
        self.h = L.clover_chunk_create(ctypes.byref(deck.s), precision)
        if not self.h:
            raise CloverError("chunk: " + L.clover_last_error().decode())

    def close(self):
        if self.h:
            lib().clover_chunk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n):
        if lib().clover_chunk_step(self.h, n) != 0:
            raise CloverError("chunk step failed")

    def run(self):
        return lib().clover_chunk_run(self.h)

    def sync(self):
        if lib().clover_chunk_sync(self.h) != 0:
            raise CloverError("chunk sync failed")

    def use_graphs(self, on):
        lib().clover_chunk_use_graphs(self.h, 1 if on else 0)

    def use_fused(self, on):
        """Fused kernels (default) or one kernel per reference loop nest; only
        before the first step."""
        lib().clover_chunk_use_fused(self.h, 1 if on else 0)

    def use_tma(self, on):
        """The fused step's stencils staged by bulk-tensor copies (default, one
        chunk) or their register-marching forms; True if the staged forms are
        in use."""
        return lib().clover_chunk_use_tma(self.h, 1 if on else 0) == 1

    @property
    def steps(self):
        return lib().clover_chunk_steps(self.h)

    @property
    def time(self):
        return lib().clover_chunk_time(self.h)

    @property
    def status(self):
        return lib().clover_chunk_status(self.h)

    @property
    def stream(self):
        return lib().clover_chunk_stream(self.h)

    @property
    def device_bytes(self):
        return lib().clover_chunk_device_bytes(self.h)

    @property
    def launches_per_step(self):
        return lib().clover_chunk_launches_per_step(self.h)

    def profile(self, on):
        """Profile mode: direct launches bracketed by events per kernel group."""
        lib().clover_chunk_profile(self.h, 1 if on else 0)

    def profile_report(self, cap=64):
        """Per kernel group since the last report: ms, algorithmic bytes, launches."""
        names = ctypes.create_string_buffer(cap * 32)
        ms = np.zeros(cap)
        by = np.zeros(cap)
        la = np.zeros(cap, dtype=np.int32)
        n = lib().clover_chunk_profile_report(self.h, names, 32, ms.ctypes.data,
                                              by.ctypes.data, la.ctypes.data, cap)
        raw = names.raw
        out = []
        for i in range(n):
            nm = raw[i * 32:(i + 1) * 32].split(b"\0")[0].decode()
            out.append({"name": nm, "ms": float(ms[i]), "bytes": float(by[i]),
                        "launches": int(la[i])})
        return out

    def dt_history(self):
        n = self.steps
        out = np.zeros(max(n, 1))
        got = lib().clover_chunk_dt_history(self.h, out.ctypes.data, n)
        return out[:got]

    def summaries(self, cap=100000):
        out = np.zeros((cap, 5))
        st = np.zeros(cap, dtype=np.int32)
        n = lib().clover_chunk_summaries(self.h, out.ctypes.data, st.ctypes.data, cap)
        return out[:n], st[:n]

    def field(self, name):
        s = self.deck.s
        a = np.zeros(field_shape(name, s.x_cells, s.y_cells, s.z_cells), order="F")
        if lib().clover_chunk_read_field(self.h, FIELD_IDS[name], a.ctypes.data) != 0:
            raise CloverError("read_field failed")
        return a

    def set_visit_dir(self, path):
        """Directory of the VTK output (clover.visit and clover.*.vtk)."""
        lib().clover_chunk_set_visit_dir(self.h, os.fsencode(path))

    def visit(self):
        """Write the current step as VTK (visit.f90) and wait for the file."""
        if lib().clover_chunk_visit(self.h) != 0:
            raise CloverError("visit failed: " + lib().clover_last_error().decode())

    def checkpoint(self, path):
        """Write the whole device state (every array, dt/time/step, the dt and
        summary histories) to path."""
        rc = lib().clover_chunk_checkpoint(self.h, os.fsencode(path))
        if rc != 0:
            raise CloverError("checkpoint failed (%d)" % rc)

    def restore(self, path):
        """Replace the device state by a checkpoint of a chunk made from the
        same deck(s) and precision; stepping on continues bit for bit."""
        rc = lib().clover_chunk_restore(self.h, os.fsencode(path))
        if rc != 0:
            raise CloverError("restore failed (%d): %s" % (rc, lib().clover_last_error().decode()))

    def dump_fields(self, path):
        """Every field in the reference layout (FP64, Fortran order) to an .npz."""
        np.savez(path, **{n: self.field(n) for n in FIELD_NAMES})

    def write_summary_log(self, path):
        """The recorded field summaries, one line per summary step, %.17g."""
        sums, steps = self.summaries()
        with open(path, "w") as f:
            f.write("step vol mass ie ke press\n")
            for st, row in zip(steps, sums):
                f.write("%d %s\n" % (st, " ".join("%.17g" % x for x in row)))

    def set_field(self, name, a):
        s = self.deck.s
        a = np.asfortranarray(a, dtype=np.float64)
        assert a.shape == field_shape(name, s.x_cells, s.y_cells, s.z_cells)
        if lib().clover_chunk_write_field(self.h, FIELD_IDS[name], a.ctypes.data) != 0:
            raise CloverError("write_field failed")


class Ensemble(Chunk):
    """Independent decks advanced together on the current CUDA device.

    Every deck keeps its own dt, time and calc_dt reduction; the decks share
    end_step, summary_frequency and calc_dt's safety factors. ``step``,
    ``run``, ``sync``, ``profile`` and ``use_graphs`` act on all decks; the
    per-deck results take a deck index."""

    def __init__(self, decks, precision=PRECISION_FP64):
        L = lib()
        self.decks = list(decks)
        self.deck = self.decks[0]
        self.precision = precision
        arr = (DeckStruct * len(self.decks))(*[d.s for d in self.decks])
        self._arr = arr
        self.h = L.clover_ensemble_create(ctypes.cast(arr, ctypes.c_void_p), len(self.decks),
                                          precision)
        if not self.h:
            raise CloverError("ensemble: " + L.clover_last_error().decode())

    def __len__(self):
        return len(self.decks)

    @property
    def cells(self):
        return sum(d.cells for d in self.decks)

    def autotune(self, trial_steps=2):
        """Pick each batched launch's schedule by timing candidates; the
        decks are set back to step 0 afterwards."""
        n = lib().clover_ensemble_autotune(self.h, trial_steps)
        if n < 0:
            raise CloverError("ensemble autotune failed")
        return n

    def reset(self):
        if lib().clover_ensemble_reset(self.h) != 0:
            raise CloverError("ensemble reset failed")

    def set_schedule(self, order=0, grid_div=1, seg=0):
        """One schedule for every batched launch (replaces tuned ones)."""
        if lib().clover_ensemble_set_schedule(self.h, order, grid_div, seg) != 0:
            raise CloverError("bad schedule")

    def schedule(self):
        """The schedule in use: one dict per batched launch."""
        n = lib().clover_ensemble_schedule(self.h, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        lib().clover_ensemble_schedule(self.h, buf, n + 1)
        out = []
        for line in buf.value.decode().splitlines():
            key, order, div, seg, blocks, items = (int(x) for x in line.split())
            out.append({"key": key, "order": order, "grid_div": div, "seg": seg,
                        "blocks": blocks, "items": items})
        return out

    def deck_status(self, d):
        return lib().clover_ensemble_status(self.h, d)

    def deck_time(self, d):
        return lib().clover_ensemble_time(self.h, d)

    def deck_dt_history(self, d):
        n = self.steps
        out = np.zeros(max(n, 1))
        got = lib().clover_ensemble_dt_history(self.h, d, out.ctypes.data, n)
        if got < 0:
            raise CloverError("bad deck index")
        return out[:got]

    def deck_summaries(self, d, cap=100000):
        out = np.zeros((cap, 5))
        st = np.zeros(cap, dtype=np.int32)
        n = lib().clover_ensemble_summaries(self.h, d, out.ctypes.data, st.ctypes.data, cap)
        if n < 0:
            raise CloverError("bad deck index")
        return out[:n], st[:n]

    def deck_field(self, d, name):
        s = self.decks[d].s
        a = np.zeros(field_shape(name, s.x_cells, s.y_cells, s.z_cells), order="F")
        if lib().clover_ensemble_read_field(self.h, d, FIELD_IDS[name], a.ctypes.data) != 0:
            raise CloverError("read_field failed")
        return a

    def field(self, name):
        return self.deck_field(0, name)

    def dump_fields(self, path, deck=0):
        np.savez(path, **{n: self.deck_field(deck, n) for n in FIELD_NAMES})

    def write_summary_log(self, path, deck=0):
        sums, steps = self.deck_summaries(deck)
        with open(path, "w") as f:
            f.write("step vol mass ie ke press\n")
            for st, row in zip(steps, sums):
                f.write("%d %s\n" % (st, " ".join("%.17g" % x for x in row)))

    def set_field(self, name, a):
        raise CloverError("ensembles are set up from their decks only")


def format_e12_4(v):
    """A value as the reference's VTK files print it (Fortran E12.4)."""
    out = ctypes.create_string_buffer(13)
    lib().clover_format_e12_4(float(v), out)
    return out.value.decode()


def draw_decks(n, seed, cells=(24, 128), end_step=150, summary_frequency=10):
    """Seeded ensemble decks of the two-state shock problem on [0,10]^3.

    Per deck: cells per axis uniform in cells (inclusive, independent per
    axis); a high-state cuboid [0,u]x[0,v]x[0,w] with u, v, w uniform in
    [1,6]; background density lognormal(ln 0.2, 0.3), region density
    lognormal(ln 1.0, 0.3), both energies uniform in [0.5, 3.0]; zero
    velocity; dt 0.04 initial and maximum, rise 1.5; end_time far beyond
    end_step * 0.04 so that every deck runs end_step steps."""
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = cells
    for _ in range(n):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, size=3))
        u, v, w = (float(x) for x in rng.uniform(1.0, 6.0, size=3))
        rho_bg = float(rng.lognormal(np.log(0.2), 0.3))
        rho_hi = float(rng.lognormal(np.log(1.0), 0.3))
        e_bg, e_hi = (float(x) for x in rng.uniform(0.5, 3.0, size=2))
        out.append(Deck.from_values(
            [dict(density=rho_bg, energy=e_bg),
             dict(density=rho_hi, energy=e_hi, geometry="cuboid", xmin=0.0, xmax=u,
                  ymin=0.0, ymax=v, zmin=0.0, zmax=w)],
            x_cells=nx, y_cells=ny, z_cells=nz, xmin=0.0, xmax=10.0, ymin=0.0, ymax=10.0,
            zmin=0.0, zmax=10.0, initial_timestep=0.04, timestep_rise=1.5, max_timestep=0.04,
            end_step=end_step, end_time=1.0e6, summary_frequency=summary_frequency))
    return out


def decompose(x_cells, y_cells, z_cells, n_chunks):
    """clover_decompose (clover.f90:108-256): the chunk grid (3,), each chunk's
    global cell range (n, 6: left, right, bottom, top, back, front) and its
    neighbours (n, 6; chunk ids from 1, -1 for an external face). Host only."""
    grid = np.zeros(3, dtype=np.int32)
    ext = np.zeros((n_chunks, 6), dtype=np.int32)
    nbr = np.zeros((n_chunks, 6), dtype=np.int32)
    rc = lib().clover_decompose(x_cells, y_cells, z_cells, n_chunks, grid.ctypes.data,
                                ext.ctypes.data, nbr.ctypes.data)
    if rc != 0:
        raise CloverError("cannot decompose %dx%dx%d cells into %d chunks"
                          % (x_cells, y_cells, z_cells, n_chunks))
    return grid, ext, nbr


class Bricks:
    """One deck decomposed into n bricks (``decompose``) and run by the
    reference's decomposed control flow in this process: the drop-in driver's
    calls on every brick, halo messages exchanged between the bricks on the
    device before each update_halo's reflective faces, dt the minimum over the
    bricks, the summaries their sum."""

    def __init__(self, deck, n_chunks):
        L = lib()
        L.clover_gpu_clear_status()
        self.deck = deck
        self.h = L.clover_bricks_create(ctypes.byref(deck.s), n_chunks)
        if not self.h:
            raise CloverError("bricks start failed: " + L.clover_gpu_error_string().decode())
        grid = np.zeros(3, dtype=np.int32)
        self.n = L.clover_bricks_count(self.h, grid.ctypes.data)
        self.grid = tuple(int(v) for v in grid)
        self.extents, self.neighbours = [], []
        for i in range(self.n):
            e = np.zeros(6, dtype=np.int32)
            nb = np.zeros(6, dtype=np.int32)
            L.clover_bricks_extent(self.h, i, e.ctypes.data, nb.ctypes.data)
            self.extents.append(tuple(int(v) for v in e))
            self.neighbours.append(tuple(int(v) for v in nb))

    def run(self, max_steps=2 ** 30):
        n = lib().clover_bricks_run(self.h, max_steps)
        st = lib().clover_gpu_status()
        if st & ~0x4:
            raise CloverError("bricks: " + lib().clover_gpu_error_string().decode())
        return n

    def dt_history(self, cap=1 << 20):
        out = np.zeros(cap)
        n = lib().clover_bricks_dt_history(self.h, out.ctypes.data, cap)
        return out[:n]

    def summaries(self, cap=100000):
        out = np.zeros((cap, 5))
        st = np.zeros(cap, dtype=np.int32)
        n = lib().clover_bricks_summaries(self.h, out.ctypes.data, st.ctypes.data, cap)
        return out[:n], st[:n]

    def brick_field(self, i, name):
        """Field `name` of brick i in its own reference layout."""
        e = self.extents[i]
        a = np.zeros(field_shape(name, e[1] - e[0] + 1, e[3] - e[2] + 1, e[5] - e[4] + 1),
                     order="F")
        if lib().clover_bricks_read_field(self.h, i, FIELD_IDS[name], a.ctypes.data, a.size) != 0:
            raise CloverError("bricks read_field failed")
        return a

    def field(self, name):
        """Field `name` of the whole deck in the reference layout: each
        brick's own cells (and nodes / faces up to its upper boundary) at its
        global place; the halo of the deck left zero."""
        s = self.deck.s
        g = np.zeros(field_shape(name, s.x_cells, s.y_cells, s.z_cells), order="F")
        extra = [g.shape[a] - (n + 4) for a, n in enumerate((s.x_cells, s.y_cells, s.z_cells))]
        for i, e in enumerate(self.extents):
            b = self.brick_field(i, name)
            src, dst = [], []
            for a in range(3):
                n_b = e[2 * a + 1] - e[2 * a] + 1 + extra[a]
                src.append(slice(2, 2 + n_b))  # local index 1.. (array index = index + 1)
                dst.append(slice(e[2 * a] + 1, e[2 * a] + 1 + n_b))
            g[tuple(dst)] = b[tuple(src)]
        return g

    def close(self):
        if self.h:
            lib().clover_bricks_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DropIn:
    """The reference control flow over the drop-in ABI with host arrays."""

    def __init__(self, deck):
        L = lib()
        L.clover_gpu_clear_status()
        self.deck = deck
        self.h = L.clover_dropin_create(ctypes.byref(deck.s))
        if not self.h:
            raise CloverError("drop-in start failed: " + L.clover_gpu_error_string().decode())

    def run(self, max_steps=2 ** 30):
        n = lib().clover_dropin_run(self.h, max_steps)
        st = lib().clover_gpu_status()
        if st & ~0x4:
            raise CloverError("drop-in: " + lib().clover_gpu_error_string().decode())
        return n

    def dt_history(self, cap=1 << 20):
        out = np.zeros(cap)
        n = lib().clover_dropin_dt_history(self.h, out.ctypes.data, cap)
        return out[:n]

    def summaries(self, cap=100000):
        out = np.zeros((cap, 5))
        st = np.zeros(cap, dtype=np.int32)
        n = lib().clover_dropin_summaries(self.h, out.ctypes.data, st.ctypes.data, cap)
        return out[:n], st[:n]

    def field(self, name):
        s = self.deck.s
        a = np.zeros(field_shape(name, s.x_cells, s.y_cells, s.z_cells), order="F")
        if lib().clover_dropin_read_field(self.h, FIELD_IDS[name], a.ctypes.data, a.size) != 0:
            raise CloverError("drop-in read_field failed")
        return a

    def close(self):
        if self.h:
            lib().clover_dropin_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
