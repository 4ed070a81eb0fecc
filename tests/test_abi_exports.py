"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares."""
import os
import re

import cloverleaf3d_ref_b200 as C

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_functions():
    names = set()
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(clover_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    lib = C.lib()
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_kernel_entry_points_present():
    names = declared_functions()
    for k in ("ideal_gas", "viscosity", "calc_dt", "pdv", "revert", "accelerate",
              "flux_calc", "advec_cell", "advec_mom", "reset_field", "field_summary",
              "update_halo", "initialise_chunk", "generate_chunk"):
        assert "clover_%s_kernel" % k in names


def test_status_without_device_is_reported_not_raised():
    lib = C.lib()
    lib.clover_gpu_clear_status()
    # no CUDA device in a CPU-only environment: the call records the error
    import ctypes
    b = [ctypes.byref(ctypes.c_int(v)) for v in (1, 4, 1, 4, 1, 4)]
    import torch
    if torch.cuda.is_available():
        return
    lib.clover_ideal_gas_kernel(*b, None, None, None, None)
    assert lib.clover_gpu_status() & 0x8
    lib.clover_gpu_clear_status()
