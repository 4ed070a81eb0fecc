"""The allocation-free field summary (clover_field_summary_kernel_noalloc).

It serves host codes whose device memory all belongs to their own pool
allocator or to a fixed budget: they cannot let the library call cudaMalloc,
so this entry point takes their device arrays and keeps its reduction
scratch in a fixed file-scope device array. Its sums must agree with the
regular entry point (clover_field_summary_kernel, given the same device
arrays in place) to the tolerance of the other parity tests, on two calls in
a row (the second call reuses the scratch the first one left behind).
"""
import ctypes

import numpy as np
import pytest

import cloverleaf3d_ref_b200 as C

pytestmark = pytest.mark.gpu

RTOL = 1e-12
NX, NY, NZ = 37, 29, 23


def _device_array(torch, host, px, pxy, planes):
    """A device copy of a reference-layout (Fortran order) array in the chunk layout."""
    py = pxy // px
    d = torch.zeros(planes * pxy, dtype=torch.float64, device="cuda")
    v = d.view(planes, py, px)
    hx, hy, hz = host.shape
    v[:hz, :hy, :hx] = torch.from_numpy(np.ascontiguousarray(host.transpose(2, 1, 0))).cuda()
    return d


def test_noalloc_field_summary_matches_regular_entry_point():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    L = C.lib()
    L.clover_gpu_release()
    L.clover_gpu_clear_status()
    rng = np.random.default_rng(7)
    b = [ctypes.c_int(v) for v in (1, NX, 1, NY, 1, NZ)]
    B = [ctypes.byref(v) for v in b]
    px, pxy, elems = ctypes.c_int(0), ctypes.c_longlong(0), ctypes.c_longlong(0)
    L.clover_gpu_layout(*B, ctypes.byref(px), ctypes.byref(pxy), ctypes.byref(elems))
    planes = elems.value // pxy.value
    cell = (NX + 4, NY + 4, NZ + 4)
    vert = (NX + 5, NY + 5, NZ + 5)
    host = {
        "volume": rng.uniform(0.5, 1.5, cell), "density0": rng.uniform(0.1, 2.0, cell),
        "energy0": rng.uniform(0.5, 3.0, cell), "pressure": rng.uniform(0.0, 1.0, cell),
        "xvel0": rng.uniform(-1, 1, vert), "yvel0": rng.uniform(-1, 1, vert),
        "zvel0": rng.uniform(-1, 1, vert),
    }
    dev = {k: _device_array(torch, np.asfortranarray(v), px.value, pxy.value, planes)
           for k, v in host.items()}
    torch.cuda.synchronize()
    names = ("volume", "density0", "energy0", "pressure", "xvel0", "yvel0", "zvel0")
    ptrs = [ctypes.c_void_p(dev[k].data_ptr()) for k in names]

    def outs():
        return [ctypes.c_double(0.0) for _ in range(5)]

    ref = outs()
    L.clover_field_summary_kernel(*B, *ptrs, *[ctypes.byref(o) for o in ref])
    assert L.clover_gpu_status() == 0, L.clover_gpu_error_string()
    want = np.array([o.value for o in ref])
    assert np.all(np.isfinite(want)) and want[0] > 0

    L.clover_field_summary_kernel_noalloc.restype = ctypes.c_int
    for _ in range(2):
        got = outs()
        rc = L.clover_field_summary_kernel_noalloc(*B, *ptrs, *[ctypes.byref(o) for o in got])
        assert rc == 0
        np.testing.assert_allclose([o.value for o in got], want, rtol=RTOL, atol=0)

    # too many planes for the fixed scratch: rejected before any launch
    big = [ctypes.c_int(v) for v in (1, NX, 1, NY, 1, 5000)]
    got = outs()
    rc = L.clover_field_summary_kernel_noalloc(*[ctypes.byref(v) for v in big], *ptrs,
                                               *[ctypes.byref(o) for o in got])
    assert rc == 0x10
    # host arrays are rejected: the entry point would need a device copy
    hp = [ctypes.c_void_p(host[k].ctypes.data) for k in names]
    rc = L.clover_field_summary_kernel_noalloc(*B, *hp, *[ctypes.byref(o) for o in got])
    assert rc == 0x10
    L.clover_gpu_release()


def test_noalloc_orders_after_queued_library_kernels():
    """The drop-in entry points queue their kernels and return at once. A
    no-alloc summary called right after in-place clover_ideal_gas_kernel calls
    on the caller's device arrays must read the pressure those calls write
    (it was zero before them): its sums equal the regular entry point's, taken
    afterwards, and the pressure sum is the ideal-gas one, not zero."""
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    L = C.lib()
    L.clover_gpu_release()
    L.clover_gpu_clear_status()
    n = (160, 144, 128)
    b = [ctypes.c_int(v) for v in (1, n[0], 1, n[1], 1, n[2])]
    B = [ctypes.byref(v) for v in b]
    px, pxy, elems = ctypes.c_int(0), ctypes.c_longlong(0), ctypes.c_longlong(0)
    L.clover_gpu_layout(*B, ctypes.byref(px), ctypes.byref(pxy), ctypes.byref(elems))
    planes = elems.value // pxy.value
    rng = np.random.default_rng(3)
    cell = (n[0] + 4, n[1] + 4, n[2] + 4)
    vert = (n[0] + 5, n[1] + 5, n[2] + 5)
    host = {
        "volume": np.full(cell, 0.25), "density0": rng.uniform(0.1, 2.0, cell),
        "energy0": rng.uniform(0.5, 3.0, cell), "pressure": np.zeros(cell),
        "soundspeed": np.zeros(cell), "xvel0": rng.uniform(-1, 1, vert),
        "yvel0": rng.uniform(-1, 1, vert), "zvel0": rng.uniform(-1, 1, vert),
    }
    dev = {k: _device_array(torch, np.asfortranarray(v), px.value, pxy.value, planes)
           for k, v in host.items()}
    torch.cuda.synchronize()
    P = {k: ctypes.c_void_p(v.data_ptr()) for k, v in dev.items()}
    names = ("volume", "density0", "energy0", "pressure", "xvel0", "yvel0", "zvel0")

    def outs():
        return [ctypes.c_double(0.0) for _ in range(5)]

    L.clover_field_summary_kernel_noalloc.restype = ctypes.c_int
    for _ in range(3):  # queued, not waited for
        L.clover_ideal_gas_kernel(*B, P["density0"], P["energy0"], P["pressure"], P["soundspeed"])
    got = outs()
    rc = L.clover_field_summary_kernel_noalloc(*B, *[P[k] for k in names],
                                               *[ctypes.byref(o) for o in got])
    assert rc == 0
    ref = outs()
    L.clover_field_summary_kernel(*B, *[P[k] for k in names], *[ctypes.byref(o) for o in ref])
    assert L.clover_gpu_status() == 0, L.clover_gpu_error_string()
    want = np.array([o.value for o in ref])
    assert want[4] > 0.0
    np.testing.assert_allclose([o.value for o in got], want, rtol=RTOL, atol=0)
    L.clover_gpu_release()
