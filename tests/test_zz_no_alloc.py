"""The allocation-free cell norm (eg_cell_norm_noalloc) against the context
entry point (eg_cell_norm) through the C-ABI.

Callers that may not allocate device memory -- their device memory belongs
to their own allocator or a fixed budget -- use eg_cell_norm_noalloc on
vectors they already hold on the device. Its scratch is a static array
inside the library, so two calls in a row must both agree with eg_cell_norm;
a host pointer must be refused rather than handed to the kernel.
"""
import ctypes as C

import numpy as np
import pytest

from mfem_euler2d_cpp_b200 import capi

pytestmark = pytest.mark.gpu
TOL = 1e-12  # operator tolerance used by the parity tests


def test_noalloc_cell_norm_matches_context_twice():
    import torch

    lib = capi.load()
    desc = capi.simple_wave_desc(16, 16, 3, 45.0)
    rng = np.random.default_rng(7)
    with capi.Context(desc, capi.default_opts()) as ctx:
        for call in range(2):
            v = rng.standard_normal(ctx.nu) * (1.0 + call)
            ctx.upload("R", v)
            expected = ctx.cell_norm("R")
            # device memory owned by the caller's own allocator (here: torch)
            dev = torch.from_numpy(v).to("cuda")
            torch.cuda.synchronize()
            out = C.c_double(-1.0)
            rc = lib.eg_cell_norm_noalloc(C.byref(desc), C.c_void_p(dev.data_ptr()), None, C.byref(out))
            assert rc == capi.OK
            assert abs(out.value - expected) <= TOL * expected


def test_noalloc_cell_norm_rejects_host_pointer():
    lib = capi.load()
    desc = capi.simple_wave_desc(4, 4, 1, 45.0)
    host = np.ones(4 * 4 * 16)
    out = C.c_double(-1.0)
    rc = lib.eg_cell_norm_noalloc(C.byref(desc), C.c_void_p(host.ctypes.data), None, C.byref(out))
    assert rc == 1  # EG_ERR_INVALID
    assert out.value == -1.0


def test_noalloc_cell_norm_rejects_descriptors_the_context_refuses():
    import torch

    lib = capi.load()
    base = capi.simple_wave_desc(4, 4, 1, 45.0)
    dev = torch.ones(4 * 4 * 16, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    swapped = capi.simple_wave_desc(4, 4, 1, 45.0)
    swapped.tensor_node[0], swapped.tensor_node[1] = 1, 0
    flat = capi.simple_wave_desc(4, 4, 1, 45.0)
    flat.area = 0.0
    for d in (swapped, flat):
        out = C.c_double(-1.0)
        assert lib.eg_cell_norm_noalloc(C.byref(d), C.c_void_p(dev.data_ptr()), None, C.byref(out)) == 1
        assert out.value == -1.0
    out = C.c_double(-1.0)
    assert lib.eg_cell_norm_noalloc(C.byref(base), C.c_void_p(dev.data_ptr()), None, C.byref(out)) == capi.OK


def test_noalloc_cell_norm_rejects_memory_of_another_device():
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second visible GPU")
    lib = capi.load()
    desc = capi.simple_wave_desc(4, 4, 1, 45.0)
    other = torch.ones(4 * 4 * 16, dtype=torch.float64, device="cuda:1")
    torch.cuda.synchronize(1)
    assert lib.eg_set_device(0) == capi.OK
    out = C.c_double(-1.0)
    assert lib.eg_cell_norm_noalloc(C.byref(desc), C.c_void_p(other.data_ptr()), None, C.byref(out)) == 1
    assert out.value == -1.0
