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
