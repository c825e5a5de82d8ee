"""Device-side initial projection and diagnostics against the reference:
Problem::Initial (the u0 the reference's own code projected, every unit
fixture, k = 0..8), Problem::Errors (the L2 errors the reference's command
line reported for its final states, at their final time), Problem::Integral
and Problem::Differences (against the host restatement kept as the checker:
eg_differences and the collocated weights of the descriptor).

Tolerances: the projection 1e-13 relative (the exact wave's sin/cos/pow on the
device round differently from the host's libm, by an ulp or two); errors 1e-8
relative (an error of 1e-7 of the state moves by ~1e-9 of itself when the
exact wave it subtracts moves by an ulp); integrals 1e-13; differences 1e-11.
"""
import ctypes as C
import json

import numpy as np
import pytest

from conftest import cli_files, manifest, rel_err, unit_files
from mfem_euler2d_cpp_b200 import capi

pytestmark = pytest.mark.gpu
_DP = C.POINTER(C.c_double)


def _opt(args, flag, default):
    return type(default)(args[args.index(flag) + 1]) if flag in args else default


@pytest.mark.parametrize("path", unit_files(), ids=lambda p: p.stem)
def test_initial_projection_matches_reference(path):
    f = np.load(path)
    d = capi.simple_wave_desc(int(f["nx"]), int(f["ny"]), int(f["k"]), float(f["alpha"]))
    with capi.Context(d, capi.default_opts()) as ctx:
        ctx.initial()
        assert rel_err(ctx.download("U"), f["u0"]) < 1e-13


@pytest.mark.parametrize("path", cli_files(), ids=lambda p: p.stem)
def test_errors_integrals_differences_of_reference_final_states(path):
    f = np.load(path)
    args = json.loads(str(f["args"]))
    scol = manifest()["summary_columns"]
    d = capi.simple_wave_desc(_opt(args, "--nx", 100), _opt(args, "--ny", 100), _opt(args, "--k", 1),
                              _opt(args, "--alpha-deg", 45.0))
    lib = capi.load()
    p = (d.k + 1) ** 2
    with capi.Context(d, capi.default_opts()) as ctx:
        for form in ("dg", "hdg"):
            s = dict(zip(scol, f[f"{form}_summary"]))
            u = np.ascontiguousarray(f[f"{form}_u"])
            ctx.upload("U", u)
            err = np.zeros(4)
            ctx._check(lib.eg_errors(ctx.h, float(s["T"]), err.ctypes.data_as(_DP)))
            ref = np.array([s["rho_L2"], s["rhou_L2"], s["rhov_L2"], s["energy_L2"]])
            assert np.max(np.abs(err - ref) / ref) < 1e-8
            integ = np.zeros(4)
            ctx._check(lib.eg_integral(ctx.h, integ.ctypes.data_as(_DP)))
            want = d.area * np.einsum("i,eic->c", np.array(d.w[:p]), u.reshape(-1, p, 4))
            assert np.max(np.abs(integ - want) / np.maximum(np.abs(want), 1e-300)) < 1e-13
        # DG/HDG differences on the device against the host restatement
        u = np.ascontiguousarray(f["dg_u"])
        v = np.ascontiguousarray(f["hdg_u"])
        ctx.upload("U", u)
        dev, host = np.zeros(4), np.zeros(4)
        ctx._check(lib.eg_state_differences(ctx.h, v.ctypes.data_as(_DP), dev.ctypes.data_as(_DP)))
        assert lib.eg_differences(C.byref(d), u.ctypes.data_as(_DP), v.ctypes.data_as(_DP),
                                  host.ctypes.data_as(_DP)) == capi.OK
        assert np.max(np.abs(dev - host) / np.maximum(host, 1e-300)) < 1e-11


def test_errors_outside_the_exact_wave_interval_are_refused():
    d = capi.simple_wave_desc(4, 4, 1, 45.0)
    lib = capi.load()
    with capi.Context(d, capi.default_opts()) as ctx:
        ctx.initial()
        out = np.zeros(4)
        assert lib.eg_errors(ctx.h, 0.5, out.ctypes.data_as(_DP)) == 18
        ctx._check(lib.eg_errors(ctx.h, 0.0, out.ctypes.data_as(_DP)))  # still usable
        assert np.all(np.isfinite(out))
