"""Mixed precision on the condensed HDG solve: an FP32 inner GMRES with FP32
block-Jacobi and an FP32 copy of X (k <= 3) or of the 16 Schur panels C_s X_o
per cell (k >= 4), inside FP64 iterative refinement that stops at the FP64
solver's own relative residual (1e-12 here).

Because every linear solve still meets the reference's residual bound, the
results are checked against the reference's FP64 outputs: the Schur solution
to 1e-9 relative, end-to-end final states to 1e-8 and L2 errors to 1e-6
relative (the acceptance bar for this mode is 1% of the FP64 error).
"""
import json
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, manifest, rel_err, unit_files
from mfem_euler2d_cpp_b200 import capi

pytestmark = pytest.mark.gpu
CLI = ROOT / "mfem_euler2d_cpp_b200" / "bin" / "euler2d"


@pytest.fixture(params=unit_files(), ids=lambda p: p.stem)
def unit(request):
    return np.load(request.param)


def test_mixed_schur_solve_meets_fp64_bound(unit):
    f = unit
    d = capi.simple_wave_desc(int(f["nx"]), int(f["ny"]), int(f["k"]), float(f["alpha"]))
    opts = capi.default_opts(form=capi.FORM_HDG, precision=capi.PRECISION_MIXED)
    with capi.Context(d, opts) as ctx:
        ctx.upload("U", f["u"])
        ctx.freeze(float(f["dt"]), check_admissible=True)
        ctx.upload("OLD", f["old"])
        ctx.set_dt(float(f["dt"]))
        ctx.upload("R", f["r"])
        ctx.condense()
        x, eq, st = ctx.linear_solve(f["rhs"])
        assert st.residual <= 1e-11
        assert rel_err(x, f["solve_hdg_x"]) < 1e-9
        # a warm-started refinement keeps the FP32 copies of the first solve
        x2, _, st2 = ctx.linear_solve(f["rhs"], x0=x, refresh=False, linear_tol=1e-13)
        assert st2.residual <= 1e-12


def test_mixed_cli_matches_reference(tmp_path):
    f = np.load(GOLDEN / "cli_c1_16x16_q3.npz")
    args = json.loads(str(f["args"])) + ["--precision", "mixed"]
    prefix = tmp_path / "run"
    proc = subprocess.run([str(CLI), *args, "--output", str(prefix)], capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr
    scol = manifest()["summary_columns"]
    for form, tol in (("dg", 1e-10), ("hdg", 1e-8)):  # mixed precision applies to the condensed form
        coeff = np.loadtxt(f"{prefix}_{form}_coefficients.csv", delimiter=",", skiprows=1)
        assert rel_err(coeff[:, 2:].reshape(-1), f[f"{form}_u"]) < tol
        import csv
        with open(f"{prefix}_{form}_summary.csv", newline="") as fh:
            row = next(csv.DictReader(fh))
        for name in ("rho_L2", "rhou_L2", "rhov_L2", "energy_L2"):
            ref = f[f"{form}_summary"][scol.index(name)]
            assert abs(float(row[name]) - ref) <= 1e-6 * ref
        assert row["precision"] == "mixed"


@pytest.mark.parametrize("n,k", [(48, 3), (32, 4)], ids=["48x48_k3_X", "32x32_k4_panels"])
def test_mixed_matches_fp64_on_a_larger_mesh(n, k):
    """One SSP-DIRK3 step with 3 updates per stage: mixed against the FP64
    engine on the same schedule (k = 3 streams X, k = 4 the Schur panels)."""
    out = {}
    for prec in (capi.PRECISION_FP64, capi.PRECISION_MIXED):
        d = capi.simple_wave_desc(n, n, k, 40.0)
        with capi.Context(d, capi.default_opts(form=capi.FORM_HDG, precision=prec)) as ctx:
            ro, keep = capi.run_options(integrator="ssp-dirk3", steps=1, newton_steps=3, cfl=1.0,
                                        form_name="hdg", precond_name="block-jacobi")
            st = capi.Stepper(ctx, ro, keep)
            while st.next() is not None:
                pass
            st.close()
            out[prec] = ctx.download("U")
    assert rel_err(out[capi.PRECISION_MIXED], out[capi.PRECISION_FP64]) < 1e-9
