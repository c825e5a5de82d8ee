"""Failure paths return the reference's error status without faulting the
GPU: every failure is made on the host side (an inadmissible state, an
iteration limit of one, a final time past the shock) and each call must
return its status while the context stays usable."""
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from mfem_euler2d_cpp_b200 import capi

pytestmark = pytest.mark.gpu
CLI = ROOT / "mfem_euler2d_cpp_b200" / "bin" / "euler2d"


def test_inadmissible_state_is_reported():
    d = capi.simple_wave_desc(4, 4, 2, 45)
    with capi.Context(d, capi.default_opts()) as ctx:
        ctx.initial()
        u = ctx.download("U")
        u[0::4] *= -1.0  # negative density everywhere
        ctx.upload("U", u)
        with pytest.raises(capi.EngineError) as exc:
            ctx.freeze(1e-3, check_admissible=True)
        assert exc.value.status == 6
        # without the admissibility check the HLL speeds reject the faces
        with pytest.raises(capi.EngineError) as exc:
            ctx.freeze(1e-3, check_admissible=False)
        assert exc.value.status == 3
        # context still usable
        ctx.initial()
        assert ctx.freeze(1e-3) > 0


def test_gmres_iteration_limit():
    d = capi.simple_wave_desc(8, 8, 2, 45)
    with capi.Context(d, capi.default_opts(form=capi.FORM_DG, max_krylov=1)) as ctx:
        ctx.initial()
        ctx.freeze(0.05)
        u = ctx.download("U")
        ctx.upload("OLD", u * 1.01)
        ctx.set_dt(0.05)
        ctx.residual()
        r = ctx.download("R")
        with pytest.raises(capi.EngineError) as exc:
            ctx.linear_solve(-r)
        assert exc.value.status == 12
        assert "GMRES iteration limit reached" in str(exc.value)


def test_cli_past_shock_time():
    proc = subprocess.run([str(CLI), "--nx", "4", "--ny", "4", "--k", "1", "--T", "0.5"],
                          capture_output=True, text=True, timeout=120)
    assert proc.returncode == 1
    assert "Exact solution requires T < 4/((gamma+1)*pi)" in proc.stderr


@pytest.mark.parametrize("form", ["dg", "hdg"])
def test_ilu_wait_limit_runs_out_and_context_recovers(form):
    """A block ILU(0) factor and apply whose waits on other CTAs can never be
    met (a progress value no CTA publishes) run out their 1 ms bound, return
    EG_ERR_WAIT_LIMIT and leave the context usable: with the default bound
    restored the same factor and apply give the reference's numbers."""
    hdg = form == "hdg"
    nx, ny, k = 12, 10, 2
    d = capi.simple_wave_desc(nx, ny, k, 35.0)
    opts = capi.default_opts(form=capi.FORM_HDG if hdg else capi.FORM_DG, precond=capi.PC_ILU0)
    with capi.Context(d, opts) as ctx:
        ctx.initial()
        u = ctx.download("U")
        dt = 0.02
        ctx.freeze(dt)
        ctx.upload("OLD", u * 0.999)
        ctx.set_dt(dt)
        ctx.residual()
        if hdg:
            ctx.condense()
        n = ctx.nl if hdg else ctx.nu
        b = np.cos(0.37 * np.arange(n))
        ctx.pc_factor(True)
        good = ctx.pc_apply(b)
        ctx.set_ilu_wait(limit_ns=1_000_000, starve=True)
        with pytest.raises(capi.EngineError) as exc:
            ctx.pc_apply(b)
        assert exc.value.status == 24
        with pytest.raises(capi.EngineError) as exc:
            ctx.pc_factor(True)
        assert exc.value.status == 24
        ctx.set_ilu_wait()  # default bound, waits reachable again
        ctx.pc_factor(True)
        again = ctx.pc_apply(b)
        assert np.array_equal(again, good)
        x, _, st = ctx.linear_solve(-ctx.download("R") if not hdg else ctx.download("RHS"))
        assert st.residual <= 1e-11 and np.all(np.isfinite(x))
