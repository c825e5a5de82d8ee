"""Update-by-update parity of the device Newton update with the reference.

Every accepted Newton update of the 16x16 Q3 workload (SSP-DIRK3, CFL 1,
3 steps x 4 stages x 3 updates, both forms) is compared with the reference's
own update at the same position of its time loop (tests/golden/traj_*.npz,
recorded by the reference's objects and pinned to its command line): the
Newton direction du -- the recovered body update for HDG -- and the
line-search damping, which must be identical.

Bar for du (FP64, 2-norm): every update agrees to 1e-10 relative to the
stage's first Newton correction (the scale of the stage solve), and every
update at least 1e-4 of that scale also agrees to 1e-10 relative to itself.
The last update of a stage is 1e-8..1e-7 of the first: its right-hand side
(the residual) is then within a few hundred roundoff units of zero, so
relative to itself du carries the rounding of the residual evaluation
(7e-7 on this workload, i.e. 4e-16 of the state) on either machine.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN, rel_err
from mfem_euler2d_cpp_b200 import capi

pytestmark = pytest.mark.gpu
DU_TOL = 1e-10


def ref_newton_steps(args):
    return args[args.index("--newton-steps") + 1]


def _opt(args, flag, default):
    return type(default)(args[args.index(flag) + 1]) if flag in args else default


@pytest.mark.parametrize("form", ["dg", "hdg"])
def test_every_newton_update_matches_reference(form):
    f = np.load(GOLDEN / "traj_c1_16x16_q3.npz")
    args = json.loads(str(f["args"]))
    nx, ny, k = _opt(args, "--nx", 100), _opt(args, "--ny", 100), _opt(args, "--k", 1)
    d = capi.simple_wave_desc(nx, ny, k, _opt(args, "--alpha-deg", 45.0))
    hdg = form == "hdg"
    opts = capi.default_opts(form=capi.FORM_HDG if hdg else capi.FORM_DG)
    ref_du, ref_damping = f[f"{form}_du"], f[f"{form}_damping"]
    with capi.Context(d, opts) as ctx:
        ro, keep = capi.run_options(integrator="ssp-dirk3", steps=_opt(args, "--steps", -1),
                                    newton_steps=_opt(args, "--newton-steps", -1), cfl=_opt(args, "--cfl", -1.0),
                                    form_name=form)
        st = capi.Stepper(ctx, ro, keep)
        per_stage = int(ref_newton_steps(args))
        worst_scale = worst_self = 0.0
        for i in range(len(ref_du)):
            s = st.next()
            assert s is not None, f"schedule ended after {i} updates"
            du = ctx.download("DU")
            diff = np.linalg.norm(du - ref_du[i])
            scale = np.linalg.norm(ref_du[i - i % per_stage])  # the stage's first correction
            own = np.linalg.norm(ref_du[i])
            worst_scale = max(worst_scale, diff / scale)
            assert diff <= DU_TOL * scale, f"update {i}: du differs by {diff / scale:.3e} of the stage scale"
            if own >= 1e-4 * scale:
                worst_self = max(worst_self, diff / own)
                assert diff <= DU_TOL * own, f"update {i}: du differs by {diff / own:.3e} of itself"
            assert s.damping == ref_damping[i], f"update {i}: damping {s.damping} vs {ref_damping[i]}"
        assert st.next() is None
        st.close()
    print(f"{form}: {len(ref_du)} updates, worst du difference {worst_scale:.3e} of the stage scale, "
          f"{worst_self:.3e} of itself above 1e-4 of it")
