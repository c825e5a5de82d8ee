"""Pins the numpy restatement in oracle/euler_oracle.py against the golden
fixtures, which the unmodified reference (built against the MFEM-subset shim)
produced.  CPU only; these are the oracle's own known-answer tests."""
import math

import numpy as np
import pytest

from conftest import GOLDEN, cli_files, manifest, rel_err, unit_files
from oracle import euler_oracle as eo

# Tolerances: operators are restated with a different summation order than the
# reference, so they agree to a few ulps of the largest term; GMRES solutions
# agree to the solve tolerance (1e-12 relative residual) times the conditioning.
OP_TOL = 1e-12
SOLVE_TOL = 1e-9


def _problem(f):
    pb = eo.Problem(int(f["nx"]), int(f["ny"]), int(f["k"]), float(f["alpha"]),
                    tables=eo.tables_from_fixture(f))
    pb.freeze(f["u"], float(f["dt"]), True)
    pb.old = np.array(f["old"])
    return pb


def _colmajor(blocks, count, rows, cols):
    return np.asarray(blocks).reshape(count, cols, rows).transpose(0, 2, 1)


@pytest.mark.parametrize("path", unit_files(), ids=lambda p: p.stem)
def test_tables_match_reference(path):
    f = np.load(path)
    k = int(f["k"])
    lx, ly, hx, hy, area = f["geometry"]
    pb = eo.Problem(int(f["nx"]), int(f["ny"]), k, float(f["alpha"]))
    assert np.allclose([pb.lx, pb.ly, pb.hx, pb.hy, pb.area], f["geometry"], rtol=1e-15, atol=0)
    tb = pb.tab
    q, p = k + 1, (k + 1) ** 2
    for mine, ref in ((tb.w, f["w"]), (tb.ew, f["ew"]), (tb.mass, f["mass"]), (tb.inv_mass, f["inv_mass"]),
                      (tb.tdx, f["tensor_dx"]), (tb.tdy, f["tensor_dy"]), (tb.fv, f["fv"])):
        assert rel_err(mine, ref) < 1e-13
    # the zero pattern of the sparse tables is the reference's
    assert np.array_equal(tb.fv.reshape(-1) == 0, np.asarray(f["fv"]) == 0)
    assert np.array_equal(tb.tdx.reshape(-1) == 0, np.asarray(f["tensor_dx"]) == 0)


@pytest.mark.parametrize("path", unit_files(), ids=lambda p: p.stem)
def test_freeze_residual_norm(path):
    f = np.load(path)
    pb = eo.Problem(int(f["nx"]), int(f["ny"]), int(f["k"]), float(f["alpha"]),
                    tables=eo.tables_from_fixture(f))
    rate = pb.freeze(f["u"], float(f["dt"]), True)
    assert rel_err(pb.a.reshape(-1), f["a"]) < OP_TOL
    assert rel_err(pb.b.reshape(-1), f["b"]) < OP_TOL
    assert abs(rate - float(f["rate"][0])) <= 1e-14 * rate
    pb.old = np.array(f["old"])
    r = pb.residual(f["u"])
    assert rel_err(r, f["r"]) < OP_TOL
    assert abs(pb.cell_norm(f["r"]) - float(f["r_norm"][0])) <= 1e-14 * float(f["r_norm"][0])
    assert pb.admissible(f["u"])


@pytest.mark.parametrize("path", unit_files(), ids=lambda p: p.stem)
def test_dg_jacobian_action_and_blocks(path):
    f = np.load(path)
    pb = _problem(f)
    pb.dg_refresh(f["u"])
    assert rel_err(pb.dg_apply(f["x"]), f["jx"]) < OP_TOL
    if "dg_blocks" in f.files:
        m, n = pb.m, pb.n
        blocks = pb.dg_jacobi_blocks(f["u"])
        assert rel_err(blocks, _colmajor(f["dg_blocks"], n, m, m)) < OP_TOL


@pytest.mark.parametrize("path", unit_files(), ids=lambda p: p.stem)
def test_condensation_schur_recovery(path):
    f = np.load(path)
    pb = _problem(f)
    X, y, rhs, D = pb.condense(f["u"], f["r"])
    assert rel_err(D, f["D"]) < OP_TOL
    assert rel_err(y.reshape(-1), f["y_hdg"]) < 1e-11
    assert rel_err(rhs, f["rhs"]) < 1e-11
    if "X" in f.files:
        assert rel_err(X, _colmajor(f["X"], pb.n, pb.m, 4 * pb.t)) < 1e-11
        assert rel_err(pb.schur_jacobi_blocks(), _colmajor(f["schur_blocks"], pb.nf, pb.t, pb.t)) < 1e-11
    assert rel_err(pb.schur_apply(f["v"]), f["sv"]) < 1e-11
    assert rel_err(pb.recover(f["lam"]), f["du"]) < 1e-11


@pytest.mark.parametrize("path", unit_files(), ids=lambda p: p.stem)
def test_weighted_gmres_solves(path):
    f = np.load(path)
    pb = _problem(f)
    # DG form: J x = -r with block-Jacobi cell blocks
    pb.dg_refresh(f["u"])
    blocks = pb.dg_jacobi_blocks(f["u"])
    lr, _ = eo.linear_solve(pb.dg_apply, blocks, -np.asarray(f["r"]), pb.cell_metric, 1e-12, 1500, 20)
    assert rel_err(lr.x, f["solve_dg_x"]) < SOLVE_TOL
    assert abs(lr.count - int(f["solve_dg_count"][0])) <= 1
    assert lr.residual <= 1e-11
    # HDG form: S lambda = rhs with Schur block Jacobi
    _, _, rhs, _ = pb.condense(f["u"], f["r"])
    lr, _ = eo.linear_solve(pb.schur_apply, pb.schur_jacobi_blocks(), rhs, pb.trace_metric, 1e-12, 1500, 20)
    assert rel_err(lr.x, f["solve_hdg_x"]) < SOLVE_TOL
    assert abs(lr.count - int(f["solve_hdg_count"][0])) <= 1


def test_initial_projection_matches_reference():
    for path in cli_files():
        f = np.load(path)
        args = list(__import__("json").loads(str(f["args"])))
        opt = lambda flag, default: type(default)(args[args.index(flag) + 1]) if flag in args else default
        pb = eo.Problem(opt("--nx", 100), opt("--ny", 100), opt("--k", 1), opt("--alpha-deg", 45.0))
        assert rel_err(pb.initial(), f["u0"]) < 1e-13


def _cli_case(name):
    f = np.load(GOLDEN / f"cli_{name}.npz")
    args = list(__import__("json").loads(str(f["args"])))
    opt = lambda flag, default: type(default)(args[args.index(flag) + 1]) if flag in args else default
    kw = dict(nx=opt("--nx", 100), ny=opt("--ny", 100), k=opt("--k", 1), alpha_deg=opt("--alpha-deg", 45.0),
              cfl=opt("--cfl", -1.0), steps=opt("--steps", -1), newton_steps=opt("--newton-steps", -1),
              integrator=opt("--integrator", "ssp-dirk3"), linear_tol=opt("--linear-tol", 1e-12),
              precond=opt("--precond", "block-jacobi"))
    return f, kw


@pytest.mark.parametrize("name", ["be1_8x8_q2", "c1_16x16_q3", "ilu_8x8_q2"])
@pytest.mark.parametrize("form", ["dg", "hdg"])
def test_time_loop_matches_reference_cli(name, form):
    f, kw = _cli_case(name)
    cols = manifest()["iteration_columns"]
    u, records, pb, time = eo.run(form=form, u0=f["u0"], **kw)
    assert rel_err(u, f[f"{form}_u"]) < 1e-10
    it = f[f"{form}_iterations"]
    assert len(records) == len(it)
    damp = np.array([r.damping for r in records])
    assert np.array_equal(damp, it[:, cols.index("damping")])
    kry = np.array([r.krylov for r in records])
    assert np.max(np.abs(kry - it[:, cols.index("krylov_iterations")])) <= 1
    rms = np.array([r.rms for r in records])
    assert rel_err(rms, it[:, cols.index("residual_physical_rms")]) < 1e-8
    summ = f[f"{form}_summary"]
    scols = manifest()["summary_columns"]
    errs = pb.errors(u, time)
    ref_errs = summ[[scols.index(c) for c in ("rho_L2", "rhou_L2", "rhov_L2", "energy_L2")]]
    assert rel_err(errs, ref_errs) < 1e-9
    drift = np.max(np.abs(pb.integral(u) - pb.integral(f["u0"])))
    assert drift < 1e-12


def test_oracle_errors_carry_reference_messages():
    pb = eo.Problem(3, 2, 1, 45.0)
    u = pb.initial()
    u[0] = -1.0
    with pytest.raises(eo.OracleError, match="Old state is inadmissible; refine mesh"):
        pb.freeze(u, 1e-3, True)
    with pytest.raises(eo.OracleError, match="Nonpositive old face state; refine mesh"):
        pb.freeze(u, 1e-3, False)
    # GMRES with a tiny iteration limit raises the reference's message
    pb2 = eo.Problem(4, 4, 2, 30.0)
    u2 = pb2.initial()
    pb2.freeze(u2, 0.05 * min(pb2.hx, pb2.hy), True)
    pb2.old = u2 * 0.99
    r = pb2.residual(u2)
    pb2.dg_refresh(u2)
    with pytest.raises(eo.OracleError, match="GMRES iteration limit reached"):
        eo.linear_solve(pb2.dg_apply, pb2.dg_jacobi_blocks(u2), -r, pb2.cell_metric, 1e-12, 2, 20)


def _ilu_of(pb, f, hdg):
    ilu = eo.BlockILU0(eo.solver_graph(pb, hdg), pb.t if hdg else pb.m)
    if hdg:
        pb.condense(f["u"], f["r"])
        eo.fill_hdg_ilu(pb, ilu)
    else:
        eo.fill_dg_ilu(pb, ilu, f["u"])
    return ilu


@pytest.mark.parametrize("path", unit_files(), ids=lambda p: p.stem)
@pytest.mark.parametrize("tag", ["dg", "hdg"])
def test_block_ilu0_fill_factor_apply(path, tag):
    f = np.load(path)
    pb = _problem(f)
    hdg = tag == "hdg"
    ilu = _ilu_of(pb, f, hdg)
    B = ilu.b
    nnzb = len(ilu.col)
    if f"ilu_{tag}_filled" in f.files:
        ref = _colmajor(f[f"ilu_{tag}_filled"], nnzb, B, B)
        assert rel_err(ilu.data, ref) < 1e-11
    ilu.factor()
    if f"ilu_{tag}_factored" in f.files:
        ref = _colmajor(f[f"ilu_{tag}_factored"], nnzb, B, B)
        off = np.ones(nnzb, bool)
        off[ilu.diag] = False
        assert rel_err(ilu.data[off], ref[off]) < 1e-10
        # diagonal entries hold the row-pivoted LU factors (LAPACK packing)
        packed = np.stack([ilu.lu[i][0] for i in range(ilu.rows)])
        assert rel_err(packed, ref[ilu.diag]) < 1e-10
    assert rel_err(ilu(f[f"ilu_{tag}_b"]), f[f"ilu_{tag}_x"]) < 1e-10
    # one weighted GMRES solve preconditioned by the ILU
    if hdg:
        rhs, apply, metric = pb.condense(f["u"], f["r"])[2], pb.schur_apply, pb.trace_metric
    else:
        pb.dg_refresh(f["u"])
        rhs, apply, metric = -np.asarray(f["r"]), pb.dg_apply, pb.cell_metric
    lr, _ = eo.linear_solve(apply, ilu, rhs, metric, 1e-12, 1500, 20)
    assert rel_err(lr.x, f[f"solve_{tag}_ilu_x"]) < SOLVE_TOL
    assert abs(lr.count - int(f[f"solve_{tag}_ilu_count"][0])) <= 1
