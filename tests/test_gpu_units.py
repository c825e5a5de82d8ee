"""GPU parity of every operator on the Newton-update path against the
reference's own outputs (fixtures from tests/golden/make_golden.py).

Tolerances (FP64): direct operators (frozen bounds, residual, Jacobian
action, condensation, Schur action, recovery, block assembly) agree to
1e-12 relative in the 2-norm; linear solves (weighted GMRES to 1e-12) agree
to 1e-10 relative, with Krylov counts within one iteration of the reference.
"""
import numpy as np
import pytest

from conftest import GOLDEN, rel_err, unit_files
from mfem_euler2d_cpp_b200 import capi

pytestmark = pytest.mark.gpu
OP_TOL = 1e-12
SOLVE_TOL = 1e-10


def _ctx(f, form, **opts):
    d = capi.simple_wave_desc(int(f["nx"]), int(f["ny"]), int(f["k"]), float(f["alpha"]))
    ctx = capi.Context(d, capi.default_opts(form=form, **opts))
    ctx.upload("U", f["u"])
    rate = ctx.freeze(float(f["dt"]), check_admissible=True)
    ctx.upload("OLD", f["old"])
    ctx.set_dt(float(f["dt"]))
    return ctx, rate


@pytest.fixture(params=unit_files(), ids=lambda p: p.stem)
def unit(request):
    return np.load(request.param)


def test_freeze_and_residual(unit):
    f = unit
    ctx, rate = _ctx(f, capi.FORM_HDG)
    with ctx:
        assert rel_err(rate, f["rate"]) < OP_TOL
        assert rel_err(ctx.download("HLL_A"), f["a"]) < OP_TOL
        assert rel_err(ctx.download("HLL_B"), f["b"]) < OP_TOL
        ctx.residual()
        assert rel_err(ctx.download("R"), f["r"]) < OP_TOL
        assert rel_err(ctx.cell_norm("R"), f["r_norm"]) < OP_TOL
        assert ctx.admissible("U")


def test_dg_jacobian_action(unit):
    f = unit
    ctx, _ = _ctx(f, capi.FORM_DG)
    with ctx:
        assert rel_err(ctx.dg_apply(f["x"]), f["jx"]) < OP_TOL
        if "dg_blocks" in f:
            ctx.pc_factor(False)
            assert rel_err(ctx.download("PC_BLOCKS"), f["dg_blocks"]) < OP_TOL


def test_hdg_condensation_schur_recovery(unit):
    f = unit
    ctx, _ = _ctx(f, capi.FORM_HDG)
    with ctx:
        ctx.upload("R", f["r"])
        ctx.condense()
        assert rel_err(ctx.download("D"), f["D"]) < OP_TOL
        assert rel_err(ctx.download("RHS"), f["rhs"]) < OP_TOL
        assert rel_err(ctx.download("Y"), f["y_hdg"]) < OP_TOL
        if "X" in f:
            assert rel_err(ctx.download("X"), f["X"]) < OP_TOL
        assert rel_err(ctx.schur_apply(f["v"]), f["sv"]) < OP_TOL
        assert rel_err(ctx.recover(f["lam"]), f["du"]) < OP_TOL
        if "schur_blocks" in f:
            ctx.pc_factor(False)
            assert rel_err(ctx.download("PC_BLOCKS"), f["schur_blocks"]) < OP_TOL


def test_dg_linear_solve(unit):
    f = unit
    ctx, _ = _ctx(f, capi.FORM_DG)
    with ctx:
        x, eq, st = ctx.linear_solve(-f["r"])
        assert rel_err(x, f["solve_dg_x"]) < SOLVE_TOL
        assert abs(st.count - int(f["solve_dg_count"][0])) <= 1
        assert st.residual <= 1e-11


def test_hdg_linear_solve(unit):
    f = unit
    ctx, _ = _ctx(f, capi.FORM_HDG)
    with ctx:
        ctx.upload("R", f["r"])
        ctx.condense()
        x, eq, st = ctx.linear_solve(f["rhs"])
        assert rel_err(x, f["solve_hdg_x"]) < SOLVE_TOL
        assert abs(st.count - int(f["solve_hdg_count"][0])) <= 1
        assert st.residual <= 1e-11


@pytest.mark.parametrize("assembly", [capi.ASSEMBLY_ELEMENT, capi.ASSEMBLY_FULL], ids=["element", "full"])
def test_assembled_operators_and_solves(unit, assembly):
    """--assembly element|full: the Schur action from the per-cell entries C X
    (all 16 panels kept at every degree), the Schur blocks read from that
    layout, and the DG and HDG solves (GMRES on the assembled block-sparse
    matrix for full assembly, on the element operators for element
    assembly) against the reference's matrix-free solves."""
    f = unit
    ctx, _ = _ctx(f, capi.FORM_HDG, assembly=assembly)
    with ctx:
        ctx.upload("R", f["r"])
        ctx.condense()
        assert rel_err(ctx.schur_apply(f["v"]), f["sv"]) < OP_TOL
        if "schur_blocks" in f:
            ctx.pc_factor(False)
            assert rel_err(ctx.download("PC_BLOCKS"), f["schur_blocks"]) < OP_TOL
        x, _, st = ctx.linear_solve(f["rhs"])
        assert rel_err(x, f["solve_hdg_x"]) < SOLVE_TOL
        assert abs(st.count - int(f["solve_hdg_count"][0])) <= 1
        assert st.residual <= 1e-11
    ctx, _ = _ctx(f, capi.FORM_DG, assembly=assembly)
    with ctx:
        x, _, st = ctx.linear_solve(-f["r"])
        assert rel_err(x, f["solve_dg_x"]) < SOLVE_TOL
        assert abs(st.count - int(f["solve_dg_count"][0])) <= 1
        assert st.residual <= 1e-11


def test_full_assembly_with_block_ilu(unit):
    """Full assembly keeps the assembled matrix apart from the ILU(0) factors."""
    f = unit
    for form in (capi.FORM_DG, capi.FORM_HDG):
        ctx, _ = _ctx(f, form, assembly=capi.ASSEMBLY_FULL, precond=capi.PC_ILU0)
        with ctx:
            if form == capi.FORM_HDG:
                ctx.upload("R", f["r"])
                ctx.condense()
                x, _, st = ctx.linear_solve(f["rhs"])
                want, count = f["solve_hdg_ilu_x"], int(f["solve_hdg_ilu_count"][0])
            else:
                x, _, st = ctx.linear_solve(-f["r"])
                want, count = f["solve_dg_ilu_x"], int(f["solve_dg_ilu_count"][0])
            assert rel_err(x, want) < SOLVE_TOL
            assert abs(st.count - count) <= 1
            assert st.residual <= 1e-11


def test_pc_apply_inverts_blocks(unit):
    """Factored block-Jacobi apply equals a dense solve with the reference blocks."""
    f = unit
    if "schur_blocks" not in f:
        pytest.skip("dense blocks stored for small cases only")
    ctx, _ = _ctx(f, capi.FORM_HDG)
    with ctx:
        ctx.upload("R", f["r"])
        ctx.condense()
        ctx.pc_factor(True)
        t = ctx.t
        blocks = f["schur_blocks"].reshape(ctx.nf, t, t).transpose(0, 2, 1)  # column-major
        b = np.sin(0.7 * np.arange(ctx.nl))
        want = np.linalg.solve(blocks, b.reshape(ctx.nf, t, 1)).ravel()
        assert rel_err(ctx.pc_apply(b), want) < 1e-11


@pytest.mark.parametrize("nx,ny,k", [(7, 5, 0), (9, 8, 2), (11, 7, 4), (7, 4, 5), (5, 3, 8)])
def test_hdg_pc_apply_matches_downloaded_inverses(nx, ny, k):
    """The Schur block-Jacobi apply multiplies each face's explicit inverse by
    that face's slice of b; the face counts leave the last group of faces a
    CTA stages partly filled."""
    d = capi.simple_wave_desc(nx, ny, k, 30.0)
    with capi.Context(d, capi.default_opts(form=capi.FORM_HDG)) as ctx:
        ctx.initial()
        u = ctx.download("U")
        ctx.freeze(1e-3, check_admissible=True)
        ctx.upload("OLD", u)
        ctx.set_dt(1e-3)
        ctx.residual()
        ctx.condense()
        ctx.pc_factor(True)
        t = ctx.t
        inv = ctx.download("PC_BLOCKS").reshape(ctx.nf, t, t).transpose(0, 2, 1)
        b = np.cos(0.37 * np.arange(ctx.nl)) + 0.1
        want = np.einsum("fij,fj->fi", inv, b.reshape(ctx.nf, t)).ravel()
        assert rel_err(ctx.pc_apply(b), want) < 1e-13


def test_hdg_jacobi_inverses_download(unit):
    """The factored Schur block-Jacobi slot holds the explicit inverses of the
    assembled blocks (both downloaded column-major): S_f Inv_f = I."""
    f = unit
    ctx, _ = _ctx(f, capi.FORM_HDG)
    with ctx:
        ctx.upload("R", f["r"])
        ctx.condense()
        t = ctx.t
        ctx.pc_factor(False)
        s = ctx.download("PC_BLOCKS").reshape(ctx.nf, t, t).transpose(0, 2, 1)
        ctx.pc_factor(True)
        inv = ctx.download("PC_BLOCKS").reshape(ctx.nf, t, t).transpose(0, 2, 1)
        prod = np.einsum("fij,fjk->fik", s, inv)
        eye = np.broadcast_to(np.eye(t), prod.shape)
        scale = np.abs(s).max(axis=(1, 2)) * np.abs(inv).max(axis=(1, 2))
        assert np.max(np.abs(prod - eye).max(axis=(1, 2)) / scale) < 1e-12


def test_pivot_reciprocal_within_one_ulp_of_division():
    """The condensation's pivot reciprocal (hardware estimate + two
    Newton-Raphson steps) against IEEE 1/x over every binary exponent of the
    normal range, both signs, plus the edges the estimate cannot take
    (subnormal and near-overflow magnitudes, which take IEEE division)."""
    import ctypes as C

    lib = capi.load()
    rng = np.random.default_rng(11)
    exps = np.arange(-1022, 1023)
    mant = rng.uniform(1.0, 2.0, size=(exps.size, 8))
    x = np.ldexp(mant, exps[:, None]).ravel()
    x = np.concatenate([x, -x, [5e-324, -5e-324, 2.2250738585072014e-308 / 3, 1e-310, np.finfo(float).max,
                                -np.finfo(float).max, 2.0 ** 1021, 2.0 ** -1021, 1.0, -1.0]])
    y = np.empty_like(x)
    rc = lib.eg_check_pivot_reciprocal(x.ctypes.data_as(C.POINTER(C.c_double)),
                                       y.ctypes.data_as(C.POINTER(C.c_double)), x.size)
    assert rc == capi.OK
    with np.errstate(over="ignore", divide="ignore"):
        ref = 1.0 / x
    finite = np.isfinite(ref) & (ref != 0)
    ulp = np.spacing(np.abs(ref[finite]))
    assert np.all(np.abs(y[finite] - ref[finite]) <= ulp)
    # overflow to infinity and results below the normal range match division exactly
    assert np.array_equal(y[~finite], ref[~finite])


@pytest.fixture(params=sorted(GOLDEN.glob("condense_*.npz")), ids=lambda p: p.stem)
def condense_case(request):
    return np.load(request.param)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_high_degree_condensation_on_many_cells(condense_case, precision):
    """k = 5..8 on meshes with more cells than the condensation launches CTAs
    (each CTA reduces several cells in its slab): D, the Schur right-hand
    side, y, the Schur action and the recovery against the reference. The
    mixed-precision context condenses in FP64 too, so it meets the same bar."""
    f = condense_case
    nx, ny, k = int(f["nx"]), int(f["ny"]), int(f["k"])
    d = capi.simple_wave_desc(nx, ny, k, float(f["alpha"]))
    prec = capi.PRECISION_MIXED if precision == "mixed" else capi.PRECISION_FP64
    with capi.Context(d, capi.default_opts(form=capi.FORM_HDG, precision=prec)) as ctx:
        ctx.initial()
        u0 = ctx.download("U")
        ctx.upload("U", f["u"])
        ctx.freeze(float(f["dt"]), check_admissible=True)
        ctx.upload("OLD", u0)
        ctx.set_dt(float(f["dt"]))
        ctx.residual()
        ctx.condense()
        assert rel_err(ctx.download("D"), f["D"]) < OP_TOL
        assert rel_err(ctx.download("RHS"), f["rhs"]) < OP_TOL
        assert rel_err(ctx.download("Y"), f["y_hdg"]) < OP_TOL
        vrng = np.random.default_rng([int(f["seed"]), 1])
        v, lam = vrng.standard_normal(ctx.nl), vrng.standard_normal(ctx.nl)
        assert rel_err(ctx.schur_apply(v), f["sv"]) < OP_TOL
        assert rel_err(ctx.recover(lam), f["du"]) < OP_TOL


@pytest.mark.parametrize("nx,ny,k", [(12, 10, 1), (10, 8, 2), (6, 5, 3), (5, 6, 4), (4, 5, 5), (14, 12, 5)])
def test_dg_pc_blocks_are_inverses(nx, ny, k):
    """After eg_pc_factor(1) the DG block-Jacobi slot holds each cell block's
    explicit inverse, column-major (the k >= 3 factor keeps its rows in pivot
    order on the device; the download restores them): inverse x block = I."""
    d = capi.simple_wave_desc(nx, ny, k, 37.0)
    with capi.Context(d, capi.default_opts(form=capi.FORM_DG)) as ctx:
        ctx.initial()
        rate = ctx.freeze(1e-3)
        ctx.freeze(0.24 / rate)
        ctx.upload("OLD", ctx.download("U") * 0.999)
        ctx.set_dt(0.24 / rate)
        m = ctx.nu // (nx * ny)
        ctx.pc_factor(False)
        blocks = ctx.download("PC_BLOCKS").reshape(nx * ny, m, m).transpose(0, 2, 1)
        ctx.pc_factor(True)
        inv = ctx.download("PC_BLOCKS").reshape(nx * ny, m, m).transpose(0, 2, 1)
        prod = np.einsum("eij,ejk->eik", inv, blocks)
        err = np.abs(prod - np.eye(m)).max(axis=(1, 2)) / (np.abs(inv).max(axis=(1, 2)) * np.abs(blocks).max(axis=(1, 2)))
        assert err.max() < 1e-13
        b = np.cos(0.3 * np.arange(ctx.nu))
        want = np.einsum("eij,ej->ei", inv, b.reshape(nx * ny, m)).ravel()
        assert rel_err(ctx.pc_apply(b), want) < 1e-13
