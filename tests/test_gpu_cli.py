"""End-to-end parity of the euler2d --device cuda command line with the
reference command line on the reference's own test configurations
(code_test/test_solver.py) and the 16x16 Q3 workload: final states, per-update
residuals, Krylov counts, damping, L2 errors, conservation drift and DG/HDG
equivalence. The single backward-Euler update pins the recovered body-DOF
increment du = u1 - u0 to 1e-10 relative."""
import csv
import json
import subprocess

import numpy as np
import pytest

from conftest import ROOT, cli_files, manifest, rel_err

pytestmark = pytest.mark.gpu
CLI = ROOT / "mfem_euler2d_cpp_b200" / "bin" / "euler2d"


def run_cli(args, out):
    prefix = out / "run"
    proc = subprocess.run([str(CLI), *args, "--output", str(prefix)], capture_output=True, text=True,
                          timeout=600)
    assert proc.returncode == 0, proc.stderr
    return prefix


def load_form(prefix, form, cols):
    coeff = np.loadtxt(f"{prefix}_{form}_coefficients.csv", delimiter=",", skiprows=1)
    with open(f"{prefix}_{form}_iterations.csv", newline="") as fh:
        rows = list(csv.DictReader(fh))
    with open(f"{prefix}_{form}_summary.csv", newline="") as fh:
        summary = next(csv.DictReader(fh))
    iters = np.array([[float(r[c]) for c in cols] for r in rows])
    return coeff[:, 2:].reshape(-1), iters, summary


@pytest.mark.parametrize("path", cli_files(), ids=lambda p: p.stem)
def test_cli_matches_reference(path, tmp_path):
    f = np.load(path)
    args = json.loads(str(f["args"]))
    meta = manifest()
    icol = meta["iteration_columns"]
    scol = meta["summary_columns"]
    prefix = run_cli(args, tmp_path)
    for form in ("dg", "hdg"):
        u, iters, summary = load_form(prefix, form, icol)
        ref_u, ref_iters, ref_summary = f[f"{form}_u"], f[f"{form}_iterations"], f[f"{form}_summary"]
        # final state and per-update increments
        assert rel_err(u, ref_u) < 1e-10
        du, ref_du = u - f["u0"], ref_u - f["u0"]
        assert rel_err(du, ref_du) < 1e-9
        assert iters.shape == ref_iters.shape
        c = {name: i for i, name in enumerate(icol)}
        for name in ("step", "stage", "newton"):
            np.testing.assert_array_equal(iters[:, c[name]], ref_iters[:, c[name]])
        assert rel_err(iters[:, c["residual_physical_rms"]], ref_iters[:, c["residual_physical_rms"]]) < 1e-8
        np.testing.assert_array_equal(iters[:, c["damping"]], ref_iters[:, c["damping"]])
        assert np.all(np.abs(iters[:, c["krylov_iterations"]] - ref_iters[:, c["krylov_iterations"]]) <= 2)
        assert rel_err(iters[:, c["dt"]], ref_iters[:, c["dt"]]) < 1e-12
        s = {name: float(summary[name]) for name in scol}
        rs = dict(zip(scol, ref_summary))
        assert s["newton_updates"] == rs["newton_updates"]
        assert s["time_steps"] == rs["time_steps"]
        assert abs(s["T"] - rs["T"]) <= 1e-14 * max(1, abs(rs["T"]))
        for name in ("rho_L2", "rhou_L2", "rhov_L2", "energy_L2"):
            assert abs(s[name] - rs[name]) <= 1e-9 * rs[name] + 1e-15
        assert s["max_conservation_drift"] < 1e-13  # the reference's own drift here: 3e-15 to 3.4e-14
        assert summary["device"] == "cuda"
        # a direct solver defaults to full assembly and no preconditioner (src/options.cpp:136-142)
        solver = args[args.index("--solver") + 1] if "--solver" in args else "gmres"
        default_assembly = "partial" if solver == "gmres" else "full"
        assembly = args[args.index("--assembly") + 1] if "--assembly" in args else default_assembly
        assert summary["assembly"] == assembly
        assert summary["solver"] == solver
        if solver != "gmres":
            assert summary["preconditioner"] == "none"
        assert int(summary["matrix_free"]) == (assembly != "full")  # src/options.cpp:135
    with open(f"{prefix}_comparison.csv", newline="") as fh:
        comp = next(csv.DictReader(fh))
    assert float(comp["max_nodal_difference"]) < 1e-8


def test_single_backward_euler_update_increment(tmp_path):
    """One damped BE update on 8x8 Q2: du agrees with the reference to 1e-10."""
    f = np.load(ROOT / "tests" / "golden" / "cli_be1_8x8_q2.npz")
    prefix = run_cli(json.loads(str(f["args"])), tmp_path)
    for form in ("dg", "hdg"):
        u = np.loadtxt(f"{prefix}_{form}_coefficients.csv", delimiter=",", skiprows=1)[:, 2:].ravel()
        assert rel_err(u - f["u0"], f[f"{form}_u"] - f["u0"]) < 1e-10


def test_code_test_assertions(tmp_path):
    """The reference's own code test (code_test/test_solver.py) against --device cuda."""
    smoke = run_cli(["--nx", "8", "--ny", "8", "--k", "1", "--cfl", ".1", "--steps", "1", "--form", "both",
                     "--no-save-solution", "--newton-tol", "1e-12", "--linear-tol", "1e-12"], tmp_path)
    for form in ("dg", "hdg"):
        with open(f"{smoke}_{form}_summary.csv", newline="") as fh:
            s = next(csv.DictReader(fh))
        assert s["integrator"] == "ssp-dirk3"
        assert int(s["time_steps"]) == 1
        assert int(s["newton_updates"]) > 0
    with open(f"{smoke}_comparison.csv", newline="") as fh:
        assert float(next(csv.DictReader(fh))["max_nodal_difference"]) < 1e-8
    be_dir = tmp_path / "be"
    be_dir.mkdir()
    be = run_cli(["--nx", "8", "--ny", "8", "--k", "2", "--cfl", ".1", "--steps", "1", "--integrator", "be",
                  "--form", "both", "--check-update", "--newton-tol", "1e-12", "--linear-tol", "1e-12",
                  "--no-save-solution"], be_dir)
    for form in ("dg", "hdg"):
        with open(f"{be}_{form}_summary.csv", newline="") as fh:
            s = next(csv.DictReader(fh))
        assert s["integrator"] == "be"
        assert int(s["fixed_newton_steps"]) == -1
        assert int(s["newton_updates"]) > 0
    with open(f"{be}_hdg_iterations.csv", newline="") as fh:
        for row in csv.DictReader(fh):
            check = float(row["update_check_relative"])
            assert np.isfinite(check) and check < 1e-8
    with open(f"{be}_comparison.csv", newline="") as fh:
        comp = next(csv.DictReader(fh))
    assert float(comp["max_nodal_difference"]) < 1e-8
    assert float(comp["solution_L2_difference"]) < 1e-8


def test_cli_writes_reference_solution_files(tmp_path):
    """The --device cuda run writes Problem::Save's files (src/problem.cpp:762-790):
    the same mesh records as the reference command line, and grid functions
    whose values equal the reference's final state to 1e-10 relative."""
    f = np.load(ROOT / "tests" / "golden" / "solution_8x6_q2.npz")
    prefix = run_cli(json.loads(str(f["args"])), tmp_path)
    records = lambda t: [ln.split() for ln in t.splitlines() if ln.strip() and not ln.startswith("#")]
    for form in ("dg", "hdg"):
        assert records(open(f"{prefix}_{form}.mesh").read()) == records(str(f[f"{form}_mesh"]))
        for name in ("rho", "rhou", "rhov", "energy"):
            text = open(f"{prefix}_{form}_{name}.gf").read()
            ref = str(f[f"{form}_{name}_gf"])
            head, ref_head = text.split("\n\n")[0], ref.split("\n\n")[0]
            assert head == ref_head
            vals = np.array(text.split("\n\n", 1)[1].split(), float)
            ref_vals = np.array(ref.split("\n\n", 1)[1].split(), float)
            assert rel_err(vals, ref_vals) < 1e-10
