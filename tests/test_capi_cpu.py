"""CPU-side checks of the C-ABI boundary: the library loads without a GPU,
exports every function include/euler2d_cuda.h declares, builds the
reference's host tables bit for bit, and the euler2d command line validates
options exactly like the reference (src/options.cpp) before touching CUDA."""
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, unit_files
from mfem_euler2d_cpp_b200 import capi

CLI = ROOT / "mfem_euler2d_cpp_b200" / "bin" / "euler2d"


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = capi.declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_status_strings_match_reference_messages():
    lib = capi.load()
    assert lib.eg_status_string(12) == b"GMRES iteration limit reached"
    assert lib.eg_status_string(16) == b"Newton line search failed"
    assert lib.eg_status_string(7) == b"Singular streaming HDG cell factor"
    assert lib.eg_status_string(14) == b"Recovered DG residual criterion failed after Schur refinement"


@pytest.mark.parametrize("path", unit_files(), ids=lambda p: p.stem)
def test_host_tables_match_reference(path):
    f = np.load(path)
    nx, ny, k, alpha = int(f["nx"]), int(f["ny"]), int(f["k"]), float(f["alpha"])
    d = capi.simple_wave_desc(nx, ny, k, alpha)
    q, p = k + 1, (k + 1) ** 2
    lx, ly, hx, hy, area = f["geometry"]
    assert (d.lx, d.ly, d.hx, d.hy, d.area) == (lx, ly, hx, hy, area)
    np.testing.assert_array_equal(np.array(d.w[:p]), f["w"])
    np.testing.assert_array_equal(np.array(d.ew[:q]), f["ew"])
    np.testing.assert_array_equal(np.array(d.inv_mass[:p]), f["inv_mass"])
    np.testing.assert_array_equal(np.array(d.mass[:p]), f["mass"])
    np.testing.assert_array_equal(np.array(d.tensor_dx[:q * q]), f["tensor_dx"])
    np.testing.assert_array_equal(np.array(d.tensor_dy[:q * q]), f["tensor_dy"])
    np.testing.assert_array_equal(np.array(d.tensor_node[:p]), f["tensor_node"])
    fv = f["fv"].reshape(4, q, p)
    fb = np.array(d.face_basis[:4 * q * q]).reshape(4, q, q)
    for s in range(4):
        for j in range(q):
            for l in range(q):
                node = j * q + l if s < 2 else l * q + j
                assert fb[s, j, l] == fv[s, j, node]
            # every other node of the reference table is zero on this face point
            on_line = {j * q + l if s < 2 else l * q + j for l in range(q)}
            assert all(fv[s, j, i] == 0 for i in range(p) if i not in on_line)


def _cli(*args):
    # run in a scratch directory: a command line that fails after parsing may
    # already have created its default output directory (code_test/results)
    with tempfile.TemporaryDirectory() as tmp:
        return subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=60, cwd=tmp)


@pytest.mark.parametrize("args,message", [
    (["--k", "9"], "Invalid mesh, degree, time or safety"),
    (["--nx", "1"], "Invalid mesh, degree, time or safety"),
    (["--form", "cg"], "Invalid form"),
    (["--integrator", "rk4"], "Invalid time integrator"),
    (["--precond", "amg"], "Invalid preconditioner"),
    (["--alpha-deg", "90"], "Require 0 < alpha-deg < 90"),
    (["--cfl", "-1"], "--cfl must be positive"),
    (["--bogus"], "Unknown option: --bogus"),
    (["--nx"], "Missing option value"),
    (["--volume-order", "5"], "Volume rule must be (k+1)^2 GL points (order 2k+1)"),
    (["--device", "cpu"], "This executable is the --device cuda path"),
    (["--assembly", "csr"], "Invalid assembly"),
    (["--solver", "direct", "--assembly", "element"], "Direct LU requires --assembly full"),
    (["--assembly", "full", "--precision", "mixed"], "--precision mixed requires --assembly partial or element"),
    # the reference's portable build has no MKL PARDISO either: same message
    (["--solver", "direct"], "--solver direct requires MFEM with MKL PARDISO"),
    # LinearSolver workspace limit (src/linear.cpp:46-47), raised before any device work
    (["--solver", "dense", "--nx", "40", "--ny", "40", "--k", "3", "--form", "dg"],
     "Dense direct solve limited to 5000 unknowns"),
])
def test_cli_rejects_invalid_options(args, message):
    proc = _cli(*args)
    assert proc.returncode == 1
    assert proc.stderr.startswith("ERROR: ")
    assert message in proc.stderr


def test_cli_help():
    proc = _cli("--help")
    assert proc.returncode == 0
    assert "--form dg|hdg|both" in proc.stdout
    assert "--assembly full|element|partial" in proc.stdout


def _mesh_records(text):
    """Non-comment, non-blank lines of an MFEM mesh v1.0 text."""
    return [ln.split() for ln in text.splitlines() if ln.strip() and not ln.startswith("#")]


def test_save_solution_writes_reference_files(tmp_path):
    """Problem::Save (src/problem.cpp:762-790) of the reference's final states:
    the mesh records, and the .gf and _coefficients.csv texts, equal the
    reference command line's files byte for byte (the mesh may add MFEM's
    geometry-type comment block)."""
    f = np.load(ROOT / "tests" / "golden" / "solution_8x6_q2.npz")
    d = capi.simple_wave_desc(8, 6, 2, 30.0)
    for form in ("dg", "hdg"):
        prefix = tmp_path / form
        capi.save_solution(d, f[f"{form}_u"], str(prefix))
        mesh = (tmp_path / f"{form}.mesh").read_text()
        assert mesh.startswith("MFEM mesh v1.0\n")
        assert _mesh_records(mesh) == _mesh_records(str(f[f"{form}_mesh"]))
        for name in ("rho", "rhou", "rhov", "energy"):
            assert (tmp_path / f"{form}_{name}.gf").read_text() == str(f[f"{form}_{name}_gf"])
        coeff = np.loadtxt(tmp_path / f"{form}_coefficients.csv", delimiter=",", skiprows=1)
        np.testing.assert_array_equal(coeff[:, 2:].reshape(-1), f[f"{form}_u"])


def test_save_solution_rejects_bad_input(tmp_path):
    d = capi.simple_wave_desc(8, 6, 2, 30.0)
    with pytest.raises(capi.EngineError):
        capi.save_solution(d, np.zeros(7), str(tmp_path / "x"))
    with pytest.raises(capi.EngineError, match="Cannot open solution output"):
        capi.save_solution(d, np.zeros(4 * 9 * 48), str(tmp_path / "missing" / "x"))


def test_workload_l2_check_counts_only_runs_that_completed_in_both():
    """The 1% bar of the batch and serve lines: joint L2 error against the
    plain FP64 run's, only where both completed."""
    from mfem_euler2d_cpp_b200 import workloads

    ref = [[3e-7, 4e-7, 0., 0.], [1e-6, 0., 0., 0.], [2e-6, 0., 0., 0.]]
    ok = [[3e-7, 4e-7, 0., 0.], [1.005e-6, 0., 0., 0.], [9e-6, 0., 0., 0.]]
    checked, worst, within = workloads.l2_check([0, 0, 20], ok, [0, 0, 0], ref)
    assert checked == 2 and abs(worst - 0.005) < 1e-12 and within
    checked, worst, within = workloads.l2_check([0, 0, 0], ok, [0, 0, 0], ref)
    assert checked == 3 and abs(worst - 3.5) < 1e-12 and not within
