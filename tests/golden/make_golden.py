"""Generate the golden fixtures in this directory from the reference itself.

Runs only where the reference sources are available (it needs the oracle
build in oracle/_ref/, made by `make -C oracle`): the unmodified reference
compiled against the MFEM-subset shim. Two kinds of fixture are written:

* units_*.npz  -- reference public API (Problem, PartialDG, StreamCondense,
  Schur operator, Recover, LinearSolver) on small meshes for k = 0..8: the
  frozen HLL bounds, residual, Jacobian action, block-Jacobi blocks,
  condensation (X, y, rhs, D), Schur action and blocks, recovery and one
  weighted GMRES solve per form, all on a seeded perturbed simple-wave state;
* cli_*.npz    -- the reference euler2d command line on the configurations
  its own tests and the headline 16x16 Q3 workload use, plus element and
  full assembly: final coefficients per form and the per-update
  _iterations.csv columns.

* traj_*.npz   -- every accepted Newton update of a command-line case: the
  Newton direction du (the recovered body update for HDG) and the damping,
  from the reference's time loop on its own objects (ref_trajectory), whose
  final state must equal the command line's.

* condense_*.npz -- condensation, Schur action and recovery at k = 5..8 on
  meshes with more cells than the device condensation has CTAs.

* c2_*.npz     -- the reference command line on the 128x128 Q4 workload (HDG
  with block Jacobi and block ILU(0), DG with block Jacobi): every
  _iterations.csv row, the summary and a strided sample of the final state.

* solution_*.npz -- the solution files of Problem::Save (src/problem.cpp:762)
  as the reference command line writes them: the .mesh text, the four .gf
  texts and the final coefficients, per form.

Usage:  python tests/golden/make_golden.py
            [--only CLI_CASE ... | --trajectories | --condense | --c2 [CASE ...] | --solution]
"""
from __future__ import annotations

import csv
import ctypes as C
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF = ROOT / "oracle" / "_ref"
DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)


def ptr(a):
    return a.ctypes.data_as(DP)


def load_ref():
    lib = C.CDLL(str(REF / "libeuler_ref.so"))
    lib.ref_problem_new.restype = C.c_void_p
    lib.ref_problem_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                    C.c_int, C.c_int, C.c_int, C.c_double]
    lib.ref_last_error.restype = C.c_char_p
    lib.ref_cell_norm.restype = C.c_double
    for name in ["ref_problem_free", "ref_sizes", "ref_geometry", "ref_tables", "ref_initial",
                 "ref_freeze", "ref_set_old", "ref_set_dt", "ref_residual", "ref_cell_norm",
                 "ref_admissible", "ref_dg_apply", "ref_dg_jacobi_blocks", "ref_hdg_condense",
                 "ref_schur_apply", "ref_schur_jacobi_blocks", "ref_recover", "ref_linear_solve",
                 "ref_ilu", "ref_set_precond"]:
        getattr(lib, name).argtypes = None
    lib.ref_problem_free.argtypes = [C.c_void_p]
    lib.ref_sizes.argtypes = [C.c_void_p, IP]
    lib.ref_geometry.argtypes = [C.c_void_p, DP]
    lib.ref_tables.argtypes = [C.c_void_p, DP, DP, DP, DP, DP, DP, DP, IP]
    lib.ref_initial.argtypes = [C.c_void_p, DP]
    lib.ref_freeze.argtypes = [C.c_void_p, DP, C.c_double, C.c_int, DP, DP, DP]
    lib.ref_set_old.argtypes = [C.c_void_p, DP]
    lib.ref_set_dt.argtypes = [C.c_void_p, C.c_double]
    lib.ref_residual.argtypes = [C.c_void_p, DP, DP]
    lib.ref_cell_norm.argtypes = [C.c_void_p, DP]
    lib.ref_admissible.argtypes = [C.c_void_p, DP]
    lib.ref_dg_apply.argtypes = [C.c_void_p, DP, DP, DP]
    lib.ref_dg_jacobi_blocks.argtypes = [C.c_void_p, DP, DP]
    lib.ref_hdg_condense.argtypes = [C.c_void_p, DP, DP, DP, DP, DP, DP]
    lib.ref_schur_apply.argtypes = [C.c_void_p, DP, DP]
    lib.ref_schur_jacobi_blocks.argtypes = [C.c_void_p, DP]
    lib.ref_recover.argtypes = [C.c_void_p, DP, DP]
    lib.ref_linear_solve.argtypes = [C.c_void_p, C.c_int, DP, DP, DP, DP, IP, DP]
    lib.ref_ilu.argtypes = [C.c_void_p, C.c_int, DP, DP, DP, DP, DP, IP]
    lib.ref_set_precond.argtypes = [C.c_void_p, C.c_int]
    lib.ref_trajectory.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.c_int, C.c_int, DP, DP, DP, IP]
    return lib


def check(lib, rc):
    if rc:
        raise RuntimeError(lib.ref_last_error().decode())


# (nx, ny, k, alpha_deg, store_dense): small meshes cover every degree;
# 16x16 Q3 is the headline workload's mesh.
UNIT_CASES = [
    (3, 2, 0, 45.0, True), (3, 2, 1, 45.0, True), (4, 3, 2, 30.0, True), (3, 3, 3, 60.0, True),
    (16, 16, 3, 45.0, False), (4, 4, 4, 30.0, True), (3, 2, 5, 45.0, False), (2, 3, 6, 52.0, False),
    (2, 2, 7, 41.0, False), (2, 2, 8, 37.0, False),
]


def make_unit(lib, nx, ny, k, alpha, dense, rng):
    h = lib.ref_problem_new(nx, ny, k, alpha, 1.1, 0, 0, 20, 1500, 1e-12)
    if not h:
        raise RuntimeError(lib.ref_last_error().decode())
    try:
        sz = np.zeros(7, np.int32)
        lib.ref_sizes(h, sz.ctypes.data_as(IP))
        n, p, m, t, nf, nu, nl = map(int, sz)
        q = k + 1
        geo = np.zeros(5)
        lib.ref_geometry(h, ptr(geo))
        w, ew, im, ms = np.zeros(p), np.zeros(q), np.zeros(p), np.zeros(p)
        tdx, tdy, fv = np.zeros(q * q), np.zeros(q * q), np.zeros(4 * q * p)
        tn = np.zeros(p, np.int32)
        lib.ref_tables(h, ptr(w), ptr(ew), ptr(im), ptr(ms), ptr(tdx), ptr(tdy), ptr(fv),
                       tn.ctypes.data_as(IP))
        u0 = np.zeros(nu)
        check(lib, lib.ref_initial(h, ptr(u0)))
        # Coarse meshes can make the projected wave inadmissible at face
        # points; blend toward the mean state as the reference's --verify does
        # (src/verification.cpp:26-30) until the state is admissible, then
        # apply a seeded node-wise perturbation.
        background = np.tile(u0.reshape(-1, 4).mean(axis=0), nu // 4)
        node_scale = np.repeat(1.0 + 0.01 * np.sin(0.37 * np.arange(nu // 4) + 0.3), 4)
        noise = 1e-5 * rng.standard_normal(nu)
        for blend in (1.0, 0.5, 0.2, 0.05):
            base = blend * u0 + (1 - blend) * background
            u = base * node_scale + noise * np.abs(base)
            if lib.ref_admissible(h, ptr(u)):
                break
        else:
            raise RuntimeError("no admissible perturbed state")
        dt = 0.05 * min(geo[2], geo[3])
        a, b, rate = np.zeros(nf * q), np.zeros(nf * q), np.zeros(1)
        check(lib, lib.ref_freeze(h, ptr(u), dt, 1, ptr(a), ptr(b), ptr(rate)))
        old = u0.copy()
        check(lib, lib.ref_set_old(h, ptr(old)))
        lib.ref_set_dt(h, dt)
        r = np.zeros(nu)
        check(lib, lib.ref_residual(h, ptr(u), ptr(r)))
        x = rng.standard_normal(nu)
        jx = np.zeros(nu)
        check(lib, lib.ref_dg_apply(h, ptr(u), ptr(x), ptr(jx)))
        out = dict(nx=nx, ny=ny, k=k, alpha=alpha, dt=dt, blend=blend, geometry=geo, w=w, ew=ew, inv_mass=im,
                   mass=ms, tensor_dx=tdx, tensor_dy=tdy, fv=fv, tensor_node=tn, u0=u0, u=u, old=old,
                   a=a, b=b, rate=rate, r=r, x=x, jx=jx,
                   r_norm=np.array([lib.ref_cell_norm(h, ptr(r))]))
        if dense:
            blocks = np.zeros(n * m * m)
            check(lib, lib.ref_dg_jacobi_blocks(h, ptr(u), ptr(blocks)))
            out["dg_blocks"] = blocks
        rhs, X, y, D = np.zeros(nl), np.zeros(n * m * 4 * t), np.zeros(nu), np.zeros(nl)
        check(lib, lib.ref_hdg_condense(h, ptr(u), ptr(r), ptr(rhs), ptr(X), ptr(y), ptr(D)))
        out.update(rhs=rhs, y_hdg=y, D=D)
        if dense:
            out["X"] = X
            sblocks = np.zeros(nf * t * t)
            check(lib, lib.ref_schur_jacobi_blocks(h, ptr(sblocks)))
            out["schur_blocks"] = sblocks
        v = rng.standard_normal(nl)
        sv = np.zeros(nl)
        check(lib, lib.ref_schur_apply(h, ptr(v), ptr(sv)))
        lam = rng.standard_normal(nl)
        du = np.zeros(nu)
        check(lib, lib.ref_recover(h, ptr(lam), ptr(du)))
        out.update(v=v, sv=sv, lam=lam, du=du)
        for form, (rhs_f, N) in {0: (-r, nu), 1: (rhs, nl)}.items():
            rr = np.ascontiguousarray(rhs_f)
            xs, eq = np.zeros(N), np.zeros(N)
            cnt, rel = np.zeros(1, np.int32), np.zeros(1)
            check(lib, lib.ref_linear_solve(h, form, ptr(u), ptr(rr), ptr(xs), ptr(eq),
                                            cnt.ctypes.data_as(IP), ptr(rel)))
            tag = "dg" if form == 0 else "hdg"
            out[f"solve_{tag}_x"] = xs
            out[f"solve_{tag}_count"] = cnt
            out[f"solve_{tag}_relres"] = rel
        # block ILU(0) of both forms: the preconditioner apply on a seeded
        # vector, the filled and factored BSR blocks on the small cases, and
        # one GMRES solve per form with block-ilu0 (block_ilu.cpp, linear.cpp)
        irng = np.random.default_rng([20261204, nx, ny, k])  # own stream: other draws unchanged
        for form, (tag, B, rows) in {0: ("dg", m, n), 1: ("hdg", t, nf)}.items():
            nz = np.zeros(1, np.int32)
            check(lib, lib.ref_ilu(h, form, ptr(u), None, None, None, None, nz.ctypes.data_as(IP)))
            nnzb = int(nz[0])
            bvec = irng.standard_normal(rows * B)
            xv = np.zeros(rows * B)
            filled, factored = np.zeros(nnzb * B * B), np.zeros(nnzb * B * B)
            check(lib, lib.ref_ilu(h, form, ptr(u), ptr(bvec), ptr(xv), ptr(filled), ptr(factored),
                                   nz.ctypes.data_as(IP)))
            out[f"ilu_{tag}_b"] = bvec
            out[f"ilu_{tag}_x"] = xv
            if (form == 0 and k <= 2) or (form == 1 and dense and k <= 3):
                out[f"ilu_{tag}_filled"] = filled
                out[f"ilu_{tag}_factored"] = factored
        lib.ref_set_precond(h, 1)
        for form, (rhs_f, N) in {0: (-r, nu), 1: (rhs, nl)}.items():
            rr = np.ascontiguousarray(rhs_f)
            xs, eq = np.zeros(N), np.zeros(N)
            cnt, rel = np.zeros(1, np.int32), np.zeros(1)
            check(lib, lib.ref_linear_solve(h, form, ptr(u), ptr(rr), ptr(xs), ptr(eq),
                                            cnt.ctypes.data_as(IP), ptr(rel)))
            tag = "dg" if form == 0 else "hdg"
            out[f"solve_{tag}_ilu_x"] = xs
            out[f"solve_{tag}_ilu_count"] = cnt
            out[f"solve_{tag}_ilu_relres"] = rel
        lib.ref_set_precond(h, 0)
        return out
    finally:
        lib.ref_problem_free(h)


def ref_cli() -> Path:
    v4 = REF / "euler2d_ref_v4"
    try:
        subprocess.run([str(v4), "--help"], capture_output=True, check=True)
        return v4
    except (OSError, subprocess.CalledProcessError):
        return REF / "euler2d_ref_v3"


# name -> argument list (the reference's code tests and the 16x16 Q3 workload)
CLI_CASES = {
    "c1_16x16_q3": ["--nx", "16", "--ny", "16", "--k", "3", "--alpha-deg", "45", "--cfl", "1",
                    "--steps", "3", "--newton-steps", "3", "--form", "both", "--assembly", "partial",
                    "--precond", "block-jacobi"],
    "be1_8x8_q2": ["--nx", "8", "--ny", "8", "--k", "2", "--alpha-deg", "45", "--cfl", "1",
                   "--steps", "1", "--newton-steps", "1", "--integrator", "be", "--form", "both"],
    "smoke_8x8_q1": ["--nx", "8", "--ny", "8", "--k", "1", "--cfl", ".1", "--steps", "1",
                     "--form", "both", "--newton-tol", "1e-12", "--linear-tol", "1e-12"],
    "ilu_8x8_q2": ["--nx", "8", "--ny", "8", "--k", "2", "--alpha-deg", "30", "--cfl", "1", "--steps", "1",
                   "--newton-steps", "2", "--form", "both", "--precond", "block-ilu0"],
    "be_converged_8x8_q2": ["--nx", "8", "--ny", "8", "--k", "2", "--cfl", ".1", "--steps", "1",
                            "--integrator", "be", "--form", "both", "--check-update",
                            "--newton-tol", "1e-12", "--linear-tol", "1e-12"],
    # element and full assembly (src/options.cpp:130-146): element-assembled
    # operators applied matrix-free, and GMRES on the assembled CSR matrix
    "element_8x8_q2": ["--nx", "8", "--ny", "8", "--k", "2", "--alpha-deg", "30", "--cfl", "1",
                       "--steps", "1", "--newton-steps", "2", "--form", "both", "--assembly", "element"],
    "full_8x8_q2": ["--nx", "8", "--ny", "8", "--k", "2", "--alpha-deg", "30", "--cfl", "1",
                    "--steps", "1", "--newton-steps", "2", "--form", "both", "--assembly", "full"],
    "full_ilu_8x8_q2": ["--nx", "8", "--ny", "8", "--k", "2", "--alpha-deg", "30", "--cfl", "1",
                        "--steps", "1", "--newton-steps", "2", "--form", "both", "--assembly", "full",
                        "--precond", "block-ilu0"],
    # dense direct LU of the full assembly (src/linear.cpp:46-49, 204-206, 224-225)
    "dense_8x8_q2": ["--nx", "8", "--ny", "8", "--k", "2", "--alpha-deg", "30", "--cfl", "1",
                     "--steps", "1", "--newton-steps", "2", "--form", "both", "--solver", "dense"],
}
ITER_COLS = ["step", "stage", "newton", "time", "dt", "cfl", "residual_physical_rms", "damping",
             "krylov_iterations", "linear_relative_residual", "dg_linear_relative_residual",
             "update_check_relative"]
SUMMARY_COLS = ["T", "actual_max_cfl", "mean_dt", "volume_dofs", "trace_dofs", "time_steps",
                "newton_updates", "rho_L2", "rhou_L2", "rhov_L2", "energy_L2", "max_conservation_drift"]


def ref_initial_state(lib, args: list[str]) -> np.ndarray:
    def opt(flag, default):
        return type(default)(args[args.index(flag) + 1]) if flag in args else default
    nx, ny, k, alpha = opt("--nx", 100), opt("--ny", 100), opt("--k", 1), opt("--alpha-deg", 45.0)
    h = lib.ref_problem_new(nx, ny, k, alpha, 1.1, 0, 0, 20, 1500, 1e-12)
    try:
        sz = np.zeros(7, np.int32)
        lib.ref_sizes(h, sz.ctypes.data_as(IP))
        u0 = np.zeros(int(sz[5]))
        check(lib, lib.ref_initial(h, ptr(u0)))
        return u0
    finally:
        lib.ref_problem_free(h)


def make_cli(exe: Path, name: str, args: list[str]) -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        prefix = Path(tmp) / "run"
        proc = subprocess.run([str(exe), *args, "--output", str(prefix)], capture_output=True, text=True)
        if proc.returncode:
            raise RuntimeError(f"{name}: {proc.stderr}")
        out = {"args": np.array(json.dumps(args))}
        for form in ("dg", "hdg"):
            coeff = np.loadtxt(f"{prefix}_{form}_coefficients.csv", delimiter=",", skiprows=1)
            out[f"{form}_u"] = coeff[:, 2:].reshape(-1)
            with open(f"{prefix}_{form}_iterations.csv", newline="") as fh:
                rows = list(csv.DictReader(fh))
            out[f"{form}_iterations"] = np.array([[float(r[c]) for c in ITER_COLS] for r in rows])
            with open(f"{prefix}_{form}_summary.csv", newline="") as fh:
                row = next(csv.DictReader(fh))
            out[f"{form}_summary"] = np.array([float(row[c]) for c in SUMMARY_COLS])
        with open(f"{prefix}_comparison.csv", newline="") as fh:
            row = next(csv.DictReader(fh))
        out["comparison"] = np.array([float(v) for v in row.values()])
        return out


# a non-square mesh so that vertex, element and boundary numbering are all visible
SOLUTION_ARGS = ["--nx", "8", "--ny", "6", "--k", "2", "--alpha-deg", "30", "--cfl", "1",
                 "--steps", "1", "--newton-steps", "2", "--form", "both"]
GF_NAMES = ("rho", "rhou", "rhov", "energy")


def make_solution(exe: Path) -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        prefix = Path(tmp) / "run"
        proc = subprocess.run([str(exe), *SOLUTION_ARGS, "--output", str(prefix)],
                              capture_output=True, text=True)
        if proc.returncode:
            raise RuntimeError(f"solution: {proc.stderr}")
        out = {"args": np.array(json.dumps(SOLUTION_ARGS))}
        for form in ("dg", "hdg"):
            out[f"{form}_mesh"] = np.array(Path(f"{prefix}_{form}.mesh").read_text())
            for name in GF_NAMES:
                out[f"{form}_{name}_gf"] = np.array(Path(f"{prefix}_{form}_{name}.gf").read_text())
            coeff = np.loadtxt(f"{prefix}_{form}_coefficients.csv", delimiter=",", skiprows=1)
            out[f"{form}_u"] = coeff[:, 2:].reshape(-1)
        return out


# (nx, ny, k, alpha_deg): high degrees on meshes with more cells than the
# condensation launches CTAs (two per SM for k = 5, 6 and one for k = 7, 8 on
# 148 SMs), so that CTAs reduce several cells each (condense_*.npz)
CONDENSE_CASES = [(18, 18, 5, 33.0), (18, 18, 6, 47.0), (13, 13, 7, 58.0), (13, 13, 8, 26.0)]


def make_condense(lib, nx, ny, k, alpha, seed):
    """Condensed HDG pieces at a perturbed state: StreamCondense's rhs, y and
    D, the Schur action on a seeded vector and the recovery of another
    (condensation.cpp:131-163, operators.cpp:147). The vectors v and lam are
    regenerated from `seed` by numpy.random.default_rng; old is the initial
    projection."""
    h = lib.ref_problem_new(nx, ny, k, alpha, 1.1, 0, 0, 20, 1500, 1e-12)
    if not h:
        raise RuntimeError(lib.ref_last_error().decode())
    try:
        sz = np.zeros(7, np.int32)
        lib.ref_sizes(h, sz.ctypes.data_as(IP))
        n, p, m, t, nf, nu, nl = map(int, sz)
        geo = np.zeros(5)
        lib.ref_geometry(h, ptr(geo))
        u0 = np.zeros(nu)
        check(lib, lib.ref_initial(h, ptr(u0)))
        rng = np.random.default_rng(seed)
        u = u0 * np.repeat(1.0 + 0.01 * np.sin(0.37 * np.arange(nu // 4) + 0.3), 4)
        u = u + 1e-5 * rng.standard_normal(nu) * np.abs(u)
        if not lib.ref_admissible(h, ptr(u)):
            raise RuntimeError("perturbed state not admissible")
        dt = 0.05 * min(geo[2], geo[3])
        a, b, rate = np.zeros(nf * (k + 1)), np.zeros(nf * (k + 1)), np.zeros(1)
        check(lib, lib.ref_freeze(h, ptr(u), dt, 1, ptr(a), ptr(b), ptr(rate)))
        check(lib, lib.ref_set_old(h, ptr(u0)))
        lib.ref_set_dt(h, dt)
        r = np.zeros(nu)
        check(lib, lib.ref_residual(h, ptr(u), ptr(r)))
        rhs, X, y, D = np.zeros(nl), np.zeros(n * m * 4 * t), np.zeros(nu), np.zeros(nl)
        check(lib, lib.ref_hdg_condense(h, ptr(u), ptr(r), ptr(rhs), ptr(X), ptr(y), ptr(D)))
        vrng = np.random.default_rng([seed, 1])
        v, lam = vrng.standard_normal(nl), vrng.standard_normal(nl)
        sv, du = np.zeros(nl), np.zeros(nu)
        check(lib, lib.ref_schur_apply(h, ptr(v), ptr(sv)))
        check(lib, lib.ref_recover(h, ptr(lam), ptr(du)))
        return dict(nx=nx, ny=ny, k=k, alpha=alpha, dt=dt, seed=seed, u=u, rhs=rhs, y_hdg=y, D=D, sv=sv, du=du)
    finally:
        lib.ref_problem_free(h)


# The headline 128x128 Q4 workload (5 SSP-DIRK3 steps x 3 Newton updates per
# stage), one form and preconditioner per case. Its final states are 13 MB
# each, so the fixture keeps every _iterations.csv row, the summary row, the
# per-component sums of squares of the final state and every STRIDE-th
# coefficient of it (c2_*.npz).
C2_ARGS = ["--nx", "128", "--ny", "128", "--k", "4", "--alpha-deg", "30", "--cfl", "1", "--steps", "5",
           "--newton-steps", "3", "--assembly", "partial"]
C2_CASES = {
    "hdg_jacobi": ["--form", "hdg", "--precond", "block-jacobi"],
    "hdg_ilu0": ["--form", "hdg", "--precond", "block-ilu0"],
    "dg_jacobi": ["--form", "dg", "--precond", "block-jacobi"],
}
C2_STRIDE = 32


def make_c2(exe: Path, names: list[str]) -> None:
    """Run the reference command line on the c2 cases in parallel (one
    process each) and write c2_<name>.npz."""
    with tempfile.TemporaryDirectory() as tmp:
        procs = {}
        for name in names:
            prefix = Path(tmp) / name
            args = C2_ARGS + C2_CASES[name]
            procs[name] = (args, prefix, subprocess.Popen([str(exe), *args, "--output", str(prefix)],
                                                          stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                                          text=True))
        for name, (args, prefix, proc) in procs.items():
            _, err = proc.communicate()
            if proc.returncode:
                raise RuntimeError(f"c2 {name}: {err}")
            form = args[args.index("--form") + 1]
            coeff = np.loadtxt(f"{prefix}_{form}_coefficients.csv", delimiter=",", skiprows=1)
            u = coeff[:, 2:].reshape(-1)
            with open(f"{prefix}_{form}_iterations.csv", newline="") as fh:
                rows = list(csv.DictReader(fh))
            with open(f"{prefix}_{form}_summary.csv", newline="") as fh:
                summ = next(csv.DictReader(fh))
            out = {"args": np.array(json.dumps(args)), "stride": np.array([C2_STRIDE]),
                   "iterations": np.array([[float(r[c]) for c in ITER_COLS] for r in rows]),
                   "summary": np.array([float(summ[c]) for c in SUMMARY_COLS]),
                   "u_sample": u[::C2_STRIDE].copy(), "u_size": np.array([u.size]),
                   "u_component_sumsq": (u.reshape(-1, 4) ** 2).sum(axis=0),
                   "mean_newton_s": np.array([float(summ["mean_newton_s"])])}
            np.savez_compressed(HERE / f"c2_{name}.npz", **out)
            print("c2", name, len(rows), "updates")


# command-line cases whose every Newton update is recorded (traj_*.npz)
TRAJ_CASES = ["c1_16x16_q3"]


def make_trajectory(lib, name: str) -> dict:
    """Newton direction du and damping of every accepted update of both forms
    (oracle/ref_harness.cpp ref_trajectory), pinned to the command line: the
    trajectory's final state must equal the cli_<name>.npz final state."""
    args = CLI_CASES[name]
    argv = (C.c_char_p * len(args))(*[a.encode() for a in args])
    cli = np.load(HERE / f"cli_{name}.npz")
    u0 = cli["u0"]
    nu = u0.size
    out = {"args": np.array(json.dumps(args))}
    for hdg, tag in ((0, "dg"), (1, "hdg")):
        cap = 4096
        du = np.zeros(cap * nu)
        damping = np.zeros(cap)
        u_final = np.zeros(nu)
        cnt = np.zeros(1, np.int32)
        check(lib, lib.ref_trajectory(len(args), argv, hdg, cap, ptr(du), ptr(damping), ptr(u_final),
                                      cnt.ctypes.data_as(IP)))
        n = int(cnt[0])
        ref_u = cli[f"{tag}_u"]
        err = np.linalg.norm(u_final - ref_u) / np.linalg.norm(ref_u)
        # the command-line fixture may come from the AVX-512 build and the
        # harness library from the AVX2 one: vectorisation changes rounding only
        if err > 1e-13:
            raise RuntimeError(f"{name} {tag}: trajectory final state differs from the command line ({err:.3e})")
        out[f"{tag}_final_vs_cli"] = np.array([err])
        if n != len(cli[f"{tag}_iterations"]):
            raise RuntimeError(f"{name} {tag}: {n} updates against {len(cli[f'{tag}_iterations'])} CSV rows")
        out[f"{tag}_du"] = du[: n * nu].reshape(n, nu)
        out[f"{tag}_damping"] = damping[:n]
    return out


def main():
    if not (REF / "libeuler_ref.so").exists():
        sys.exit("oracle/_ref is not built: run `make -C oracle` where the reference is available")
    lib = load_ref()
    only = sys.argv[sys.argv.index("--only") + 1:] if "--only" in sys.argv else None
    if "--c2" in sys.argv:  # the 128x128 Q4 cases (several CPU minutes each, run in parallel)
        names = sys.argv[sys.argv.index("--c2") + 1:] or list(C2_CASES)
        make_c2(ref_cli(), names)
        return
    if "--solution" in sys.argv:  # regenerate just the solution files
        np.savez_compressed(HERE / "solution_8x6_q2.npz", **make_solution(ref_cli()))
        print("solution 8x6 q2")
        return
    if "--condense" in sys.argv:  # regenerate just the high-degree condensation cases
        for i, (nx, ny, k, alpha) in enumerate(CONDENSE_CASES):
            np.savez_compressed(HERE / f"condense_{nx}x{ny}_k{k}.npz",
                                **make_condense(lib, nx, ny, k, alpha, 7000 + i))
            print("condense", nx, ny, k)
        return
    if "--trajectories" in sys.argv:  # regenerate just the per-update trajectories
        for name in TRAJ_CASES:
            np.savez_compressed(HERE / f"traj_{name}.npz", **make_trajectory(lib, name))
            print("trajectory", name)
        return
    if only:  # regenerate just the named command-line cases (and the manifest)
        exe = ref_cli()
        for name in only:
            data = make_cli(exe, name, CLI_CASES[name])
            data["u0"] = ref_initial_state(lib, CLI_CASES[name])
            np.savez_compressed(HERE / f"cli_{name}.npz", **data)
            print("cli", name)
        meta = json.loads((HERE / "manifest.json").read_text())
        meta["cli_cases"] = CLI_CASES
        (HERE / "manifest.json").write_text(json.dumps(meta, indent=1))
        return
    rng = np.random.default_rng(20261203)
    for nx, ny, k, alpha, dense in UNIT_CASES:
        data = make_unit(lib, nx, ny, k, alpha, dense, rng)
        np.savez_compressed(HERE / f"units_{nx}x{ny}_k{k}.npz", **data)
        print("unit", nx, ny, k)
    exe = ref_cli()
    for name, args in CLI_CASES.items():
        data = make_cli(exe, name, args)
        data["u0"] = ref_initial_state(lib, args)
        np.savez_compressed(HERE / f"cli_{name}.npz", **data)
        print("cli", name)
    for name in TRAJ_CASES:
        np.savez_compressed(HERE / f"traj_{name}.npz", **make_trajectory(lib, name))
        print("trajectory", name)
    for i, (nx, ny, k, alpha) in enumerate(CONDENSE_CASES):
        np.savez_compressed(HERE / f"condense_{nx}x{ny}_k{k}.npz", **make_condense(lib, nx, ny, k, alpha, 7000 + i))
        print("condense", nx, ny, k)
    np.savez_compressed(HERE / "solution_8x6_q2.npz", **make_solution(exe))
    print("solution 8x6 q2")
    meta = {"iteration_columns": ITER_COLS, "summary_columns": SUMMARY_COLS,
            "unit_cases": UNIT_CASES, "cli_cases": CLI_CASES}
    (HERE / "manifest.json").write_text(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
