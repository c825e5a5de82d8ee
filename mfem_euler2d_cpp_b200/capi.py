"""ctypes binding of the C-ABI in include/euler2d_cuda.h.

This is the reference-facing boundary seen from Python: plain pointers and
sizes, int status codes mapped to the reference's error messages. There is no
CPU fallback: importing succeeds without a GPU (the library loads), but every
compute call needs a CUDA device and raises EngineError otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "lib" / "libeuler2d_cuda.so"
HEADER_PATH = _PKG.parent / "include" / "euler2d_cuda.h"

MAX_Q = 9
MAX_P = MAX_Q * MAX_Q

# status codes (enum eg_status)
OK = 0
STATUS_NAMES = {
    0: "EG_OK", 1: "EG_ERR_INVALID", 2: "EG_ERR_CUDA", 3: "EG_ERR_NONPOSITIVE_FACE",
    4: "EG_ERR_ROE_SOUND", 5: "EG_ERR_DEGENERATE_HLL", 6: "EG_ERR_INADMISSIBLE",
    7: "EG_ERR_SINGULAR_CELL", 8: "EG_ERR_SINGULAR_JACOBI", 9: "EG_ERR_SINGULAR_ILU",
    10: "EG_ERR_GMRES_BREAKDOWN", 11: "EG_ERR_GMRES_NONFINITE", 12: "EG_ERR_GMRES_LIMIT",
    13: "EG_ERR_LINEAR_RESIDUAL", 14: "EG_ERR_RECOVERED", 15: "EG_ERR_DG_LINEAR",
    16: "EG_ERR_LINE_SEARCH", 17: "EG_ERR_OUT_OF_MEMORY", 18: "EG_ERR_STEP_INTERVAL",
    19: "EG_ERR_NEWTON_CONVERGE", 20: "EG_ERR_DIRK_INADMISSIBLE", 21: "EG_ERR_INITIAL",
    22: "EG_ERR_UPDATE_EQUATION", 23: "EG_ERR_UPDATE_EQUIVALENCE", 24: "EG_ERR_WAIT_LIMIT",
    25: "EG_ERR_CONTEXT_LOST",
}
FORM_DG, FORM_HDG = 0, 1
SOLVER_GMRES, SOLVER_DENSE = 0, 1
PC_JACOBI, PC_ILU0 = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
ASSEMBLY_PARTIAL, ASSEMBLY_FULL, ASSEMBLY_ELEMENT = 0, 1, 2
SLOT = dict(U=0, OLD=1, R=2, DU=3, RHS=4, LAMBDA=5, D=6, X=7, Y=8, PC_BLOCKS=9, HLL_A=10, HLL_B=11)


class EngineError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Desc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("k", C.c_int),
        ("gamma", C.c_double), ("safety", C.c_double), ("alpha", C.c_double),
        ("lx", C.c_double), ("ly", C.c_double), ("hx", C.c_double), ("hy", C.c_double),
        ("area", C.c_double),
        ("w", C.c_double * MAX_P), ("ew", C.c_double * MAX_Q), ("ex", C.c_double * MAX_Q),
        ("inv_mass", C.c_double * MAX_P), ("mass", C.c_double * MAX_P),
        ("tensor_dx", C.c_double * MAX_P), ("tensor_dy", C.c_double * MAX_P),
        ("face_basis", C.c_double * (4 * MAX_Q * MAX_Q)),
        ("tensor_node", C.c_int * MAX_P),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("form", C.c_int), ("precond", C.c_int), ("assembly", C.c_int), ("precision", C.c_int),
        ("restart", C.c_int), ("max_krylov", C.c_int), ("linear_tol", C.c_double),
        ("check_update", C.c_int), ("solver", C.c_int),
    ]


class UpdateStats(C.Structure):
    _fields_ = [
        ("residual_norm", C.c_double), ("damping", C.c_double),
        ("krylov_iterations", C.c_int), ("attempts", C.c_int),
        ("linear_relative_residual", C.c_double), ("dg_linear_relative_residual", C.c_double),
        ("residual_s", C.c_double), ("validation_s", C.c_double), ("jacobian_s", C.c_double),
        ("condensation_s", C.c_double), ("assembly_s", C.c_double), ("setup_s", C.c_double),
        ("solve_s", C.c_double), ("recovery_s", C.c_double), ("line_search_s", C.c_double),
        ("iteration_s", C.c_double), ("device_ms", C.c_double), ("update_check", C.c_double),
    ]


class LinearStats(C.Structure):
    _fields_ = [("count", C.c_int), ("residual", C.c_double), ("rhs_norm", C.c_double)]


class RunOpts(C.Structure):
    _fields_ = [
        ("integrator", C.c_int), ("steps", C.c_int), ("newton_steps", C.c_int),
        ("max_newton", C.c_int), ("dt", C.c_double), ("cfl", C.c_double), ("end", C.c_double),
        ("tol", C.c_double), ("timing_only", C.c_int), ("save_solution", C.c_int),
        ("prefix", C.c_char_p), ("form_name", C.c_char_p), ("assembly_name", C.c_char_p),
        ("solver_name", C.c_char_p), ("precond_name", C.c_char_p),
        ("ilu_ordering_name", C.c_char_p), ("check_update", C.c_int),
    ]


class RunResult(C.Structure):
    _fields_ = [
        ("errors", C.c_double * 4), ("seconds", C.c_double), ("drift", C.c_double),
        ("newton_seconds", C.c_double), ("final_time", C.c_double), ("mean_newton_s", C.c_double),
        ("newton_device_ms", C.c_double), ("updates", C.c_int), ("time_steps", C.c_int),
    ]


class BatchStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("updates", C.c_longlong), ("failed", C.c_int)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("workers", C.c_int), ("budget_bytes", C.c_longlong),
                ("keep_contexts", C.c_int), ("keep_states", C.c_int)]


class Request(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("k", C.c_int), ("alpha_deg", C.c_double),
                ("steps", C.c_int), ("newton_steps", C.c_int), ("cfl", C.c_double),
                ("form", C.c_int), ("precond", C.c_int), ("precision", C.c_int)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("updates", C.c_int), ("submit_s", C.c_double), ("start_s", C.c_double),
                ("finish_s", C.c_double), ("final_time", C.c_double), ("errors", C.c_double * 4),
                ("drift", C.c_double), ("bytes", C.c_longlong)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_longlong), ("failed", C.c_longlong), ("peak_bytes", C.c_longlong),
                ("peak_running", C.c_int)]


_lib = None
_DP = C.POINTER(C.c_double)


def load() -> C.CDLL:
    """Load the in-tree engine; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"CUDA engine not built: {LIB_PATH} missing (run __graft_entry__.build())")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "eg_desc_simple_wave": (C.c_int, [C.POINTER(Desc), C.c_int, C.c_int, C.c_int, C.c_double,
                                          C.c_double, C.c_double]),
        "eg_opts_default": (None, [C.POINTER(Opts)]),
        "eg_set_device": (C.c_int, [C.c_int]),
        "eg_profile_enable": (C.c_int, [vp, C.c_int]),
        "eg_profile_reset": (C.c_int, [vp]),
        "eg_profile_query": (C.c_int, [vp, C.c_int, _DP, C.POINTER(C.c_longlong)]),
        "eg_launch_count": (C.c_longlong, [vp]),
        "eg_set_ilu_wait": (C.c_int, [vp, C.c_ulonglong, C.c_int]),
        "eg_check_pivot_reciprocal": (C.c_int, [_DP, _DP, C.c_longlong]),
        "eg_cell_norm_noalloc": (C.c_int, [C.POINTER(Desc), C.c_void_p, C.c_void_p, _DP]),
        "eg_create": (C.c_int, [C.POINTER(Desc), C.POINTER(Opts), C.POINTER(vp)]),
        "eg_destroy": (None, [vp]),
        "eg_last_error": (C.c_char_p, [vp]),
        "eg_status_string": (C.c_char_p, [C.c_int]),
        "eg_stream": (vp, [vp]),
        "eg_set_opts": (C.c_int, [vp, C.POINTER(Opts)]),
        "eg_sizes": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "eg_device_bytes": (C.c_longlong, [vp]),
        "eg_upload": (C.c_int, [vp, C.c_int, _DP]),
        "eg_download": (C.c_int, [vp, C.c_int, _DP]),
        "eg_initial": (C.c_int, [vp]),
        "eg_freeze": (C.c_int, [vp, C.c_double, C.c_int, _DP]),
        "eg_set_dt": (C.c_int, [vp, C.c_double]),
        "eg_residual": (C.c_int, [vp]),
        "eg_cell_norm": (C.c_int, [vp, C.c_int, _DP]),
        "eg_admissible": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int)]),
        "eg_dg_apply": (C.c_int, [vp, _DP, _DP]),
        "eg_condense": (C.c_int, [vp]),
        "eg_schur_apply": (C.c_int, [vp, _DP, _DP]),
        "eg_recover": (C.c_int, [vp, _DP, _DP]),
        "eg_pc_factor": (C.c_int, [vp, C.c_int]),
        "eg_pc_apply": (C.c_int, [vp, _DP, _DP]),
        "eg_pc_size": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
        "eg_linear_solve": (C.c_int, [vp, _DP, _DP, _DP, C.c_int, C.c_double,
                                      C.POINTER(LinearStats)]),
        "eg_stage_begin": (C.c_int, [vp, C.c_double]),
        "eg_newton_residual": (C.c_int, [vp, _DP]),
        "eg_newton_update": (C.c_int, [vp, C.c_double, C.c_double, C.POINTER(UpdateStats)]),
        "eg_integral": (C.c_int, [vp, _DP]),
        "eg_errors": (C.c_int, [vp, C.c_double, _DP]),
        "eg_differences": (C.c_int, [C.POINTER(Desc), _DP, _DP, _DP]),
        "eg_save_solution": (C.c_int, [C.POINTER(Desc), _DP, C.c_char_p]),
        "eg_state_differences": (C.c_int, [vp, _DP, _DP]),
        "eg_run": (C.c_int, [vp, C.POINTER(RunOpts), C.POINTER(RunResult)]),
        "eg_stepper_create": (C.c_int, [vp, C.POINTER(RunOpts), C.POINTER(vp)]),
        "eg_stepper_next": (C.c_int, [vp, C.POINTER(UpdateStats)]),
        "eg_stepper_destroy": (None, [vp]),
        "eg_stepper_finish": (C.c_int, [vp, C.POINTER(RunResult)]),
        "eg_batch_create": (C.c_int, [C.c_int, C.POINTER(Desc), C.POINTER(Opts), C.c_int, C.POINTER(vp)]),
        "eg_batch_run": (C.c_int, [vp, C.POINTER(RunOpts), C.c_int, C.POINTER(BatchStats)]),
        "eg_batch_result": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(RunResult)]),
        "eg_batch_context": (vp, [vp, C.c_int]),
        "eg_batch_destroy": (None, [vp]),
        "eg_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(vp)]),
        "eg_server_submit": (C.c_int, [vp, C.POINTER(Request), C.POINTER(C.c_longlong)]),
        "eg_server_poll": (C.c_int, [vp, C.c_longlong, C.POINTER(RequestResult)]),
        "eg_server_state": (C.c_int, [vp, C.c_longlong, _DP]),
        "eg_server_drain": (C.c_int, [vp, C.POINTER(ServerStats)]),
        "eg_server_clock": (C.c_double, [vp]),
        "eg_server_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def simple_wave_desc(nx: int, ny: int, k: int, alpha_deg: float, gamma: float = 3.0,
                     safety: float = 1.1) -> Desc:
    lib = load()
    d = Desc()
    rc = lib.eg_desc_simple_wave(C.byref(d), nx, ny, k, alpha_deg, gamma, safety)
    if rc != OK:
        raise EngineError(rc, "invalid simple-wave description")
    return d


def save_solution(desc: Desc, u: np.ndarray, prefix: str) -> None:
    """Problem::Save (src/problem.cpp:762-790) of a host body vector: prefix.mesh,
    prefix_{rho,rhou,rhov,energy}.gf and prefix_coefficients.csv."""
    lib = load()
    u = np.ascontiguousarray(u, dtype=np.float64)
    q = desc.k + 1
    if u.size != 4 * q * q * desc.nx * desc.ny:
        raise EngineError(1, "body vector size does not match the description")
    rc = lib.eg_save_solution(C.byref(desc), _ptr(u), str(prefix).encode())
    if rc != OK:
        raise EngineError(rc, lib.eg_last_error(None).decode())


def default_opts(**kw) -> Opts:
    lib = load()
    o = Opts()
    lib.eg_opts_default(C.byref(o))
    for key, val in kw.items():
        setattr(o, key, val)
    return o


class Context:
    """One problem instance resident on the GPU (an eg_ctx)."""

    def __init__(self, desc: Desc, opts: Opts):
        self.lib = load()
        self.desc = desc
        self.opts = opts
        h = C.c_void_p()
        rc = self.lib.eg_create(C.byref(desc), C.byref(opts), C.byref(h))
        if rc != OK:
            raise EngineError(rc, self.lib.eg_status_string(rc).decode())
        self.h = h
        s = (C.c_int * 7)()
        self.lib.eg_sizes(self.h, s)
        self.n, self.p, self.m, self.t, self.nf, self.nu, self.nl = list(s)
        self.q = desc.k + 1

    def close(self):
        if getattr(self, "h", None):
            self.lib.eg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != OK:
            msg = (self.lib.eg_last_error(self.h) or b"").decode() or self.lib.eg_status_string(rc).decode()
            raise EngineError(rc, msg)

    def slot_size(self, slot: str) -> int:
        return {"U": self.nu, "OLD": self.nu, "R": self.nu, "DU": self.nu, "RHS": self.nl,
                "LAMBDA": self.nl, "D": self.nl, "X": self.n * self.m * 4 * self.t, "Y": self.nu,
                "HLL_A": self.nf * self.q, "HLL_B": self.nf * self.q,
                "PC_BLOCKS": self.pc_size()}[slot]

    def upload(self, slot: str, x: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.size == self.slot_size(slot)
        self._check(self.lib.eg_upload(self.h, SLOT[slot], _ptr(x)))

    def download(self, slot: str) -> np.ndarray:
        out = np.empty(self.slot_size(slot))
        self._check(self.lib.eg_download(self.h, SLOT[slot], _ptr(out)))
        return out

    def initial(self):
        self._check(self.lib.eg_initial(self.h))

    def freeze(self, stage_dt: float, check_admissible: bool = True) -> float:
        rate = C.c_double()
        self._check(self.lib.eg_freeze(self.h, stage_dt, int(check_admissible), C.byref(rate)))
        return rate.value

    def set_dt(self, dt: float):
        self._check(self.lib.eg_set_dt(self.h, dt))

    def residual(self):
        self._check(self.lib.eg_residual(self.h))

    def cell_norm(self, slot: str) -> float:
        v = C.c_double()
        self._check(self.lib.eg_cell_norm(self.h, SLOT[slot], C.byref(v)))
        return v.value

    def admissible(self, slot: str) -> bool:
        v = C.c_int()
        self._check(self.lib.eg_admissible(self.h, SLOT[slot], C.byref(v)))
        return bool(v.value)

    def dg_apply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.nu)
        self._check(self.lib.eg_dg_apply(self.h, _ptr(x), _ptr(y)))
        return y

    def condense(self):
        self._check(self.lib.eg_condense(self.h))

    def schur_apply(self, v: np.ndarray) -> np.ndarray:
        v = np.ascontiguousarray(v, dtype=np.float64)
        y = np.empty(self.nl)
        self._check(self.lib.eg_schur_apply(self.h, _ptr(v), _ptr(y)))
        return y

    def recover(self, lam: np.ndarray) -> np.ndarray:
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        du = np.empty(self.nu)
        self._check(self.lib.eg_recover(self.h, _ptr(lam), _ptr(du)))
        return du

    def pc_size(self) -> int:
        count = C.c_longlong()
        self._check(self.lib.eg_pc_size(self.h, C.byref(count)))
        return count.value

    def set_ilu_wait(self, limit_ns: int = 0, starve: bool = False):
        """Test setting of the block ILU(0) device waits (eg_set_ilu_wait)."""
        self._check(self.lib.eg_set_ilu_wait(self.h, int(limit_ns), int(starve)))

    def pc_factor(self, factor: bool = True):
        self._check(self.lib.eg_pc_factor(self.h, int(factor)))

    def pc_apply(self, b: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty_like(b)
        self._check(self.lib.eg_pc_apply(self.h, _ptr(b), _ptr(x)))
        return x

    def linear_solve(self, rhs: np.ndarray, x0: np.ndarray | None = None, refresh: bool = True,
                     linear_tol: float | None = None):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros_like(rhs) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        eq = np.empty_like(rhs)
        st = LinearStats()
        tol = self.opts.linear_tol if linear_tol is None else linear_tol
        self._check(self.lib.eg_linear_solve(self.h, _ptr(rhs), _ptr(x), _ptr(eq), int(refresh), tol,
                                             C.byref(st)))
        return x, eq, st

    def stage_begin(self, stage_dt: float):
        self._check(self.lib.eg_stage_begin(self.h, stage_dt))

    def newton_residual(self) -> float:
        v = C.c_double()
        self._check(self.lib.eg_newton_residual(self.h, C.byref(v)))
        return v.value

    def newton_update(self, residual_norm: float, old_norm: float) -> UpdateStats:
        st = UpdateStats()
        self._check(self.lib.eg_newton_update(self.h, residual_norm, old_norm, C.byref(st)))
        return st

    def upload_ptr(self, slot: str, ptr: int):
        """Upload from a raw host or device address (no intermediate copy)."""
        self._check(self.lib.eg_upload(self.h, SLOT[slot], C.cast(C.c_void_p(ptr), _DP)))

    def download_ptr(self, slot: str, ptr: int):
        self._check(self.lib.eg_download(self.h, SLOT[slot], C.cast(C.c_void_p(ptr), _DP)))

    def stream_ptr(self) -> int:
        return int(self.lib.eg_stream(self.h) or 0)

    def device_bytes(self) -> int:
        return int(self.lib.eg_device_bytes(self.h))


def run_options(*, integrator: str = "ssp-dirk3", steps: int = -1, newton_steps: int = -1,
                max_newton: int = 30, dt: float = 1e-3, cfl: float = -1.0, end: float = 0.2,
                tol: float = 1e-12, timing_only: bool = True, save_solution: bool = False,
                prefix: str = "run", form_name: str = "hdg", precond_name: str = "block-jacobi",
                check_update: bool = False) -> tuple[RunOpts, list]:
    keep = [s.encode() for s in (prefix, form_name, "partial", "gmres", precond_name, "none")]
    ro = RunOpts(1 if integrator == "be" else 0, steps, newton_steps, max_newton, dt, cfl, end, tol,
                 int(timing_only), int(save_solution), keep[0], keep[1], keep[2], keep[3], keep[4],
                 keep[5], int(check_update))
    return ro, keep


class Stepper:
    """Advances the SSP-DIRK3/BE schedule one accepted Newton update per call."""

    def __init__(self, ctx: Context, ro: RunOpts, keep=None):
        self.ctx = ctx
        self._keep = (ro, keep)
        h = C.c_void_p()
        ctx._check(ctx.lib.eg_stepper_create(ctx.h, C.byref(ro), C.byref(h)))
        self.h = h

    def next(self) -> UpdateStats | None:
        st = UpdateStats()
        rc = self.ctx.lib.eg_stepper_next(self.h, C.byref(st))
        if rc == -1:
            return None
        self.ctx._check(rc)
        return st

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.eg_stepper_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def declared_symbols(header: Path = HEADER_PATH) -> list[str]:
    """Function names declared in the public header."""
    import re
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(eg_[a-z0-9_]+)\s*\(", text)))


class Batch:
    """Independent instances run to completion together (eg_batch_*): one
    context and CUDA stream per instance, `threads` host workers."""

    def __init__(self, descs: list, opts: list, device: int = 0):
        self.lib = load()
        n = len(descs)
        da, oa = (Desc * n)(*descs), (Opts * n)(*opts)
        h = C.c_void_p()
        rc = self.lib.eg_batch_create(n, da, oa, device, C.byref(h))
        if rc != OK:
            raise EngineError(rc, (self.lib.eg_last_error(None) or b"").decode())
        self.h, self.n = h, n

    def run(self, ro: RunOpts, threads: int = 16, check: bool = True) -> BatchStats:
        """Runs every instance; with check=False failures are only counted
        (per-instance statuses via result())."""
        st = BatchStats()
        rc = self.lib.eg_batch_run(self.h, C.byref(ro), threads, C.byref(st))
        if rc != OK and check:
            raise EngineError(rc, self.lib.eg_status_string(rc).decode())
        return st

    def result(self, i: int) -> tuple[int, RunResult]:
        status, res = C.c_int(), RunResult()
        self.lib.eg_batch_result(self.h, i, C.byref(status), C.byref(res))
        return status.value, res

    def state(self, i: int, nu: int) -> np.ndarray:
        out = np.empty(nu)
        ctx = self.lib.eg_batch_context(self.h, i)
        rc = self.lib.eg_download(ctx, SLOT["U"], _ptr(out))
        if rc != OK:
            raise EngineError(rc, self.lib.eg_status_string(rc).decode())
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.eg_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """Request loop with admission against a device-memory budget (eg_server_*)."""

    def __init__(self, workers: int = 8, budget_bytes: int = 120 << 30, device: int = 0,
                 keep_contexts: bool = True, keep_states: bool = False):
        self.lib = load()
        o = ServerOpts(device, workers, budget_bytes, int(keep_contexts), int(keep_states))
        h = C.c_void_p()
        rc = self.lib.eg_server_create(C.byref(o), C.byref(h))
        if rc != OK:
            raise EngineError(rc, self.lib.eg_status_string(rc).decode())
        self.h = h

    def submit(self, nx, ny, k, alpha_deg, steps, newton_steps=3, cfl=1.0, form=FORM_HDG, precond=PC_JACOBI,
               precision=PRECISION_FP64) -> int:
        r = Request(nx, ny, k, alpha_deg, steps, newton_steps, cfl, form, precond, precision)
        rid = C.c_longlong()
        rc = self.lib.eg_server_submit(self.h, C.byref(r), C.byref(rid))
        if rc != OK:
            raise EngineError(rc, self.lib.eg_status_string(rc).decode())
        return rid.value

    def poll(self, rid: int) -> RequestResult | None:
        res = RequestResult()
        rc = self.lib.eg_server_poll(self.h, rid, C.byref(res))
        return res if rc == OK else None

    def state(self, rid: int, nu: int) -> np.ndarray:
        out = np.empty(nu)
        rc = self.lib.eg_server_state(self.h, rid, _ptr(out))
        if rc != OK:
            raise EngineError(rc, "no stored state for this request")
        return out

    def drain(self) -> ServerStats:
        st = ServerStats()
        self.lib.eg_server_drain(self.h, C.byref(st))
        return st

    def clock(self) -> float:
        return float(self.lib.eg_server_clock(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.eg_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
