#!/usr/bin/env python3
"""Benchmark: mean seconds per accepted Newton update on one B200.

Workload (default): 128x128 periodic Q4 simple wave, gamma=3, alpha=30 deg,
condensed HDG with partial assembly and block-Jacobi right-preconditioned
GMRES, SSP-DIRK3 at CFL 1, 3 Newton updates per stage. A "step" is one
accepted Newton update of that schedule (residual -> condensation -> Schur
GMRES -> recovery -> validation -> line search), advanced through the C-ABI
stepper. Inputs are synthetic: the seeded, deterministic simple-wave initial
condition (no dataset exists for this problem).

Arms
  (default)        the CUDA engine (mfem_euler2d_cpp_b200/lib/libeuler2d_cuda.so)
  --impl reference the reference's own CPU code (oracle/_ref, the unmodified
                   reference sources built against the MFEM-subset shim), one
                   thread on the host, bounded sample of the same workload.

Multi-GPU: the update does not shard across GPUs in this build; N ranks run N
independent replicas (weak scaling, no data-path collective). value is the
whole-job time per update: max over ranks of the timed region / (N * K).
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "c2": dict(nx=128, ny=128, k=4, alpha=30.0, form="hdg", precond="block-jacobi", cfl=1.0, steps=5,
               newton_steps=3,
               label="128x128 periodic Q4 simple wave (gamma=3, alpha=30deg), HDG condensed, partial "
                     "assembly, block-Jacobi GMRES, SSP-DIRK3 CFL 1, 5 steps x 3 Newton updates"),
    "c1": dict(nx=16, ny=16, k=3, alpha=45.0, form="hdg", precond="block-jacobi", cfl=1.0, steps=3,
               newton_steps=3,
               label="16x16 periodic Q3 simple wave (gamma=3, alpha=45deg), HDG condensed, partial "
                     "assembly, block-Jacobi GMRES, SSP-DIRK3 CFL 1, 3 steps x 3 Newton updates"),
    "c3": dict(nx=256, ny=256, k=3, alpha=45.0, form="hdg", precond="block-jacobi", cfl=1.0, steps=5,
               newton_steps=3,
               label="256x256 periodic Q3 simple wave (gamma=3, alpha=45deg), HDG condensed, FP64"),
}
# The 256x256 Q3 accuracy run: to T = 0.2, FP64 and mixed precision, accuracy
# and conservation of the mixed path against the FP64 path (the FP64 oracle).
C3_ACCURACY = dict(nx=256, ny=256, k=3, alpha=45.0, form="hdg", precond="block-jacobi", cfl=1.0, end=0.2,
                   label="256x256 periodic Q3 simple wave (gamma=3, alpha=45deg), HDG condensed, SSP-DIRK3 "
                         "CFL 1 to T=0.2, Newton to tol 1e-12, FP64 and mixed precision")
METRIC = "mean s per accepted Newton update"
K_NAMES = ["residual", "dg_apply", "dg_jacobi", "condense", "schur_apply", "recover",
           "recovered_residual", "schur_jacobi", "pc_apply", "krylov", "freeze", "admissible", "vector"]


# DRAM bytes (read + write) per cell of one launch, from one ncu capture of the
# kernel on a 64x64 mesh of the same degree (profiles/condense_gj2_q4_64x64.txt,
# profiles/panel_gemv_q4_64x64.txt); per-launch traffic grows with the cell count.
NCU_TRAFFIC_PER_CELL = {("condense", 4): 512.70e6 / 4096, ("schur_apply", 4): 216.24e6 / 4096}


def traffic(name, w):
    per = NCU_TRAFFIC_PER_CELL.get((name, w["k"]))
    return None if per is None else per * w["nx"] * w["ny"]


def sizes(w):
    q = w["k"] + 1
    p, n = q * q, w["nx"] * w["ny"]
    m, t = 4 * p, 4 * q
    return dict(q=q, p=p, n=n, m=m, t=t, nf=2 * n, nu=n * m, nl=2 * n * t)


def algorithmic(w):
    """Per-launch algorithmic bytes / flops of the hot kernels (FP64)."""
    s = sizes(w)
    n, m, t, q, p, nu, nl, nf = s["n"], s["m"], s["t"], s["q"], s["p"], s["nu"], s["nl"], s["nf"]
    return {
        # k >= 4 streams the 16 panels C_s X_o of a cell, lower degrees X and C
        "schur_apply": ("hbm", 8.0 * ((n * 16 * t * t if q >= 5 else n * m * 4 * t + 64 * n * q) + 3 * nl)),
        "recover": ("hbm", 8.0 * (n * m * 4 * t + n * m + nl + nu)),
        "dg_apply": ("hbm", 8.0 * (2 * nu + 32 * n * p + 32 * nf * q)),
        "residual": ("hbm", 8.0 * (3 * nu + 6 * nf * q)),
        "pc_apply": ("hbm", 8.0 * (nf * t * t + 2 * nl) if w["form"] == "hdg" else 8.0 * (n * m * m + 2 * nu)),
        "condense": ("fp64", n * (2.0 / 3.0 * m ** 3 + 2.0 * m * m * (4 * t + 1))),
        "dg_jacobi": ("fp64", n * (2.0 / 3.0 * m ** 3)),
    }


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, out: Path, gpu_index: int):
        self.out, self.gpu_index, self.proc = out, gpu_index, None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.fh = open(self.out, "w")
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                      "-i", str(self.gpu_index), "-lms", "200"], stdout=self.fh,
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in self.out.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1].split()[0]), smax=float(parts[2].split()[0]),
                                 power=float(parts[3].split()[0]) if parts[3][0].isdigit() else 0.0,
                                 hw=parts[5], hwt=parts[6], swt=parts[7], pcap=parts[8]))
            except (ValueError, IndexError):
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        reasons = []
        for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                          ("swt", "sw_thermal_slowdown"), ("pcap", "sw_power_cap")):
            if any(r[key].lower().startswith("active") for r in rows):
                reasons.append(name)
        return {"sm_mhz": float(np.median([r["sm"] for r in rows])),
                "sm_max_mhz": max(r["smax"] for r in rows), "reasons": reasons, "samples": len(rows),
                "power_w_max": max(r["power"] for r in rows)}


# ------------------------------------------------------------ CPU reference
def ref_binary():
    ref = ROOT / "oracle" / "_ref"
    for name in ("euler2d_ref_v4", "euler2d_ref_v3"):
        exe = ref / name
        if exe.exists():
            try:
                subprocess.run([str(exe), "--help"], capture_output=True, check=True, timeout=30)
                return exe
            except (OSError, subprocess.CalledProcessError, subprocess.TimeoutExpired):
                continue
    return None


def run_reference_updates(w, newton_steps: int, timeout: float = 900.0, integrator: str = "ssp-dirk3"):
    """Run the reference CLI on the first SSP-DIRK3 step of the workload with
    `newton_steps` updates per stage, single-threaded on one core. Returns the
    per-update iteration_s list (the reference's own update timer)."""
    exe = ref_binary()
    if exe is None:
        return None, "oracle/_ref binaries not built"
    env = dict(os.environ)
    for name in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        env[name] = "1"
    with tempfile.TemporaryDirectory() as tmp:
        prefix = Path(tmp) / "ref"
        cmd = [str(exe), "--nx", str(w["nx"]), "--ny", str(w["ny"]), "--k", str(w["k"]),
               "--alpha-deg", str(w["alpha"]), "--cfl", str(w["cfl"]), "--steps", "1",
               "--newton-steps", str(newton_steps), "--form", w["form"], "--precond", w["precond"],
               "--assembly", "partial", "--integrator", integrator, "--no-save-solution", "--output",
               str(prefix)]
        if shutil.which("taskset"):
            cmd = ["taskset", "-c", "0"] + cmd
        proc = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
        if proc.returncode:
            return None, proc.stderr.strip()[-300:]
        with open(f"{prefix}_{w['form']}_iterations.csv", newline="") as fh:
            times = [float(r["iteration_s"]) for r in csv.DictReader(fh)]
    return times, exe.name


def run_to_time(w, precision, local):
    """The whole time loop of the workload (eg_run): Newton to the reference's
    tolerance in every stage, to T = w['end']. Returns the run result."""
    from mfem_euler2d_cpp_b200 import capi

    ctx = make_context(w, w["form"], local, precision=precision)
    ro, keep = capi.run_options(integrator="ssp-dirk3", steps=-1, newton_steps=-1, cfl=w["cfl"], end=w["end"],
                                form_name=w["form"], precond_name=w["precond"])
    res = capi.RunResult()
    # the time loop prints the reference's one-line summary on stdout; keep
    # this process's stdout to the single JSON line
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        t0 = time.perf_counter()
        rc = ctx.lib.eg_run(ctx.h, capi.C.byref(ro), capi.C.byref(res))
        wall = time.perf_counter() - t0
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    ctx._check(rc)
    ctx.close()
    del keep
    return res, wall


def c3_accuracy(local, cpu: bool):
    """256x256 Q3 simple wave: FP64 and mixed-precision runs to T = 0.2; final L2
    errors and conservation drift of both, and the mixed path's error against
    the FP64 path's (the FP64 oracle). cpu: also the reference's CPU cost of
    one Newton update on the same mesh (backward Euler, one update)."""
    w = C3_ACCURACY
    out = {"workload": w["label"]}
    runs = {}
    for prec in ("fp64", "mixed"):
        res, wall = run_to_time(w, prec, local)
        runs[prec] = res
        out[prec] = {"updates": res.updates, "time_steps": res.time_steps, "final_time": res.final_time,
                     "l2_errors": list(res.errors), "conservation_drift": res.drift,
                     "mean_newton_device_s": res.newton_device_ms * 1e-3 / max(res.updates, 1),
                     "time_loop_s": wall}
    e64 = np.sqrt(np.sum(np.square(runs["fp64"].errors)))
    emx = np.sqrt(np.sum(np.square(runs["mixed"].errors)))
    out["joint_l2_error"] = {"fp64": e64, "mixed": emx, "mixed_vs_fp64_relative": abs(emx - e64) / e64}
    out["within_1pct_of_fp64"] = bool(abs(emx - e64) <= 0.01 * e64)
    out["mixed_speedup_per_update"] = (out["fp64"]["mean_newton_device_s"] /
                                       max(out["mixed"]["mean_newton_device_s"], 1e-30))
    if cpu:
        times, src = run_reference_updates(dict(w, newton_steps=1), 1, integrator="be")
        out["cpu_reference_per_update_s"] = float(np.mean(times)) if times else None
        out["cpu_reference_sample"] = ("one backward-Euler Newton update on the same mesh, degree and CFL "
                                       f"(the same update algorithm), {src}, one core") if times else src
    return out


def reference_status(nx, k, alpha, steps=3, newton_steps=3, timeout=600.0):
    """Outcome of the reference command line on one batch instance: (exit
    code, its last stderr line or "ok")."""
    exe = ref_binary()
    if exe is None:
        return None, "oracle/_ref binaries not built"
    with tempfile.TemporaryDirectory() as tmp:
        cmd = [str(exe), "--nx", str(nx), "--ny", str(nx), "--k", str(k), "--alpha-deg", repr(alpha), "--cfl", "1",
               "--steps", str(steps), "--newton-steps", str(newton_steps), "--form", "hdg", "--timing-only",
               "--no-save-solution", "--output", str(Path(tmp) / "ref")]
        proc = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    msg = proc.stderr.strip().splitlines()[-1] if proc.returncode and proc.stderr.strip() else "ok"
    return proc.returncode, msg


def batch_c4(threads: int, cpu: bool):
    """The uneven-instance batch (64 seeded instances, nx = ny from 8 to 64, k 1..6, 3 steps x 3 updates):
    the batched mixed-precision path against the plain FP64 path one instance
    at a time; instances that fail here are run through the reference's own
    command line and its outcome is recorded beside them."""
    from mfem_euler2d_cpp_b200 import workloads

    out = workloads.run_batch(count=64, seed=0, threads=threads, precision="mixed")
    cfg = out.pop("config", {})
    out["instances"] = cfg.get("instances")
    if cpu:
        ref = []
        for i, tpl, status in out["failed_instances"]:
            rc, msg = reference_status(tpl[0], tpl[2], tpl[3])
            ref.append({"instance": i, "nx": tpl[0], "k": tpl[2], "status_here": status,
                        "reference_exit": rc, "reference_message": msg})
        out["failed_instances_in_the_reference"] = ref
    return out


def serve_c5():
    """The served request stream, bounded: 48 requests of its distribution (Poisson
    arrivals at 200 requests/s, 1..10 SSP-DIRK3 steps, k 2..6, meshes 20^2 to
    64^2; the full distribution's 128^2 Q7-Q8 requests take minutes each),
    served by 16 workers in mixed precision against the plain FP64 path one
    request at a time, with every request's L2 error checked against that
    run's."""
    from mfem_euler2d_cpp_b200 import workloads

    out = workloads.run_serve(requests=48, rate=200.0, seed=1, workers=16, budget_gb=120.0, precision="mixed",
                              max_nx=64, max_k=6)
    out["config"]["sample"] = "first 48 requests of the seeded stream, nx <= 64, k <= 6"
    return out


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------- helpers
def dist_setup(gpus: int, backend: str = "nccl"):
    """One process per GPU (torchrun's RANK/LOCAL_RANK/WORLD_SIZE/MASTER_*):
    the replicas share nothing on the data path; the process group carries
    only the barriers and the max-over-ranks of the timings. `gloo` runs the
    same plumbing on CPU processes (tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_seconds_per_update(elapsed_ms_max: float, steps: int, world: int) -> float:
    """Whole-job value: every replica ran `steps` accepted updates within the
    slowest rank's elapsed time."""
    return elapsed_ms_max * 1e-3 / (steps * world)


def make_context(w, form, device=0, precision="fp64"):
    from mfem_euler2d_cpp_b200 import capi

    lib = capi.load()
    if lib.eg_set_device(device) != capi.OK:
        raise RuntimeError("eg_set_device failed")
    d = capi.simple_wave_desc(w["nx"], w["ny"], w["k"], w["alpha"])
    o = capi.default_opts(form=capi.FORM_HDG if form == "hdg" else capi.FORM_DG,
                          precond=capi.PC_JACOBI if w["precond"] == "block-jacobi" else capi.PC_ILU0,
                          precision=capi.PRECISION_MIXED if precision == "mixed" else capi.PRECISION_FP64)
    return capi.Context(d, o)


def make_stepper(ctx, w, total_updates, form):
    from mfem_euler2d_cpp_b200 import capi

    per_step = 4 * w["newton_steps"]
    steps = max(w["steps"], math.ceil(total_updates / per_step) + 1)
    ro, keep = capi.run_options(integrator="ssp-dirk3", steps=steps, newton_steps=w["newton_steps"],
                                cfl=w["cfl"], form_name=form, precond_name=w["precond"])
    return capi.Stepper(ctx, ro, keep)


def timed_updates(ctx, stepper, K, world, events_stream, host_io=None):
    """Time exactly K accepted updates with CUDA events on the engine stream.
    host_io (a pinned numpy array holding the live state) adds, to every step,
    the H2D upload of the state from it before the update and the D2H read of
    the updated state back into it: each update starts from the state the
    previous one returned."""
    import torch

    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    device_ms = 0.0
    krylov = 0
    barrier(world)
    torch.cuda.synchronize()
    start.record(events_stream)
    for _ in range(K):
        if host_io is not None:
            ctx.upload_ptr("U", host_io.ctypes.data)
        st = stepper.next()
        if st is None:
            raise RuntimeError("schedule exhausted")
        device_ms += st.device_ms
        krylov += st.krylov_iterations
        if host_io is not None:
            ctx.download_ptr("U", host_io.ctypes.data)
    end.record(events_stream)
    end.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    timed_updates.krylov = krylov
    return start.elapsed_time(end), device_ms


def fp64_gemm_peak():
    """Measured FP64 GEMM rate (torch/cuBLAS DGEMM, 4096^3, best of 5)."""
    import torch

    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ------------------------------------------------------------------- arms
def run_ours(args, world, rank, local):
    import torch

    from mfem_euler2d_cpp_b200 import capi

    w = dict(WORKLOADS[args.workload])
    K, W = args.steps, args.warmup
    torch.cuda.set_device(local)
    ctx = make_context(w, w["form"], local)
    KP = min(K, 10)  # updates of the profiled block (per-class CUDA events)
    stepper = make_stepper(ctx, w, W + 2 * K + KP, w["form"])
    ext = torch.cuda.ExternalStream(ctx.stream_ptr())
    for _ in range(W):
        if stepper.next() is None:
            raise RuntimeError("schedule exhausted during warm-up")
    launches0 = ctx.lib.eg_launch_count(ctx.h)
    phys = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            phys = int(vis.split(",")[local])
        except ValueError:
            phys = local
    sampler = ClockSampler(Path(tempfile.gettempdir()) / f"eg_clocks_{rank}.csv", phys)
    sampler.start()
    time.sleep(0.3)
    elapsed_ms, dev_ms = timed_updates(ctx, stepper, K, world, ext)
    krylov_main = timed_updates.krylov
    clocks = sampler.stop()
    launches = ctx.lib.eg_launch_count(ctx.h) - launches0
    # end to end: the state crosses the host boundary every update
    nu = ctx.nu
    pin = torch.empty(nu, dtype=torch.float64, pin_memory=True).numpy()
    pin[:] = ctx.download("U")
    e2e_ms, _ = timed_updates(ctx, stepper, K, world, ext, host_io=pin)
    # per-class kernel times from a separate block of KP updates: the event
    # pairs of the class profiler stay out of the timed regions above
    ctx.lib.eg_profile_reset(ctx.h)
    ctx.lib.eg_profile_enable(ctx.h, 1)
    timed_updates(ctx, stepper, KP, world, ext)
    prof = {}
    for i, name in enumerate(K_NAMES):
        import ctypes as C

        ms, cnt = C.c_double(), C.c_longlong()
        ctx.lib.eg_profile_query(ctx.h, i, C.byref(ms), C.byref(cnt))
        prof[name] = (ms.value, cnt.value)
    ctx.lib.eg_profile_enable(ctx.h, 0)
    elapsed_ms = max_over_ranks(world, elapsed_ms)
    e2e_ms = max_over_ranks(world, e2e_ms)
    dev_ms = max_over_ranks(world, dev_ms)
    dev_bytes = ctx.device_bytes()
    ctx_sizes = sizes(w)
    stepper.close()
    ctx.close()
    torch.cuda.synchronize()

    def secondary(wx, form, precision, label):
        """W warm-up updates, K updates timed without the class profiler, then
        KP profiled updates for the per-class kernel times."""
        cx = make_context(wx, form, local, precision=precision)
        st = make_stepper(cx, wx, W + K + KP, form)
        ex = torch.cuda.ExternalStream(cx.stream_ptr())
        for _ in range(W):
            st.next()
        ms_, dev_ = timed_updates(cx, st, K, world, ex)
        kry_ = timed_updates.krylov
        cx.lib.eg_profile_reset(cx.h)
        cx.lib.eg_profile_enable(cx.h, 1)
        timed_updates(cx, st, KP, world, ex)
        prof_ = {}
        for i, name in enumerate(K_NAMES):
            import ctypes as C

            kms, cnt = C.c_double(), C.c_longlong()
            cx.lib.eg_profile_query(cx.h, i, C.byref(kms), C.byref(cnt))
            if cnt.value:
                prof_[name] = round(kms.value / KP, 3)
        cx.lib.eg_profile_enable(cx.h, 0)
        ms_ = max_over_ranks(world, ms_)
        st.close()
        cx.close()
        out = {"value": job_seconds_per_update(ms_, K, world), "unit": "s", "ms_per_step": ms_ / K,
               "mean_newton_device_s": dev_ * 1e-3 / K, "krylov_per_update": kry_ / K,
               "kernel_ms_per_update": prof_, "profiled_updates": KP}
        out.update(label)
        return out

    # DG form of the same workload (secondary line)
    dg = None if args.no_dg else secondary(w, "dg", "fp64", {"form": "dg"})
    # the same HDG workload in mixed precision (secondary line)
    mixed = None if args.no_mixed else secondary(w, "hdg", "mixed", {"precision": "mixed"})
    # the same HDG workload preconditioned by block ILU(0) (secondary line)
    ilu = None if args.no_ilu else secondary(dict(w, precond="block-ilu0"), "hdg", "fp64",
                                             {"precond": "block-ilu0"})

    if rank != 0:
        return None
    peaks, peak_src = measured_peaks()
    alg = algorithmic(w)
    dominant = max(prof, key=lambda k: prof[k][0])
    roofline = None
    fp64_peak = None
    dom_ms, dom_launch = prof[dominant]
    ops_per = {"schur_apply": 2, "condense": 2}.get(dominant, 1)
    nops = max(1, dom_launch // ops_per)
    if dominant in alg:
        kind, units = alg[dominant]
        avg_s = dom_ms * 1e-3 / nops
        if kind == "hbm":
            achieved = units / avg_s / 1e9
            peak = peaks["hbm_gbs"]
            roofline = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": peak,
                        "unit": "GB/s", "frac": achieved / peak, "traffic": traffic(dominant, w),
                        "algorithmic_bytes_per_launch": units, "avg_launch_ms": avg_s * 1e3,
                        "launches": nops, "peak_source": f"{peak_src} hbm_gbs"}
        else:
            fp64_peak = fp64_gemm_peak()
            achieved = units / avg_s / 1e12
            roofline = {"kernel": dominant, "bound": "tensor", "pipe": "fp64 mma (m8n8k4)",
                        "achieved": achieved, "peak": fp64_peak,
                        "unit": "TFLOP/s", "frac": achieved / fp64_peak, "traffic": traffic(dominant, w),
                        "algorithmic_flops_per_launch": units, "avg_launch_ms": avg_s * 1e3,
                        "launches": nops,
                        "peak_source": "measured FP64 DGEMM (torch.matmul float64 4096^3) on this GPU"}
    # second roofline line for the HBM-bound Schur apply (the matrix-free hot loop)
    hbm_lines = {}
    for name in ("schur_apply", "recover", "pc_apply", "residual", "dg_apply"):
        ms, cnt = prof[name]
        # kernels per operation: the Schur action (panel GEMV + face combine) and
        # the residual (face values, then the cell kernel) launch two
        per = 2 if name in ("schur_apply", "residual") else 1
        n_op = cnt // per
        if n_op and name in alg:
            avg_s = ms * 1e-3 / n_op
            ach = alg[name][1] / avg_s / 1e9
            hbm_lines[name] = {"achieved_gbs": ach, "frac": ach / peaks["hbm_gbs"], "avg_launch_ms": avg_s * 1e3,
                               "launches": n_op, "traffic": traffic(name, w)}
    # the dense-contraction classes against the FP64 DGEMM of this GPU
    tensor_lines = {}
    for name in ("condense", "dg_jacobi"):
        if name == "condense":
            ms, cnt = prof["condense"]
            launches_ = cnt // 2
        else:
            ms = (dg or {}).get("kernel_ms_per_update", {}).get("dg_jacobi")
            launches_ = None
        if name == "condense" and launches_:
            if fp64_peak is None:
                fp64_peak = fp64_gemm_peak()
            avg_s = ms * 1e-3 / launches_
            ach = alg["condense"][1] / avg_s / 1e12
            tensor_lines["condense"] = {"achieved_tflops": ach, "frac": ach / fp64_peak, "avg_launch_ms": avg_s * 1e3,
                                        "algorithmic_flops": alg["condense"][1],
                                        "peak_tflops": fp64_peak, "peak_source": "measured FP64 DGEMM, this GPU"}
        elif name == "dg_jacobi" and ms:
            if fp64_peak is None:
                fp64_peak = fp64_gemm_peak()
            # one factor per DG update (the reference's n 2/3 m^3 LU count)
            ach = alg["dg_jacobi"][1] / (ms * 1e-3) / 1e12
            tensor_lines["dg_jacobi"] = {"achieved_tflops": ach, "frac": ach / fp64_peak, "ms_per_update": ms,
                                         "algorithmic_flops": alg["dg_jacobi"][1], "peak_tflops": fp64_peak}
    c3 = None if args.no_c3 else c3_accuracy(local, cpu=(world == 1 and not args.no_cpu_baseline))
    batch = None if args.no_batch else batch_c4(threads=32, cpu=(world == 1 and not args.no_cpu_baseline))
    serve = None if (args.no_serve or world > 1) else serve_c5()  # one GPU: the request loop's device 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        times, src = run_reference_updates(w, 1)
        if times:
            cpu = {"value": float(np.mean(times)), "unit": "s", "cores": 1, "kind": "reference",
                   "sample": f"first SSP-DIRK3 step of the same workload, 1 Newton update per stage "
                             f"({len(times)} updates), reference's own per-update timer; {src} on "
                             f"'{cpu_model()}', one thread pinned with taskset",
                   "per_update_s": times}
        else:
            cpu = {"value": None, "unit": "s", "cores": 1, "kind": "reference", "sample": f"unavailable: {src}"}
        if ilu is not None:
            times_i, _ = run_reference_updates(dict(w, precond="block-ilu0"), 1)
            if times_i:
                ilu["cpu_reference_s"] = float(np.mean(times_i))
                ilu["cpu_reference_per_update_s"] = times_i
    value = job_seconds_per_update(elapsed_ms, K, world)
    line = {
        "metric": f"{METRIC} (HDG, {w['nx']}x{w['ny']} Q{w['k']}, block-Jacobi)",
        "value": value, "unit": "s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": elapsed_ms / K, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: deterministic simple-wave initial condition (gamma=3) projected on the mesh",
        "config": {"workload": w["label"], "nx": w["nx"], "ny": w["ny"], "k": w["k"], "alpha_deg": w["alpha"],
                   "form": w["form"], "precond": w["precond"], "integrator": "ssp-dirk3", "cfl": w["cfl"],
                   "newton_steps_per_stage": w["newton_steps"], "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (condensed responses X are %.2f GB per update)"
                         % (8 * ctx_sizes["n"] * ctx_sizes["m"] * 4 * ctx_sizes["t"] / 1e9),
                   "body_dofs": ctx_sizes["nu"], "trace_dofs": ctx_sizes["nl"],
                   "device_bytes": dev_bytes},
        "updates_per_s": K * world / (elapsed_ms * 1e-3),
        "mean_newton_device_s": dev_ms * 1e-3 / K,
        "e2e": {"value": e2e_ms * 1e-3 / (K * world), "unit": "s", "h2d_bytes_per_step": 8 * ctx_sizes["nu"],
                "d2h_bytes_per_step": 8 * ctx_sizes["nu"],
                "path": "per update: eg_upload(U) from pinned host memory holding the state the previous update "
                        "returned, eg_stepper_next, eg_download(U) back into it"},
        "roofline": roofline,
        "hbm_kernels": hbm_lines,
        "tensor_kernels": tensor_lines,
        "profiled_updates": KP,
        "kernel_ms": {k: round(v[0], 3) for k, v in prof.items() if v[1]},
        "kernel_ms_per_update": {k: round(v[0] / KP, 3) for k, v in prof.items() if v[1]},
        "kernel_launches": {k: v[1] for k, v in prof.items() if v[1]},
        "krylov_per_update": krylov_main / K,
        "gpu_launches": int(launches),
        "cpu_baseline": cpu,
        "clocks": clocks,
        "dg": dg,
        "ilu": ilu,
        "mixed": mixed,
        "c3_accuracy": c3,
        "batch_c4": batch,
        "serve_c5": serve,
    }
    return line


def run_reference_arm(args, world, rank):
    if rank != 0:
        return None
    w = dict(WORKLOADS[args.workload])
    K, W = args.steps, args.warmup
    # bounded sample: at most 12 reference updates (about 3 minutes at 128^2 Q4)
    total = min(W + K, args.ref_max_updates)
    n_per_stage = max(1, math.ceil(total / 4))
    times, src = run_reference_updates(w, n_per_stage, timeout=1800)
    if not times:
        return {"impl": "reference", "unavailable": f"reference CPU build could not run: {src}"}
    warm = min(W, len(times) - 1)
    timed = times[warm:warm + K]
    value = float(np.mean(timed))
    return {
        "impl": "reference",
        "metric": f"{METRIC} (HDG, {w['nx']}x{w['ny']} Q{w['k']}, block-Jacobi)",
        "value": value, "unit": "s", "n_gpus": world, "steps": len(timed), "warmup": warm,
        "requested_steps": K, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: deterministic simple-wave initial condition (gamma=3) projected on the mesh",
        "config": {"workload": w["label"], "nx": w["nx"], "ny": w["ny"], "k": w["k"],
                   "form": w["form"], "precond": w["precond"], "parallelism": "single-threaded CPU"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference",
                         "sample": f"first SSP-DIRK3 step, {n_per_stage} Newton updates per stage "
                                   f"({len(times)} updates, first {warm} untimed); unmodified reference "
                                   f"sources built against the MFEM-subset shim ({src}) on '{cpu_model()}'"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "per_update_s": timed,
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c2")
    ap.add_argument("--no-dg", action="store_true", help="skip the secondary DG-form measurement")
    ap.add_argument("--no-ilu", action="store_true", help="skip the secondary block-ILU(0) measurement")
    ap.add_argument("--no-mixed", action="store_true", help="skip the secondary mixed-precision measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c3", action="store_true", help="skip the 256x256 Q3 run to T=0.2 (FP64 and mixed)")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-instance uneven batch")
    ap.add_argument("--no-serve", action="store_true", help="skip the 48-request serve sample")
    ap.add_argument("--ref-max-updates", type=int, default=12)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        ap.error("--warmup must be >= 3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference_arm(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    world, rank, local = dist_setup(args.gpus)
    try:
        line = run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
