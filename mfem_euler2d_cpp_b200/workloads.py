"""Many-instance workloads on one GPU, on the engine's batch and request-loop
entry points (eg_batch_*, eg_server_*).

batch  Uneven instances run together: `count` seeded
       simple-wave problems (gamma = 3) with nx = ny drawn from
       {8,16,24,32,48,64}, k uniform in 1..6 and alpha uniform in (15, 75)
       degrees, each advanced 3 SSP-DIRK3 steps x 3 Newton updates at CFL 1
       (HDG, block Jacobi; mixed precision by default: FP64 residual and
       refinement, FP32 preconditioner and inner Schur GMRES). Reports
       accepted Newton updates/s of the concurrent batch, of the plain FP64
       path one instance at a time and of the batch's precision one at a
       time, and checks every instance's L2 error against its FP64 run.

serve  A Poisson stream of time-advance requests (exponential inter-arrival
       times at `rate` requests/s): steps uniform in 1..10, nx = ny from
       {20,32,64,128}, k uniform in 2..8, alpha uniform in (15, 75) degrees,
       3 Newton updates per stage, CFL 1 or less where the steps would leave
       the smooth interval of the exact wave (request_cfl). Requests are submitted at their arrival
       times to a request loop with a device-memory budget; reports solves/s
       and p50/p99 latency (finish - arrival), beside the same stream served
       one request at a time by the plain FP64 path, and checks every
       request's L2 error against that run's (within 1%).

    python -m mfem_euler2d_cpp_b200.workloads batch --count 64 --seed 0
    python -m mfem_euler2d_cpp_b200.workloads serve --requests 2000 --rate 200 --seed 1

Each prints one JSON line. Inputs are synthetic and seeded (numpy
default_rng); the sampled instance list is part of the output.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import capi


# the uneven batch: nx = ny uniform over these sizes, k uniform in 1..6
C4_SIZES = (8, 16, 24, 32, 48, 64)


def batch_instances(count: int, seed: int, sizes=C4_SIZES):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(sizes))
        out.append((n, n, int(rng.integers(1, 7)), float(rng.uniform(15.0, 75.0))))
    return out


def _joint(errors):
    return float(np.sqrt(np.sum(np.square(errors))))


def l2_check(statuses, errors, ref_statuses, ref_errors, bar=0.01):
    """Every run that completed in both (status 0) has its joint L2 error
    (the 2-norm of the four component errors) within `bar` (relative) of the
    reference run's. Returns (checked, worst relative difference, all within)."""
    checked, worst, within = 0, 0.0, True
    for st, e, rst, re in zip(statuses, errors, ref_statuses, ref_errors):
        if st == 0 and rst == 0:
            e0, e1 = _joint(re), _joint(e)
            rel = abs(e1 - e0) / e0
            worst = max(worst, rel)
            within &= rel <= bar
            checked += 1
    return checked, worst, bool(within)


def run_batch(count=64, seed=0, threads=32, precision="mixed", steps=3, newton_steps=3, sizes=C4_SIZES):
    """The instances run concurrently in `precision`, against the plain FP64
    path one instance at a time (and `precision` one at a time, which
    separates what concurrency buys from what the precision buys). Every
    instance that completes in both is checked: its joint L2 error within 1%
    of the FP64 run's. Instances that fail keep their status."""
    inst = batch_instances(count, seed, sizes)
    descs = [capi.simple_wave_desc(*t) for t in inst]
    ro, keep = capi.run_options(integrator="ssp-dirk3", steps=steps, newton_steps=newton_steps, cfl=1.0,
                                form_name="hdg")
    runs = {}
    for label, prec_name, nthreads in (("batched", precision, threads), ("fp64_one_at_a_time", "fp64", 1),
                                       (f"{precision}_one_at_a_time", precision, 1)):
        prec = capi.PRECISION_MIXED if prec_name == "mixed" else capi.PRECISION_FP64
        opts = [capi.default_opts(form=capi.FORM_HDG, precision=prec) for _ in inst]
        with capi.Batch(descs, opts) as b:
            st = b.run(ro, threads=nthreads, check=False)
            statuses = [b.result(i)[0] for i in range(count)]
            errors = [list(b.result(i)[1].errors) for i in range(count)]
        runs[label] = {"seconds": st.seconds, "updates": st.updates,
                       "updates_per_s": st.updates / st.seconds if st.seconds > 0 else 0.,
                       "failed": st.failed, "statuses": statuses, "errors": errors}
    bat, ref64 = runs["batched"], runs["fp64_one_at_a_time"]
    same_prec = runs[f"{precision}_one_at_a_time"]
    checked, worst, within = l2_check(bat["statuses"], bat["errors"], ref64["statuses"], ref64["errors"])
    return {
        "metric": "accepted Newton updates/s (batched uneven instances)",
        "value": bat["updates_per_s"], "unit": "updates/s", "higher_is_better": True,
        "baseline_fp64_one_at_a_time": ref64["updates_per_s"],
        "speedup_vs_fp64_one_at_a_time": bat["updates_per_s"] / ref64["updates_per_s"],
        f"{precision}_one_at_a_time": same_prec["updates_per_s"],
        "speedup_vs_same_precision_one_at_a_time": bat["updates_per_s"] / same_prec["updates_per_s"],
        "seconds": bat["seconds"], "updates": bat["updates"],
        "failed_instances": [(i, inst[i], bat["statuses"][i]) for i in range(count) if bat["statuses"][i] != 0],
        "fp64_statuses_of_failed": [ref64["statuses"][i] for i in range(count) if bat["statuses"][i] != 0],
        "l2_check": {"instances_checked": checked, "worst_relative_difference_vs_fp64": worst,
                     "all_within_1pct": bool(within)},
        "results_identical_alone_and_batched": bat["errors"] == same_prec["errors"],
        "config": {"workload": "uneven seeded simple-wave instances (nx = ny 8..64, k 1..6)", "count": count,
                   "seed": seed, "threads": threads, "precision": precision, "steps": steps,
                   "newton_steps_per_stage": newton_steps, "sizes": list(sizes), "instances": inst},
        "data": "synthetic: seeded simple-wave instances (gamma=3)",
    }


def serve_requests(n: int, rate: float, seed: int, max_nx=128, max_k=8):
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    # meshes coarser than 20 x 20 are left out: their stages can be
    # inadmissible (status 20), in the reference as here
    sizes = [s for s in (20, 32, 64, 128) if s <= max_nx]
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        nx = int(rng.choice(sizes))
        steps = int(rng.integers(1, 11))
        out.append({"arrival": t, "nx": nx, "k": int(rng.integers(2, max_k + 1)),
                    "alpha": float(rng.uniform(15.0, 75.0)), "steps": steps, "cfl": request_cfl(nx, steps)})
    return out


def request_cfl(nx: int, steps: int) -> float:
    """CFL of a request: 1, or less when `steps` steps at CFL 1 would leave
    the simple wave's smooth interval t < 4/((gamma+1) pi) = 1/pi. A step at
    CFL c advances about c h / 2.2 with h >= 2/nx the cell width (wave
    speeds stay near 2.2 for gamma = 3), so t_end ~ steps c / (1.1 nx); the
    bound keeps t_end near 0.15."""
    return min(1.0, 0.15 * 1.1 * nx / steps)


def _serve(reqs, workers, budget_bytes, precision):
    prec = capi.PRECISION_MIXED if precision == "mixed" else capi.PRECISION_FP64
    with capi.Server(workers=workers, budget_bytes=budget_bytes) as s:
        t0 = s.clock()
        ids = []
        for r in reqs:
            wait = t0 + r["arrival"] - s.clock()
            if wait > 0:
                time.sleep(wait)
            ids.append(s.submit(r["nx"], r["nx"], r["k"], r["alpha"], steps=r["steps"], newton_steps=3,
                                cfl=r["cfl"], precision=prec))
        st = s.drain()
        res = [s.poll(i) for i in ids]
    lat = np.array([x.finish_s - x.submit_s for x in res])
    ok = [x.status == 0 for x in res]
    span = max(x.finish_s for x in res) - min(x.submit_s for x in res)
    return {"solves_per_s": sum(ok) / span, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "completed": int(st.completed), "failed": int(st.failed),
            "peak_running": int(st.peak_running), "peak_bytes": int(st.peak_bytes),
            "updates": int(sum(x.updates for x in res)), "span_s": span,
            "errors": [list(x.errors) for x in res], "statuses": [x.status for x in res]}


def run_serve(requests=2000, rate=200.0, seed=1, workers=16, budget_gb=120.0, precision="mixed", max_nx=128,
              max_k=8):
    """The request stream served by `workers` in `precision`, against the
    plain FP64 path serving the same stream one request at a time. Every
    request that completes in both is checked: its joint L2 error within 1%
    of the FP64 run's."""
    reqs = serve_requests(requests, rate, seed, max_nx, max_k)
    budget = int(budget_gb * (1 << 30))
    served = _serve(reqs, workers, budget, precision)
    single = _serve(reqs, 1, budget, "fp64")
    checked, worst, within = l2_check(served["statuses"], served["errors"], single["statuses"], single["errors"])
    for d in (served, single):
        d.pop("errors")
        d["failed_statuses"] = sorted({s for s in d.pop("statuses") if s != 0})
    return {
        "metric": "solves/s with p50/p99 request latency (served time-advance requests)",
        "value": served["solves_per_s"], "unit": "solves/s", "higher_is_better": True,
        "p50_s": served["p50_s"], "p99_s": served["p99_s"], "served": served, "fp64_one_at_a_time": single,
        "speedup_vs_fp64_one_at_a_time": served["solves_per_s"] / single["solves_per_s"]
        if single["solves_per_s"] > 0 else None,
        "l2_check": {"requests_checked": checked, "worst_relative_difference_vs_fp64": worst,
                     "all_within_1pct": bool(within)},
        "config": {"workload": "Poisson stream of simple-wave time-advance requests", "requests": requests,
                   "rate_per_s": rate, "seed": seed, "workers": workers, "budget_gb": budget_gb,
                   "precision": precision, "max_nx": max_nx, "max_k": max_k, "newton_steps_per_stage": 3},
        "data": "synthetic: seeded request stream (gamma=3)",
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    b = sub.add_parser("batch")
    b.add_argument("--count", type=int, default=64)
    b.add_argument("--seed", type=int, default=0)
    b.add_argument("--threads", type=int, default=32)
    b.add_argument("--precision", choices=("fp64", "mixed"), default="mixed")
    s = sub.add_parser("serve")
    s.add_argument("--requests", type=int, default=2000)
    s.add_argument("--rate", type=float, default=200.0)
    s.add_argument("--seed", type=int, default=1)
    s.add_argument("--workers", type=int, default=16)
    s.add_argument("--budget-gb", type=float, default=120.0)
    s.add_argument("--precision", choices=("fp64", "mixed"), default="mixed")
    s.add_argument("--max-nx", type=int, default=128)
    s.add_argument("--max-k", type=int, default=8)
    args = ap.parse_args(argv)
    if args.cmd == "batch":
        line = run_batch(args.count, args.seed, args.threads, args.precision)
    else:
        line = run_serve(args.requests, args.rate, args.seed, args.workers, args.budget_gb, args.precision,
                         args.max_nx, args.max_k)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
