"""Run one engine operator repeatedly on a simple-wave state, for kernel
timing and Nsight Compute captures.

    python -m mfem_euler2d_cpp_b200.profile_kernels --nx 64 --ny 64 --k 4 --op condense --reps 3

The state is the projected initial wave frozen at a CFL-1 stage step of the
first SSP-DIRK3 stage; each operator is called through the C-ABI and timed
with CUDA events on the engine's stream (printed as one JSON line).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json

import numpy as np

from . import capi

OPS = ("condense", "schur_apply", "recover", "pc_factor", "pc_apply", "dg_apply", "residual",
       "linear_solve", "dg_jacobi")
PRECONDS = {"block-jacobi": capi.PC_JACOBI, "block-ilu0": capi.PC_ILU0}
ASSEMBLY = {"partial": capi.ASSEMBLY_PARTIAL, "element": capi.ASSEMBLY_ELEMENT, "full": capi.ASSEMBLY_FULL}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--nx", type=int, default=64)
    ap.add_argument("--ny", type=int, default=64)
    ap.add_argument("--k", type=int, default=4)
    ap.add_argument("--alpha", type=float, default=30.0)
    ap.add_argument("--op", choices=OPS, default="condense")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--precond", choices=sorted(PRECONDS), default="block-jacobi")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--assembly", choices=sorted(ASSEMBLY), default="partial")
    ap.add_argument("--form", choices=("dg", "hdg"), default=None,
                    help="form of the context (default: dg for dg_apply/dg_jacobi, hdg otherwise)")
    args = ap.parse_args(argv)
    lib = capi.load()
    if args.form is None:
        form = capi.FORM_DG if args.op in ("dg_apply", "dg_jacobi") else capi.FORM_HDG
    else:
        form = capi.FORM_DG if args.form == "dg" else capi.FORM_HDG
    d = capi.simple_wave_desc(args.nx, args.ny, args.k, args.alpha)
    prec = capi.PRECISION_MIXED if args.precision == "mixed" else capi.PRECISION_FP64
    opts = capi.default_opts(form=form, precond=PRECONDS[args.precond], precision=prec,
                             assembly=ASSEMBLY[args.assembly])
    with capi.Context(d, opts) as ctx:
        ctx.initial()
        rate = ctx.freeze(1e-3)
        dt = 0.24169426078821 / rate  # first SSP-DIRK3 stage at CFL 1
        ctx.freeze(dt)
        u = ctx.download("U")
        ctx.upload("OLD", u * 0.999)
        ctx.set_dt(dt)
        ctx.residual()
        if form == capi.FORM_HDG:
            ctx.condense()
            ctx.pc_factor(True)
        else:
            ctx.pc_factor(True)
        rng = np.random.default_rng(0)
        vb = rng.standard_normal(ctx.nu)
        vt = rng.standard_normal(ctx.nl)
        out_counts = []
        lib.eg_profile_reset(ctx.h)
        lib.eg_profile_enable(ctx.h, 1)
        for _ in range(args.reps):
            if args.op == "condense":
                ctx.condense()
            elif args.op == "schur_apply":
                ctx.schur_apply(vt)
            elif args.op == "recover":
                ctx.recover(vt)
            elif args.op in ("pc_factor", "dg_jacobi"):
                ctx.pc_factor(True)
            elif args.op == "pc_apply":
                ctx.pc_apply(vt if form == capi.FORM_HDG else vb)
            elif args.op == "dg_apply":
                ctx.dg_apply(vb)
            elif args.op == "residual":
                ctx.residual()
            elif args.op == "linear_solve":
                rhs = ctx.download("RHS") if form == capi.FORM_HDG else -ctx.download("R")
                _, _, st = ctx.linear_solve(rhs)
                out_counts.append(st.count)
        names = ["residual", "dg_apply", "dg_jacobi", "condense", "schur_apply", "recover",
                 "recovered_residual", "schur_jacobi", "pc_apply", "krylov", "freeze", "admissible",
                 "vector"]
        out = {"op": args.op, "nx": args.nx, "ny": args.ny, "k": args.k, "reps": args.reps,
               "precond": args.precond, "precision": args.precision, "assembly": args.assembly}
        if out_counts:
            out["krylov_counts"] = out_counts
        for i, name in enumerate(names):
            ms, cnt = C.c_double(), C.c_longlong()
            lib.eg_profile_query(ctx.h, i, C.byref(ms), C.byref(cnt))
            if cnt.value:
                out[name] = {"ms": ms.value, "launches": cnt.value}
        print(json.dumps(out))


if __name__ == "__main__":
    main()
