"""In-tree build of the CUDA engine and the euler2d command line.

Outputs (git-ignored, shipped with the tree):
  mfem_euler2d_cpp_b200/lib/libeuler2d_cuda.so   C-ABI of include/euler2d_cuda.h
  mfem_euler2d_cpp_b200/bin/euler2d              drop-in command line (--device cuda)

Device code is compiled for sm_100a only. The CUDA runtime is linked
statically so the library has no run-time dependency on a libcudart path.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libeuler2d_cuda.so"
CLI = PKG / "bin" / "euler2d"

CUDA_SOURCES = ["eg_cell.cu", "eg_hdg.cu", "eg_krylov.cu", "eg_api.cu", "eg_run.cu", "eg_ilu.cu", "eg_mixed.cu", "eg_noalloc.cu", "eg_dginv.cu", "eg_field.cu", "eg_dense.cu"]
CXX_SOURCES = ["eg_setup.cpp", "eg_batch.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + proc.stdout + proc.stderr)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    CLI.parent.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "euler2d_cuda.h"]
    jobs = []
    objs = []
    for src in CUDA_SOURCES:
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if _stale(obj, [CSRC / src] + headers):
            cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", "-c", str(CSRC / src), "-o", str(obj)]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for src in CXX_SOURCES:
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if _stale(obj, [CSRC / src] + headers):
            jobs.append(["g++", "-O3", "-std=c++17", "-fPIC", "-c", str(CSRC / src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(_run, jobs))
    if _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "--cudart=static", "-o", str(LIB), *map(str, objs)])
    main_src = CSRC / "euler2d_main.cpp"
    if _stale(CLI, [main_src, LIB, ROOT / "include" / "euler2d_cuda.h"]):
        _run(["g++", "-O2", "-std=c++17", "-o", str(CLI), str(main_src), f"-L{LIB.parent}",
              "-leuler2d_cuda", "-Wl,-rpath,$ORIGIN/../lib"])
    if verbose:
        print(f"built {LIB} and {CLI}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
