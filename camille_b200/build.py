"""Build camille_b200/liblee_b200.so, the sm_100a CUDA library behind include/lee_b200.h, and
camille_b200/lee_run, the deck-driven runner linked against it.

nvcc cross-compiles for sm_100a without a GPU. The setup kernels (lee_setup.cu) are
compiled with --fmad=false so the FP64 metric, Jacobian and mean-gradient generation
rounds like the reference's x86-64 build; the time-advance kernels use FMA.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liblee_b200.so")
RUNNER = os.path.join(PKG, "lee_run")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")] + ARCH
UNITS = {
    "lee_setup.cu": ["--fmad=false"],
    "lee_step.cu": [],
    "lee_tma.cu": [],
    "lee_capi.cu": [],
    "lee_host_core.cu": [],
    "lee_host_setup.cu": [],
    "lee_host_kernels.cu": [],
    "lee_host_batch.cu": [],
    "lee_host_step.cu": [],
    "lee_host_adjoint.cu": [],
    "lee_host_overset.cu": [],
    "lee_static.cu": [],
    "lee_bc.cu": [],
    "lee_adjoint.cu": [],
    "lee_batch.cu": [],
    "lee_filter.cu": [],
    "lee_filter_pair.cu": [],
    "lee_stage_pair.cu": [],
    "lee_adjoint_tma.cu": [],
    "lee_adjoint_gen.cu": [],
    "lee_host_adjoint_gen.cu": [],
    "lee_host_scalar.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isfile(cand) or cand == "nvcc"):
            return cand
    return "nvcc"


def _compile(args: list[str]) -> None:
    r = subprocess.run(args, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed: " + " ".join(args) + "\n" + r.stdout[-2000:] + r.stderr[-6000:])


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    headers.append(os.path.join(ROOT, "include", "lee_b200.h"))
    newest_header = max(os.path.getmtime(h) for h in headers)
    jobs, objs = [], []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
        objs.append(obj)
        fresh = os.path.isfile(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header)
        if not fresh:
            extra2 = list(extra) + (["-Xptxas", "-v"] if ptxas_info else [])
            jobs.append([nvcc()] + COMMON + extra2 + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        list(ex.map(_compile, jobs))
    if jobs or not os.path.isfile(LIB):
        _compile([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"])
    runner_src = os.path.join(CSRC, "lee_run.cpp")
    if not os.path.isfile(RUNNER) or os.path.getmtime(RUNNER) < max(os.path.getmtime(LIB), os.path.getmtime(runner_src)):
        # the deck-driven runner links the library by name and finds it beside itself
        _compile(["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), runner_src, "-o", RUNNER,
                  "-L", PKG, "-llee_b200", "-Wl,-rpath,$ORIGIN"])
    if verbose:
        print(LIB)
        print(RUNNER)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
