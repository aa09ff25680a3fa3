"""Build the compiled reference with its time advance handed to the B200 library (test
infrastructure): the reference's own translation units as oracle/build_ref.py compiled them
(oracle/_ref/obj, the same patches and flags), its own src/core/main.cpp as the driver, and
oracle/ref_solve_b200.cpp in place of src/solver/solver.cpp, linked against
camille_b200/liblee_b200.so. Output: oracle/_ref/camille_b200_solve (git-ignored; it travels to
the GPU box with the library it links by a relative rpath). tests/test_integration_gpu.py runs it
on the reference's own input files.

Usage: python oracle/build_integration.py   (after oracle/build_ref.py and camille_b200/build.py)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
OWN = os.path.join(OUT, "integration_obj")   # kept apart: oracle/build_ref.py links every object in OBJ
WORK = os.path.join(OUT, "src")
MINIMPI = os.path.join(HERE, "minimpi")
EXE = os.path.join(OUT, "camille_b200_solve")
LIBDIR = os.path.join(ROOT, "camille_b200")

# the reference's flags (see oracle/build_ref.py for why the old string ABI)
CXX = ["g++", "-O3", "-std=c++11", "-w", "-D_GLIBCXX_USE_CXX11_ABI=0", "-I", MINIMPI, "-I", WORK]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stderr[-4000:])


def available() -> bool:
    return os.path.isfile(EXE) and os.access(EXE, os.X_OK)


def build() -> str:
    if not os.path.isdir(OBJ) or not os.path.isdir(WORK):
        raise FileNotFoundError("build the reference first: python oracle/build_ref.py")
    lib = os.path.join(LIBDIR, "liblee_b200.so")
    if not os.path.isfile(lib):
        raise FileNotFoundError("build the library first: python camille_b200/build.py")
    os.makedirs(OWN, exist_ok=True)
    main_o = os.path.join(OWN, "main.o")
    solve_o = os.path.join(OWN, "solve.o")
    _run(CXX + ["-c", os.path.join(WORK, "core", "main.cpp"), "-o", main_o])
    _run(CXX + ["-I", os.path.join(WORK, "solver"), "-I", os.path.join(ROOT, "include"), "-c",
                os.path.join(HERE, "ref_solve_b200.cpp"), "-o", solve_o])
    skip = {"driver.o", "solver_solver.o"}
    objs = sorted(os.path.join(OBJ, o) for o in os.listdir(OBJ) if o.endswith(".o") and o not in skip)
    rel = os.path.relpath(LIBDIR, OUT)
    _run(["g++", "-O3", "-o", EXE, main_o, solve_o] + objs +
         ["-L", LIBDIR, "-llee_b200", "-Wl,-rpath,$ORIGIN/" + rel, "-lpthread"])
    return EXE


if __name__ == "__main__":
    print(build())
    sys.exit(0)
