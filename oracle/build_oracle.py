"""Compile the C restatement (oracle/lee_oracle.c) into oracle/liblee_oracle.so.

Test infrastructure only. Built without FMA contraction, like the reference's
own x86-64 -O3 build, so the restatement's rounding follows the reference's. The point
and line loops run on all host threads (OpenMP); each point's arithmetic is unchanged.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblee_oracle.so")


def build() -> str:
    src = os.path.join(HERE, "lee_oracle.c")
    if os.path.isfile(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    cmd = ["gcc", "-O2", "-std=c11", "-D_GNU_SOURCE", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp",
           "-Wall", "-Wno-unused-variable", "-o", LIB, src, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build())
    sys.exit(0)
