"""Build the camille reference as the oracle (test infrastructure only).

Recipe: copy the reference's ``src/`` from the read-only checkout into
``oracle/_ref/src`` (git-ignored), apply the documented oracle patches there,
and compile every translation unit of the reference's own build list
(``src/*/Makefile`` FILE_SRC) with g++ -O3 -std=c++11 against ``minimpi``,
linking ``ref_driver.cpp`` in place of ``src/core/main.cpp``. Outputs go only to
``oracle/_ref/``: ``camille_ref`` (the solver) and ``minimpi_run`` (the
multi-rank launcher). Nothing is copied into the repository's history.

Patches (each a small edit made by this script, not a stored diff):
  P1  src/metrics/metrics.cpp:290-307 -- the 3-D branch of compute_Jacobian
      exits; enable the determinant formula that is present there as comments.
  P2  src/solver/source.cpp:98-100 -- the empty CASE_KBK_COMBUSTOR source branch
      calls oracle_monopole_source() (ref_patch_source.cpp), which is active
      only when ORACLE_MONOPOLE is set.
  P3  src/core/simulation.cpp:222-226 -- the five initial-data writes are
      skipped when ORACLE_NO_WRITE is set (they write GBs at 256^3).

Usage: python oracle/build_ref.py [--src /path/to/reference] [--jobs N]
(the default source is $CAMILLE_REFERENCE, else the read-only checkout, see reference_root)
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
MINIMPI = os.path.join(HERE, "minimpi")

# The reference's own per-directory build lists (src/*/Makefile FILE_SRC),
# without src/core/main.cpp, which ref_driver.cpp replaces.
TUS = {
    "core": ["input.cpp", "state.cpp", "simulation.cpp"],
    "geometry": ["geometry.cpp"],
    "io": ["tecplot.cpp", "fluent.cpp", "plot3d.cpp", "overture.cpp", "io.cpp"],
    "math": ["matrix.cpp", "math.cpp"],
    "metrics": ["metrics.cpp"],
    "overset": ["overset.cpp"],
    "parallel": ["parallel.cpp", "decomp.cpp"],
    "solver": ["solver.cpp", "temporal_discretization.cpp", "source.cpp",
               "spatial_discretization.cpp", "boundary_condition.cpp"],
}
C_TUS = {"io": ["plot3d_format.c"]}


def _patch_p1(path: str) -> None:
    lines = open(path).read().split("\n")
    exit_idx = [i for i, l in enumerate(lines) if "3-D Jacobian computation is not implemented yet" in l]
    if len(exit_idx) != 1:
        raise RuntimeError("P1: anchor not found exactly once")
    i0 = exit_idx[0]
    start = next(i for i in range(i0, len(lines)) if re.match(r"^\s*//\s*for \(int k", lines[i]))
    end = next(i for i in range(start, len(lines)) if re.match(r"^\s*//\s*\} // i\s*$", lines[i]))
    for i in range(start, end + 1):
        lines[i] = re.sub(r"^(\s*)//", r"\1", lines[i], count=1)
    del lines[i0]
    open(path, "w").write("\n".join(lines))


def _patch_p2(path: str) -> None:
    s = open(path).read()
    pat = re.compile(r'(else if \(mystate->simulation == "CASE_KBK_COMBUSTOR"\)\s*\{)(\s*\})')
    if len(pat.findall(s)) != 1:
        raise RuntimeError("P2: anchor not found exactly once")
    s = pat.sub(r"\1\n      oracle_monopole_source(mygrid, mystate, rhs, time);\2", s)
    decl = ("void oracle_monopole_source(Geometry::StructuredGrid *, State *, double **, double);\n\n"
            "namespace source {")
    s = s.replace("namespace source {", decl, 1)
    open(path, "w").write(s)


def _patch_p3(path: str) -> None:
    s = open(path).read()
    n = 0
    for call in ("io::write_grid(", "io::write_metrics(", "io::write_solution(",
                 "io::write_solution_mean(", "io::write_solution_aux("):
        pat = re.compile(r"^(\s*)" + re.escape(call), re.M)
        s, k = pat.subn(r'\1if (!std::getenv("ORACLE_NO_WRITE")) ' + call, s, count=1)
        n += k
    if n != 5:
        raise RuntimeError("P3: anchors not found")
    open(path, "w").write(s)


def _make_writable(root: str) -> None:
    for d, _, files in os.walk(root):
        os.chmod(d, 0o755)
        for f in files:
            os.chmod(os.path.join(d, f), 0o644)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: " + " ".join(cmd) + "\n" + r.stderr[-4000:])


def build(src_root: str, jobs: int = 8) -> str:
    src = os.path.join(src_root, "src")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference sources not found under {src_root}")
    work = os.path.join(OUT, "src")
    obj = os.path.join(OUT, "obj")
    if os.path.isdir(work):
        _make_writable(work)
        shutil.rmtree(work)
    shutil.copytree(src, work)
    _make_writable(work)
    os.makedirs(obj, exist_ok=True)
    _patch_p1(os.path.join(work, "metrics", "metrics.cpp"))
    _patch_p2(os.path.join(work, "solver", "source.cpp"))
    _patch_p3(os.path.join(work, "core", "simulation.cpp"))

    # -D_GLIBCXX_USE_CXX11_ABI=0: src/core/macros_inlines.h's cstr_to_constchar
    # returns c_str() of a by-value std::string copy, which the deck tokenizer
    # (src/core/input.cpp:956-958) hands to strtok. That pointer is valid only
    # with the copy-on-write strings the reference was written against; with the
    # C++11 string ABI it dangles and the deck parses as garbage.
    cxx = ["g++", "-O3", "-std=c++11", "-w", "-D_GLIBCXX_USE_CXX11_ABI=0", "-I", MINIMPI, "-I", work]
    jobs_list = []
    for d, files in TUS.items():
        for f in files:
            jobs_list.append(cxx + ["-c", os.path.join(work, d, f), "-o",
                                    os.path.join(obj, f"{d}_{f[:-4]}.o")])
    for d, files in C_TUS.items():
        for f in files:
            jobs_list.append(["gcc", "-O3", "-w", "-c", os.path.join(work, d, f), "-o",
                              os.path.join(obj, f"{d}_{f[:-2]}.o")])
    for f, name in ((os.path.join(HERE, "ref_driver.cpp"), "driver.o"),
                    (os.path.join(HERE, "ref_patch_source.cpp"), "patch_source.o"),
                    (os.path.join(MINIMPI, "minimpi.cpp"), "minimpi.o")):
        jobs_list.append(cxx + ["-c", f, "-o", os.path.join(obj, name)])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(_run, jobs_list))
    objs = sorted(os.path.join(obj, o) for o in os.listdir(obj) if o.endswith(".o"))
    exe = os.path.join(OUT, "camille_ref")
    _run(["g++", "-O3", "-o", exe] + objs + ["-lpthread"])
    _run(["g++", "-O2", "-std=c++11", "-o", os.path.join(OUT, "minimpi_run"),
          os.path.join(MINIMPI, "minimpi_run.cpp")])
    return exe


def reference_root() -> str:
    """Where the reference checkout lies: $CAMILLE_REFERENCE, else the read-only checkout this
    recipe was written against."""
    return os.environ.get("CAMILLE_REFERENCE", "/root/reference")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=reference_root())
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args()
    print(build(a.src, a.jobs))
    return 0


if __name__ == "__main__":
    sys.exit(main())
