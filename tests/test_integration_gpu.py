"""The boundary proved end to end: the compiled reference with its src/solver/solver.cpp replaced by
the binding oracle/ref_solve_b200.cpp (built by oracle/build_integration.py), linked against the
CUDA library. The reference's own main, deck reader, PLOT3D readers, BC file, sponge strengths,
report line and solution writer run unchanged; only the time advance goes through the C ABI.

GPU: on the golden workloads (FIX_DT at the reference's time step, one report at the last step)
the solution file that the reference's io::write_solution_on_the_fly writes matches the golden
state of the compiled reference within 1e-10 relative L2; a FIX_CFL run matches the live compiled
reference's own FIX_CFL run, dt sequence included. CPU: without a GPU the binding stops with the
library's message (camille's graceful_exit returns 0, so the message is the signal).
"""
from __future__ import annotations

import glob
import os
import re
import subprocess

import numpy as np
import pytest

from camille_b200 import api, plot3d
from oracle import build_integration, run_ref
from tests.conftest import golden_case, load_golden

EXE = build_integration.EXE


def _binary():
    if not build_integration.available():
        if not run_ref.available():
            pytest.skip("oracle/_ref is not built (python oracle/build_ref.py)")
        build_integration.build()
    return EXE


def _run(wd, ic, env_extra=None):
    env = dict(os.environ, ORACLE_NO_WRITE="1")
    env.update(env_extra or {})
    return subprocess.run([_binary(), ic], cwd=wd, env=env, capture_output=True, text=True, timeout=600)


def _written_solution(wd, nvar=5):
    """The last solution file; with more than five slots the reference writes it in the PLOT3D
    function format (io::write_solution, src/io/io.cpp:740-760)."""
    out = sorted(f for f in glob.glob(os.path.join(wd, "*.q")) if os.path.basename(f) not in ("ic.q", "mean.q"))
    assert out, f"no solution file written in {sorted(os.listdir(wd))}"
    if nvar != 5:
        return plot3d.read_function(out[-1])[0]
    fields, _ = plot3d.read_solution(out[-1], nvar=nvar)
    return fields[0]


def test_binding_without_a_gpu_stops_with_the_library_message(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    case = golden_case("pulse2d_48")
    ic = case.write_reference_inputs(str(tmp_path), 0.1, 2, report=2)
    p = _run(str(tmp_path), ic)
    assert ">>> lee_b200: lee_create" in p.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["pulse2d_48", "curvi3d_16", "shear2d_40x32", "waves2d_40x32"])
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_reference_driver_through_the_c_abi(tmp_path, name, precision):
    g = load_golden(name)
    case = golden_case(name)
    n = int(g["nsteps"])
    wd = str(tmp_path)
    ic = case.write_reference_inputs(wd, float(g["dt"]), n, report=n)
    p = _run(wd, ic, {"LEE_B200_PRECISION": precision})
    assert p.returncode == 0 and "lee_b200:" not in p.stdout, p.stdout[-2000:] + p.stderr[-2000:]
    # the reference's report line of the last step, printed by its own io::report_timeadvancing
    assert re.search(rf"Time step:\s+{n}\b", p.stdout), p.stdout[-1500:]
    y = _written_solution(wd)
    if precision == "fp64":
        assert api.rel_l2(y, g["stepn"]) <= 1e-10
    else:
        assert api.rel_l2(y[4], g["stepn"][4]) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_lee_scalar_deck_through_the_c_abi(tmp_path, precision):
    """PHYSICAL_MODEL = LEE_SCALAR: the reference's driver hands its 5 + n slots to the library
    (lee_set_scalars, lee_set_mean_scalars, lee_upload_scalars, lee_download_scalars) and writes
    them with its own solution writer."""
    name = "scalar2d_40x32"
    g = load_golden(name)
    case = golden_case(name)
    n = int(g["nsteps"])
    nv = 5 + case.num_scalars
    wd = str(tmp_path)
    ic = case.write_reference_inputs(wd, float(g["dt"]), n, report=n)
    p = _run(wd, ic, {"LEE_B200_PRECISION": precision})
    assert p.returncode == 0 and "lee_b200:" not in p.stdout, p.stdout[-2000:] + p.stderr[-2000:]
    y = _written_solution(wd, nvar=nv)
    if precision == "fp64":
        assert api.rel_l2(y, g["stepn"]) <= 1e-10
    else:
        for v in range(4, nv):
            assert api.rel_l2(y[v], g["stepn"][v]) <= 1e-5


@pytest.mark.gpu
def test_fix_cfl_through_the_c_abi_matches_the_reference(tmp_path):
    if not run_ref.available():
        pytest.skip("oracle/_ref is not built")
    case = golden_case("curvi3d_16")
    n = 6
    ref = run_ref.run(case, mode="run", nsteps=n, dt=None)
    yr = run_ref.assemble(case, ref["ranks"])[0]
    wd = str(tmp_path)
    ic = case.write_reference_inputs(wd, None, n, report=n)
    p = _run(wd, ic)
    assert p.returncode == 0 and "lee_b200:" not in p.stdout, p.stdout[-2000:]
    y = _written_solution(wd)
    assert api.rel_l2(y, yr) <= 1e-10
