"""camille_b200/lee_run: the reference's input files run through the library without its MPI driver.

CPU: ``--parse-only`` reads the deck (comments, backslash continuation, a repeated name, keyword
lookups), the PLOT3D headers, the restart's step and time and the BC file (with indices counted
from a block's end) the way the reference does, and refuses what the library does not implement;
the monopole standing in for CASE_SCATTERING_TWOCYLINDER's source reproduces the reference's.

GPU: on the golden workloads (FIX_DT at the reference's time step) the written solution file
matches the compiled reference's state within 1e-10 relative L2 and the Solver path bit for bit,
the report lines follow io::report_timeadvancing / ReportSolution::minmax; a FIX_CFL restart and
the reference's own CASE_SCATTERING_TWOCYLINDER source match the live compiled reference.
"""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

from camille_b200 import api, build, cases, plot3d

from tests.conftest import golden_case, load_golden

RUNNER = build.RUNNER


@pytest.fixture(scope="module")
def runner():
    if not os.path.isfile(RUNNER):
        build.build()
    return RUNNER


def _run(runner, wd, *args, check=True):
    p = subprocess.run([runner, "ic.q", *args], cwd=wd, capture_output=True, text=True, timeout=600)
    if check and p.returncode != 0:
        raise AssertionError(f"lee_run failed ({p.returncode}):\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
    return p


def _rewrite_deck(wd, edit):
    path = os.path.join(wd, "camille.in")
    lines = open(path).read().splitlines()
    open(path, "w").write("\n".join(edit(lines)) + "\n")


# ---------------------------------------------------------------------------------------------
# CPU: reading the inputs
# ---------------------------------------------------------------------------------------------

def test_parse_only_reads_deck_files_and_bc(runner, tmp_path):
    case = cases.curvi3d(n=16, seed=2, npulses=8, nsteps=5, halfwidth=2.0)
    case.fd_scheme, case.filter_scheme, case.filter_strength, case.filter_blend = "FDO11P", "SFO11P", 0.3, 0.7
    wd = str(tmp_path)
    case.write_reference_inputs(wd, 0.125, 17, step=3, time=0.375, report=4)

    def edit(lines):
        out = []
        for ln in lines:
            if ln.startswith("TEMPORAL_SCHEME"):
                # a comment, a continuation and a repeated name: the later line wins
                out += ["TEMPORAL_SCHEME = RUNGE_KUTTA4   # overridden below",
                        "GAMMA_SPECIFICHEAT = 1.3", "TEMPORAL_SCHEME = \\", "RUNGE_KUTTA2"]
            else:
                out.append(ln)
        return out

    _rewrite_deck(wd, edit)
    n = 16
    with open(os.path.join(wd, "bc.in"), "a") as f:
        f.write("   # indented comment line\n\n")
        f.write(f"0 neumann +eta 2 -2 0 0 -4 -0\n")
        f.write(f"0 wall_slip_kinematic -ZETA 0 -0 +1 -1 -0 -0\n")
    info = json.loads(_run(runner, wd, "--parse-only").stdout)
    assert info["num_dim"] == 3 and info["blocks"] == [[n, n, n]]
    assert info["gamma"] == 1.3 and info["rk"] == 2
    assert info["fd"][0] == api.FD["FDO11P"]
    assert info["filter"] == [api.FILTER["SFO11P"], 0, 0.3, 0.7]  # SFO11P has no ORDER_ACCURACY
    assert info["sponge"] == [case.sponge_order, case.sponge_constant]
    assert info["fix"] == "FIX_DT" and info["dt"] == 0.125 and info["num_time_steps"] == 17
    assert info["report"] == 4 and info["step"] == 3 and info["time"] == 0.375
    assert info["overset"] == "NONE" and info["monopole"] is None
    bcs = info["bc"]
    assert len(bcs) == len(case.boundaries) + 2
    for got, bd in zip(bcs, case.boundaries):
        assert got == [bd.block, cases.BC_TYPES[bd.kind], bd.dir, bd.end,
                       bd.lo[0], bd.hi[0], bd.lo[1], bd.hi[1], bd.lo[2], bd.hi[2]]
    assert bcs[-2] == [0, 100, 1, 0, 2, n - 3, 0, 0, n - 5, n - 1]
    assert bcs[-1] == [0, 201, 2, 1, 0, n - 1, 1, n - 2, n - 1, n - 1]


def test_parse_only_overset_monopole_and_twocylinder(runner, tmp_path):
    case = golden_case("cylinder2d_64")
    wd = str(tmp_path / "a")
    case.write_reference_inputs(wd, None, 40)
    info = json.loads(_run(runner, wd, "--parse-only").stdout)
    assert info["fix"] == "FIX_CFL" and info["cfl"] == case.cfl
    assert info["overset"] == "OVERTURE" and info["overset_order"] == case.overset.order
    assert info["monopole"] == [float(v) for v in case.monopole]
    assert info["blocks"] == [list(b.dims) for b in case.blocks]
    case2 = cases.pulse2d(n=48, length=4.0, sponge=8, nsteps=10)
    case2.simulation = "CASE_SCATTERING_TWOCYLINDER"
    wd2 = str(tmp_path / "b")
    case2.write_reference_inputs(wd2, 0.01, 10)
    info2 = json.loads(_run(runner, wd2, "--parse-only").stdout)
    assert info2["monopole"] == list(cases.TWOCYLINDER_SOURCE)


def test_parse_only_reads_the_harmonic_wave(runner, tmp_path):
    for case in (golden_case("waves2d_40x32"), golden_case("jet3d_14")):
        wd = str(tmp_path / case.name)
        case.write_reference_inputs(wd, 0.01, 2)
        info = json.loads(_run(runner, wd, "--parse-only").stdout)
        w = case.harmonic_wave
        hw = w.halfwidth if w.form == "WAVEFORM_GAUSSIAN_ROUNDJET" else 0.0
        assert info["wave"] == [cases.WAVE_TYPES[w.wave_type], cases.WAVE_FORMS[w.form], w.direction, w.amplitude,
                                w.wavelength, hw]
        assert [b[1] for b in info["bc"]] == [cases.BC_TYPES[bd.kind] for bd in case.boundaries]
        assert info["axisym"] is False


def test_parse_only_reads_the_jet_source(runner, tmp_path):
    case = cases.jet2d_source(nx=40, ny=32, nsteps=2)
    wd = str(tmp_path)
    case.write_reference_inputs(wd, 0.01, 2)
    info = json.loads(_run(runner, wd, "--parse-only").stdout)
    assert info["jet2d"] is True and info["monopole"] is None


def test_parse_only_reads_axisymmetry(runner, tmp_path):
    case = golden_case("axisym2d_48x32")
    wd = str(tmp_path)
    case.write_reference_inputs(wd, 0.01, 2)
    info = json.loads(_run(runner, wd, "--parse-only").stdout)
    assert info["axisym"] is True
    assert 903 in [b[1] for b in info["bc"]]
    _rewrite_deck(wd, lambda lines: ["AXISYMMETRY = TRUE, AXIS_OF_SYMMETRY = Y" if ln.startswith("AXISYMMETRY")
                                     else ln for ln in lines])
    p = _run(runner, wd, "--parse-only", check=False)
    assert p.returncode != 0 and "The axis of symmetry should be x" in p.stderr


@pytest.mark.parametrize("key,value,message", [
    ("PHYSICAL_MODEL", "LINEAR_ACOUSTICS", "the library runs LEE"),
    # check_consistency_wave (src/core/input.cpp:629-656): an acoustic wave of another shape,
    # and the amplitude range
    ("HARMONIC_WAVE", "WAVE_ACOUSTIC, AMPLITUDE = 0.1, SHAPE = WAVEFORM_GAUSSIAN_ROUNDJET, DIRECTION = X, "
     "WAVELENGTH = 2.0, HALFWIDTH = 1.0", "Unknown spatial distribution of acoustic waves."),
    ("HARMONIC_WAVE", "WAVE_ENTROPY, AMPLITUDE = 1.5, SHAPE = WAVEFORM_HOMOGENEOUS, DIRECTION = Y, "
     "WAVELENGTH = 2.0", "The wave amplitude should be between 0 and 1."),
    ("FIX_DT_OR_CFL", "FIX_NOTHING", "either DT or CFL"),
])
def test_refuses_what_the_library_does_not_implement(runner, tmp_path, key, value, message):
    case = cases.pulse2d(n=48, sponge=8, nsteps=2)
    wd = str(tmp_path)
    case.write_reference_inputs(wd, 0.01, 2)
    _rewrite_deck(wd, lambda lines: [f"{key} = {value}" if ln.split(" ")[0] == key else ln for ln in lines])
    p = _run(runner, wd, "--parse-only", check=False)
    assert p.returncode != 0 and message in p.stderr


def test_refuses_an_unimplemented_boundary_type(runner, tmp_path):
    case = cases.pulse2d(n=48, sponge=8, nsteps=2)
    wd = str(tmp_path)
    case.write_reference_inputs(wd, 0.01, 2)
    with open(os.path.join(wd, "bc.in"), "a") as f:
        f.write("0 dirichlet_harmonic_wave +XI 0 0 0 -0 0 0\n")
    p = _run(runner, wd, "--parse-only", check=False)
    assert p.returncode != 0 and "dirichlet_harmonic_wave" in p.stderr


def test_parse_only_reads_lee_scalar(runner, tmp_path):
    """PHYSICAL_MODEL = LEE_SCALAR, NUMBER_SCALAR = n with the 5 + n slot mean and restart files;
    the reference's own checks on n and on SIMULATION (src/core/input.cpp:113-117, :596-606)."""
    case = golden_case("scalar2d_40x32")
    wd = str(tmp_path)
    case.write_reference_inputs(wd, 0.01, 2)
    info = json.loads(_run(runner, wd, "--parse-only").stdout)
    assert info["scalars"] == 2
    _rewrite_deck(wd, lambda lines: ["SIMULATION = CASE_KBK_COMBUSTOR" if ln.startswith("SIMULATION") else ln
                                     for ln in lines])
    p = _run(runner, wd, "--parse-only", check=False)
    assert p.returncode != 0 and "is not implemented for PHYSICAL_MODEL = LEE_SCALAR" in p.stderr
    case.write_reference_inputs(wd, 0.01, 2)
    _rewrite_deck(wd, lambda lines: ["PHYSICAL_MODEL = LEE_SCALAR, NUMBER_SCALAR = 0"
                                     if ln.startswith("PHYSICAL_MODEL") else ln for ln in lines])
    p = _run(runner, wd, "--parse-only", check=False)
    assert p.returncode != 0 and "at least one scalar should be solved for" in p.stderr


def test_twocylinder_monopole_is_the_reference_source(oracle_lib):
    """The monopole lee_run sets for CASE_SCATTERING_TWOCYLINDER, run in the oracle, against the
    compiled reference applying its own source (src/solver/source.cpp:60-92)."""
    from oracle import run_ref
    if not run_ref.available():
        pytest.skip("oracle/_ref/camille_ref not built here")
    case = cases.pulse2d(n=48, length=4.0, sponge=8, nsteps=24)
    case.simulation = "CASE_SCATTERING_TWOCYLINDER"
    s = api.Solver(oracle_lib, case)
    dt = s.compute_dt()
    s.advance(24, dt)
    ref = run_ref.assemble(case, run_ref.run(case, nsteps=24, dt=dt)["ranks"])[0]
    assert api.rel_l2(s.download(0)[0], ref) <= 1e-13


# ---------------------------------------------------------------------------------------------
# GPU: running the case
# ---------------------------------------------------------------------------------------------

def _final_solution(wd, counter):
    qs, taus = plot3d.read_solution(os.path.join(wd, f"camille.{counter:06d}.q"))
    return qs, taus


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["pulse2d_48", "curvi3d_16", "shear2d_40x32", "wall3d_14", "cylinder2d_64",
                                  "waves2d_40x32", "jet3d_14", "axisym2d_48x32"])
def test_fix_dt_run_matches_reference_and_solver(runner, product_lib, tmp_path, name):
    case = golden_case(name)
    g = load_golden(name)
    dt, nsteps = float(g["dt"]), int(g["nsteps"])
    report = nsteps // 2 if nsteps % 2 == 0 else nsteps
    wd = str(tmp_path)
    case.write_reference_inputs(wd, dt, nsteps, report=report)
    p = _run(runner, wd)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("Time step:")]
    assert [int(ln.split(",")[0].split(":")[1]) for ln in lines] == list(range(report, nsteps + 1, report))
    qs, taus = _final_solution(wd, 1)
    assert not os.path.exists(os.path.join(wd, "camille.000002.q"))
    s = api.Solver(product_lib, case)
    s.advance(nsteps, dt)
    for b in range(len(case.blocks)):
        y, step, t = s.download(b)
        np.testing.assert_array_equal(qs[b], y)
        assert taus[b][2] == step == nsteps and taus[b][3] == t
        ref = g["stepn"] if "stepn" in g else g[f"stepn_{b}"]
        assert api.rel_l2(qs[b], ref) <= 1e-10
    # the min/max report of the last step against the written state
    rep = open(os.path.join(wd, "report", "solution", "solution")).read().splitlines()
    assert len(rep) == len(lines)
    parts = rep[-1].split(", ")[2:]
    for v, part in enumerate(parts):
        lo, hi = (float(x) for x in part.split(": ")[1].split(" ~ "))
        allv = np.concatenate([q[v].ravel() for q in qs])
        assert lo == pytest.approx(allv.min(), rel=1e-6, abs=1e-300)
        assert hi == pytest.approx(allv.max(), rel=1e-6, abs=1e-300)


@pytest.mark.gpu
def test_state_minmax_matches_the_downloaded_state(product_lib):
    case = golden_case("cylinder2d_64")
    for precision in (api.FP64, api.FP32_COMPENSATED):
        s = api.Solver(product_lib, case, precision=precision)
        s.advance(7, s.compute_dt())
        mn, mx = s.state_minmax()
        ys = [s.download(b)[0] for b in range(len(case.blocks))]
        for v in range(5):
            allv = np.concatenate([y[v].ravel() for y in ys])
            assert mn[v] == allv.min() and mx[v] == allv.max()


@pytest.mark.gpu
def test_fix_cfl_restart_matches_the_live_reference(runner, tmp_path):
    from oracle import run_ref
    case = cases.curvi3d(n=16, seed=3, npulses=6, nsteps=12, halfwidth=2.0)
    wd = str(tmp_path)
    case.write_reference_inputs(wd, None, 15, step=3, time=0.25, report=4)
    p = _run(runner, wd)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("Time step:")]
    assert [int(ln.split(",")[0].split(":")[1]) for ln in lines] == [4, 8, 12]
    # step 15 is not a report step: no solution file beyond the restart state's
    assert os.path.exists(os.path.join(wd, "camille.000000.q"))
    assert not os.path.exists(os.path.join(wd, "camille.000001.q"))
    # to step 12, a report step: state, time and dt against the reference's
    wd2 = str(tmp_path / "twelve")
    case.write_reference_inputs(wd2, None, 12, step=3, time=0.25, report=3)
    _run(runner, wd2)
    qs, taus = _final_solution(wd2, 1)
    ref = run_ref.run(case, nsteps=12, dt=None, step=3, time=0.25)
    r0 = ref["ranks"][0]
    st = run_ref.assemble(case, ref["ranks"])[0]
    assert taus[0][2] == r0["step"] == 12
    assert abs(taus[0][3] - r0["time"]) <= 1e-14 * r0["time"]
    assert api.rel_l2(qs[0], st) <= 1e-10
    dt_printed = float(lines[-1].split("dt: ")[1].split(",")[0])
    assert dt_printed == pytest.approx(r0["dt"], rel=1e-6)


@pytest.mark.gpu
def test_twocylinder_source_matches_the_live_reference(runner, product_lib, tmp_path):
    from oracle import run_ref
    case = cases.pulse2d(n=48, length=4.0, sponge=8, nsteps=24)
    case.simulation = "CASE_SCATTERING_TWOCYLINDER"
    dt = api.Solver(product_lib, case).compute_dt()
    wd = str(tmp_path)
    case.write_reference_inputs(wd, dt, 24, report=24)
    _run(runner, wd)
    qs, _ = _final_solution(wd, 1)
    ref = run_ref.assemble(case, run_ref.run(case, nsteps=24, dt=dt)["ranks"])[0]
    assert api.rel_l2(qs[0], ref) <= 1e-10
    # the source did act: without it the state differs
    plain = cases.pulse2d(n=48, length=4.0, sponge=8, nsteps=24)
    s = api.Solver(product_lib, plain)
    s.advance(24, dt)
    assert api.rel_l2(s.download(0)[0], ref) > 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["scalar2d_40x32", "scalar3d_14", "scalar_cylinder2d_64"])
def test_lee_scalar_run_matches_reference_and_solver(runner, product_lib, tmp_path, name):
    """A LEE_SCALAR deck: the 5 + n slot solution file (function format) equals the Solver's state bit
    for bit and the reference's within 1e-10; the report line carries the scalars under the
    reference's names."""
    from tests.test_oracle_pin import full_state
    case = golden_case(name)
    g = load_golden(name)
    dt, nsteps = float(g["dt"]), int(g["nsteps"])
    nv = 5 + case.num_scalars
    wd = str(tmp_path)
    case.write_reference_inputs(wd, dt, nsteps, report=nsteps)
    _run(runner, wd)
    # more than five slots: the PLOT3D function format, as the reference writes it
    qs = plot3d.read_function(os.path.join(wd, "camille.000001.q"))
    s = api.Solver(product_lib, case)
    s.advance(nsteps, dt)
    for b in range(len(case.blocks)):
        np.testing.assert_array_equal(qs[b], full_state(s, b))
        ref = g["stepn"] if "stepn" in g else g[f"stepn_{b}"]
        assert api.rel_l2(qs[b], ref) <= 1e-10
    rep = open(os.path.join(wd, "report", "solution", "solution")).read().splitlines()[-1]
    names = [part.split(": ")[0] for part in rep.split(", ")[2:]]
    assert names[5:] == ["Z0'", "Z01'", "Z012'"][:case.num_scalars]
    for k in range(case.num_scalars):
        lo, hi = (float(x) for x in rep.split(", ")[2 + 5 + k].split(": ")[1].split(" ~ "))
        allv = np.concatenate([q[5 + k].ravel() for q in qs])
        assert lo == pytest.approx(allv.min(), rel=1e-6, abs=1e-300)
        assert hi == pytest.approx(allv.max(), rel=1e-6, abs=1e-300)
