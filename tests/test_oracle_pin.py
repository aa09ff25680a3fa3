"""Pin the CPU oracle (oracle/lee_oracle.c) to the camille reference.

1. Against the committed golden fixtures (outputs of the compiled reference, made by
   tests/golden/make_golden.py): setup products, one RHS, one filter, the FIX_CFL dt,
   and the state after 1 and N steps must match to the last bit.
2. Against the compiled reference run live (skipped where oracle/_ref is not built):
   the other scheme combinations the reference offers (FDO11P, SFO11P, RK2, the
   4th-order filter) and the sponge-free 2-D case.
"""
from __future__ import annotations

import numpy as np
import pytest

from camille_b200 import api, cases
from tests.conftest import golden_case, load_golden

NAMES = ["pulse2d_48", "curvi3d_16", "shear2d_40x32", "wall3d_14", "waves2d_40x32", "jet3d_14", "axisym2d_48x32"]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_setup_matches_golden(oracle_lib, name):
    g = load_golden(name)
    case = golden_case(name)
    s = api.Solver(oracle_lib, case)
    np.testing.assert_array_equal(s.get_setup(0, api.SETUP_METRICS), g["metrics"])
    np.testing.assert_array_equal(s.get_setup(0, api.SETUP_JACOBIAN)[0], g["jacobian"])
    np.testing.assert_array_equal(s.get_setup(0, api.SETUP_MEAN_GRADIENT), g["mean_gradient"])
    np.testing.assert_array_equal(s.get_setup(0, api.SETUP_SPONGE)[0], g["sponge"])
    assert s.compute_dt() == float(g["dt"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_operators_match_golden(oracle_lib, name):
    g = load_golden(name)
    case = golden_case(name)
    s = api.Solver(oracle_lib, case)
    np.testing.assert_array_equal(s.eval_rhs(0, 0.0), g["rhs"])
    s.apply_filter()
    np.testing.assert_array_equal(s.download(0)[0], g["filter"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_steps_match_golden(oracle_lib, name):
    g = load_golden(name)
    case = golden_case(name)
    dt = float(g["dt"])
    s = api.Solver(oracle_lib, case)
    s.advance(1, dt)
    y, step, t = s.download(0)
    np.testing.assert_array_equal(y, g["step1"])
    assert step == 1 and t == dt
    s.advance(int(g["nsteps"]) - 1, dt)
    np.testing.assert_array_equal(s.download(0)[0], g["stepn"])


def _live_cases():
    c1 = cases.curvi3d(n=14, nsteps=3, halfwidth=2.0)
    c1.fd_scheme, c1.filter_scheme, c1.filter_strength = "FDO11P", "SFO11P", 0.2
    c2 = cases.pulse2d(n=40, length=39 * 100.0 / 255.0, sponge=6, nsteps=4)
    c2.rk, c2.filter_order = "RUNGE_KUTTA2", 4
    c3 = cases.pulse2d(n=36, length=35 * 100.0 / 255.0, sponge=0, nsteps=3)
    c3.filter_blend = 0.75
    c4 = cases.curvi3d(n=12, nsteps=2, mach=0.3, halfwidth=2.0)
    c4.filter_scheme = "NONE"
    # the wave forms the golden fixtures leave out (acoustic homogeneous along y, entropy
    # homogeneous along z in 2-D), and the plane wave along y with RK2
    W = cases.HarmonicWave
    c5 = cases.waves2d(nx=24, ny=20, nsteps=6, wave=W("WAVE_ACOUSTIC", "WAVEFORM_HOMOGENEOUS", 1, 2e-3, 3.0))
    c6 = cases.waves2d(nx=24, ny=20, nsteps=6, wave=W("WAVE_ENTROPY", "WAVEFORM_HOMOGENEOUS", 2, 1e-3, 5.0))
    c7 = cases.jet3d(n=12, nsteps=3, wave=W("WAVE_ACOUSTIC", "WAVEFORM_PLANE", 1, 1e-3, 5.0))
    c7.rk = "RUNGE_KUTTA2"
    c8 = cases.axisym2d(nx=32, nr=20, nsteps=6)
    c8.rk, c8.filter_scheme, c8.filter_strength = "RUNGE_KUTTA2", "SFO11P", 0.25
    c9 = cases.jet2d_source(nx=40, ny=32, nsteps=8)
    return {"axisym_rk2_sfo11p_2d": c8, "jet2d_source_2d": c9, "fdo11p_sfo11p_3d": c1, "rk2_filter4_2d": c2, "blend_2d": c3, "nofilter_3d": c4,
            "wave_acoustic_homogeneous_2d": c5, "wave_entropy_homogeneous_2d": c6, "wave_plane_rk2_3d": c7}


@pytest.mark.parametrize("label", list(_live_cases().keys()))
def test_oracle_matches_reference_live(oracle_lib, label):
    from oracle import run_ref
    if not run_ref.available():
        pytest.skip("oracle/_ref/camille_ref not built here")
    case = _live_cases()[label]
    s = api.Solver(oracle_lib, case)
    r1 = run_ref.run(case, mode="run", nsteps=1, dt=None)
    dt = s.compute_dt()
    assert dt == r1["result"]["dt"]
    ref_rhs = run_ref.assemble(case, run_ref.run(case, mode="rhs")["ranks"])[0]
    np.testing.assert_array_equal(s.eval_rhs(0, 0.0), ref_rhs)
    ref = run_ref.assemble(case, run_ref.run(case, mode="run", nsteps=case.nsteps, dt=dt)["ranks"])[0]
    s.advance(case.nsteps, dt)
    np.testing.assert_array_equal(s.download(0)[0], ref)


def overset_case(name: str):
    from tests.golden.make_golden import OVERSET_WORKLOADS
    return OVERSET_WORKLOADS[name]()


def check_overset_maps(solver, g, case):
    """Receiver and donor maps, normalised weights and iblank equal the reference's
    (per donor block, in file order, as overset::initialize_donor lists them)."""
    m = solver.get_overset()
    for b in range(len(case.blocks)):
        sel = m["donor_block"] == b
        np.testing.assert_array_equal(m["donor_l0"][sel], g[f"donor_l0_{b}"])
        np.testing.assert_array_equal(m["weights"][sel], g[f"weights_{b}"])
        np.testing.assert_array_equal(m["recv_l0"][m["recv_block"] == b], g[f"recv_l0_{b}"])


OVERSET_NAMES = ["cylinder2d_64", "holes2d", "holes3d"]


@pytest.mark.parametrize("name", OVERSET_NAMES)
def test_oracle_overset_matches_golden(oracle_lib, name):
    g = load_golden(name)
    case = overset_case(name)
    s = api.Solver(oracle_lib, case)
    check_overset_maps(s, g, case)
    assert s.compute_dt() == float(g["dt"])
    for b in range(len(case.blocks)):
        np.testing.assert_array_equal(s.eval_rhs(b, 0.0), g[f"rhs_{b}"])
    dt = float(g["dt"])
    s.advance(1, dt)
    for b in range(len(case.blocks)):
        np.testing.assert_array_equal(s.download(b)[0], g[f"step1_{b}"])
    s.advance(int(g["nsteps"]) - 1, dt)
    for b in range(len(case.blocks)):
        np.testing.assert_array_equal(s.download(b)[0], g[f"stepn_{b}"])


def test_oracle_reads_the_overset_file_like_the_arrays(oracle_lib, tmp_path):
    case = overset_case("cylinder2d_64")
    path = str(tmp_path / "overset.bin")
    case.overset.write(path)
    a = api.Solver(oracle_lib, case).get_overset()
    b = api.Solver(oracle_lib, case, overset_file=path).get_overset()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_oracle_overset_matches_reference_live(oracle_lib):
    """A second overset layout run live on two reference ranks: a finer O-grid, a wider seam
    overlap and three fringe layers."""
    from oracle import run_ref
    if not run_ref.available():
        pytest.skip("oracle/_ref/camille_ref not built here")
    case = cases.cylinder2d(nb=56, length=14.0, ntheta=80, nr=20, r_out=3.2, first_cell=0.04, r_cut=0.9,
                            seam_overlap=10.5, fringe=3, sponge=5, nsteps=12, pulse=(-1.5, -0.4, 1e-3, 0.4))
    s = api.Solver(oracle_lib, case)
    dt = s.compute_dt()
    assert dt == run_ref.run(case, mode="run", nsteps=1, dt=None, nprocs=2)["result"]["dt"]
    ref = run_ref.assemble(case, run_ref.run(case, mode="run", nsteps=case.nsteps, dt=dt, nprocs=2)["ranks"])
    s.advance(case.nsteps, dt)
    for b in range(2):
        np.testing.assert_array_equal(s.download(b)[0], ref[b])


def _transitions(iblank: np.ndarray, axis: int) -> set:
    """The hole-closure branches that occur along one axis of an (nz, ny, nx) iblank array, as the
    reference's per-line scan meets them (src/solver/spatial_discretization.cpp:1356-1652)."""
    BL, RC, FL = 1, -1, 0
    lines = np.moveaxis(iblank, axis, -1).reshape(-1, iblank.shape[axis])
    seen = set()
    for ln in lines:
        if ln[0] == BL:
            seen.add("hole at line start")
        if ln[-1] == BL:
            seen.add("hole at line end")
        for a, b in zip(ln[:-1], ln[1:]):
            if b == BL:
                seen.add({FL: "hole after fluid", RC: "hole after receiver", BL: "hole after hole"}[int(a)])
            elif a == BL:
                seen.add("fluid after hole" if b == FL else "receiver after hole")
    return seen


@pytest.mark.parametrize("name", ["holes2d", "holes3d"])
def test_hole_layouts_exercise_every_closure_branch(name):
    """The hand-set hole workloads meet every branch of the hole scan along every direction
    (the F8 branch, a hole after a plain fluid point, among them), on the iblank the reference
    itself built from the overset file."""
    g = load_golden(name)
    ib = np.rint(g["iblank_0"]).astype(int)
    nd = 3 if ib.shape[0] > 1 else 2
    want = {"hole after fluid", "hole after receiver", "hole after hole", "fluid after hole",
            "receiver after hole", "hole at line start", "hole at line end"}
    for axis in range(3 - nd, 3):
        assert _transitions(ib, axis) == want, (name, axis, want - _transitions(ib, axis))


# ---- passive scalars (PHYSICAL_MODEL = LEE_SCALAR) ------------------------------------------

SCALAR_NAMES = ["scalar2d_40x32", "scalar3d_14"]


def full_state(solver, b):
    """The 5 + n slots of block b: the LEE slots, then the passive scalars."""
    return np.concatenate([solver.download(b)[0], solver.download_scalars(b)])


@pytest.mark.parametrize("name", SCALAR_NAMES)
def test_oracle_scalars_match_golden(oracle_lib, name):
    """Two (2-D) and one (3-D) passive scalars through the slip wall, Neumann faces, sponges
    and the sheared mean: the LEE slots' setup and right-hand side are unchanged by them, the
    filter and every step match the reference on all 5 + n slots."""
    g = load_golden(name)
    case = golden_case(name)
    nd = case.num_dim
    s = api.Solver(oracle_lib, case)
    np.testing.assert_array_equal(s.get_setup(0, api.SETUP_MEAN_GRADIENT), g["mean_gradient"][:5 * nd])
    assert s.compute_dt() == float(g["dt"])
    np.testing.assert_array_equal(s.eval_rhs(0, 0.0), g["rhs"][:5])
    s.apply_filter()
    np.testing.assert_array_equal(full_state(s, 0), g["filter"])
    dt = float(g["dt"])
    s = api.Solver(oracle_lib, case)
    s.advance(1, dt)
    np.testing.assert_array_equal(full_state(s, 0), g["step1"])
    s.advance(int(g["nsteps"]) - 1, dt)
    np.testing.assert_array_equal(full_state(s, 0), g["stepn"])


def test_oracle_scalars_through_overset_match_golden(oracle_lib):
    name = "scalar_cylinder2d_64"
    g = load_golden(name)
    case = overset_case(name)
    s = api.Solver(oracle_lib, case)
    check_overset_maps(s, g, case)
    dt = float(g["dt"])
    assert s.compute_dt() == dt
    s.advance(1, dt)
    for b in range(len(case.blocks)):
        np.testing.assert_array_equal(full_state(s, b), g[f"step1_{b}"])
    s.advance(int(g["nsteps"]) - 1, dt)
    for b in range(len(case.blocks)):
        np.testing.assert_array_equal(full_state(s, b), g[f"stepn_{b}"])


def test_scalars_are_set_before_the_blocks(oracle_lib):
    """lee_set_scalars after lee_set_block is refused (the slots are laid out with the block)."""
    case = golden_case("pulse2d_48")
    s = api.Solver(oracle_lib, case, prepare=False)
    with pytest.raises(api.LeeError, match="before lee_set_block"):
        s._chk(oracle_lib.set_scalars(s.ctx, 2))
