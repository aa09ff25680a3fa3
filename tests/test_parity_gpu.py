"""Parity of the CUDA path with the camille reference (golden fixtures made by running
the compiled reference) and with the CPU oracle at larger sizes.

Tolerances (relative L2 over all state variables): FP64 within 1e-12 after one step
and within 1e-10 after N steps; operator-level FP64 results within 1e-12; setup
products within 1e-13. The FP32-compensated form is held to 1e-5 relative L2 in p'
against the FP64 reference.
"""
from __future__ import annotations

import numpy as np
import pytest

from camille_b200 import api, cases
from tests.conftest import golden_case, load_golden

pytestmark = pytest.mark.gpu
NAMES = ["pulse2d_48", "curvi3d_16", "shear2d_40x32", "wall3d_14", "waves2d_40x32", "jet3d_14", "axisym2d_48x32"]


def rl2(a, b):
    return api.rel_l2(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("name", NAMES)
def test_setup_products(product_lib, name):
    g = load_golden(name)
    s = api.Solver(product_lib, golden_case(name))
    assert rl2(s.get_setup(0, api.SETUP_METRICS), g["metrics"]) <= 1e-14
    assert rl2(s.get_setup(0, api.SETUP_JACOBIAN)[0], g["jacobian"]) <= 1e-14
    mg = s.get_setup(0, api.SETUP_MEAN_GRADIENT)
    scale = max(1.0, float(np.abs(g["mean_gradient"]).max()))
    assert float(np.abs(mg - g["mean_gradient"]).max()) <= 1e-13 * scale
    sp = s.get_setup(0, api.SETUP_SPONGE)[0]
    assert float(np.abs(sp - g["sponge"]).max()) <= 1e-13 * max(1.0, float(g["sponge"].max()))
    dt = s.compute_dt()
    assert abs(dt - float(g["dt"])) <= 1e-14 * float(g["dt"])


@pytest.mark.parametrize("name", NAMES)
def test_rhs_and_filter(product_lib, name):
    g = load_golden(name)
    s = api.Solver(product_lib, golden_case(name))
    assert rl2(s.eval_rhs(0, 0.0), g["rhs"]) <= 1e-12
    s.apply_filter()
    assert rl2(s.download(0)[0], g["filter"]) <= 1e-13


@pytest.mark.parametrize("name", NAMES)
def test_fp64_steps(product_lib, name):
    g = load_golden(name)
    dt = float(g["dt"])
    s = api.Solver(product_lib, golden_case(name))
    s.advance(1, dt)
    y, step, t = s.download(0)
    assert step == 1 and t == dt
    assert rl2(y, g["step1"]) <= 1e-12
    s.advance(int(g["nsteps"]) - 1, dt)
    assert rl2(s.download(0)[0], g["stepn"]) <= 1e-10


@pytest.mark.parametrize("name", NAMES)
def test_fp32_compensated_steps(product_lib, name):
    g = load_golden(name)
    dt = float(g["dt"])
    s = api.Solver(product_lib, golden_case(name), precision=api.FP32_COMPENSATED)
    s.advance(int(g["nsteps"]), dt)
    y = s.download(0)[0]
    assert rl2(y[4], g["stepn"][4]) <= 1e-5


def _larger():
    a = cases.pulse2d(n=128, length=127 * 100.0 / 255.0, sponge=20, nsteps=60)
    b = cases.curvi3d(n=40, nsteps=12, halfwidth=3.0)
    c = cases.curvi3d(n=24, nsteps=6, halfwidth=2.0)
    c.fd_scheme, c.filter_scheme, c.filter_strength = "FDO11P", "SFO11P", 0.2
    d = cases.pulse2d(n=64, length=63 * 100.0 / 255.0, sponge=10, nsteps=10)
    d.rk, d.filter_order, d.filter_blend = "RUNGE_KUTTA2", 4, 0.6
    e = cases.shear2d(nx=130, ny=96, nsteps=40)
    f = cases.wall3d(n=40, nsteps=8, halfwidth=3.0)
    g = cases.waves2d(nx=96, ny=64, nsteps=40)
    h = cases.jet3d(n=40, nsteps=10)
    i = cases.waves2d(nx=64, ny=48, nsteps=20,
                      wave=cases.HarmonicWave("WAVE_ENTROPY", "WAVEFORM_HOMOGENEOUS", 2, 1e-3, 4.0))
    j = cases.axisym2d(nx=128, nr=80, nsteps=40)
    k = cases.jet2d_source(nx=160, ny=96, nsteps=40)
    return {"pulse2d_128": a, "curvi3d_40": b, "fdo11p_3d_24": c, "rk2_2d_64": d, "shear2d_130x96": e,
            "wall3d_40": f, "waves2d_96x64": g, "jet3d_40": h, "entropy2d_64x48": i, "axisym2d_128x80": j,
            "jet2d_source_160x96": k}


@pytest.mark.parametrize("label", list(_larger().keys()))
def test_fp64_matches_oracle(product_lib, oracle_lib, label):
    case = _larger()[label]
    o = api.Solver(oracle_lib, case)
    dt = o.compute_dt()
    p = api.Solver(product_lib, case)
    assert abs(p.compute_dt() - dt) <= 1e-14 * dt
    assert rl2(p.eval_rhs(0, 0.3), o.eval_rhs(0, 0.3)) <= 1e-12
    o.advance(1, dt)
    p.advance(1, dt)
    assert rl2(p.download(0)[0], o.download(0)[0]) <= 1e-12
    o.advance(case.nsteps - 1, dt)
    p.advance(case.nsteps - 1, dt)
    yo, so, to = o.download(0)
    yp, sp, tp = p.download(0)
    assert (so, to) == (sp, tp)
    assert rl2(yp, yo) <= 1e-10


@pytest.mark.parametrize("label", ["pulse2d_128", "curvi3d_40", "shear2d_130x96", "wall3d_40", "waves2d_96x64",
                                   "jet3d_40", "axisym2d_128x80"])
def test_fp32_compensated_error_vs_oracle(product_lib, oracle_lib, label):
    case = _larger()[label]
    o = api.Solver(oracle_lib, case)
    dt = o.compute_dt()
    o.advance(case.nsteps, dt)
    p = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    p.advance(case.nsteps, dt)
    err = rl2(p.download(0)[0][4], o.download(0)[0][4])
    assert err <= 1e-5, err


def _wide():
    a = cases.curvi3d(n=136, nsteps=1, halfwidth=6.0, sponge=8)
    b = cases.curvi3d(n=72, nsteps=1, halfwidth=4.0)
    b.fd_scheme, b.filter_scheme, b.filter_strength = "FDO11P", "SFO11P", 0.3
    c = cases.pulse2d(n=520, length=519 * 100.0 / 255.0, sponge=20, nsteps=1)
    d = cases.curvi3d(n=68, nsteps=1, halfwidth=4.0)
    d.filter_order, d.filter_blend = 4, 0.7
    return {"curvi3d_136": a, "sfo11p_3d_72": b, "pulse2d_520": c, "filter4_3d_68": d}


def _uniform_cases():
    a = cases.pulse2d(n=128, length=127 * 100.0 / 255.0, sponge=20, nsteps=40)
    a.monopole = (3.0, -2.0, 0.0, 1e-3, 0.5, 3.0, 20.0)
    b = cases.curvi3d(n=40, nsteps=12, halfwidth=3.0)
    c = cases.curvi3d(n=44, nsteps=10, halfwidth=3.0, sponge=4)
    c.monopole = (20.0, 22.0, 21.0, 1e-3, 0.7, 2.5, 0.0)
    c.rk = "RUNGE_KUTTA2"
    return {"pulse2d_128_monopole": a, "curvi3d_40": b, "curvi3d_44_sponge_monopole_rk2": c}


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("label", list(_uniform_cases().keys()))
def test_stage_kernels_fp32_compensated(product_lib, oracle_lib, label, kernel):
    """Both TMA stage kernels of the compensated form (one point per thread; two, in packed
    FP32): the right-hand side against the oracle within 1e-6, and the steps within 1e-5 in p'."""
    case = _uniform_cases()[label]
    o = api.Solver(oracle_lib, case)
    dt = o.compute_dt()
    p = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED, stage_kernel=kernel)
    assert p.info().stage_kernel == kernel
    assert rl2(p.eval_rhs(0, 0.7), o.eval_rhs(0, 0.7)) <= 1e-6
    o.advance(case.nsteps, dt)
    p.advance(case.nsteps, dt)
    err = rl2(p.download(0)[0][4], o.download(0)[0][4])
    assert err <= 1e-5, err


_ORACLE_FILTERED = {}


def _oracle_filtered(oracle_lib, label):
    if label not in _ORACLE_FILTERED:
        o = api.Solver(oracle_lib, _wide()[label])
        o.apply_filter()
        _ORACLE_FILTERED[label] = o.download(0)[0]
    return _ORACLE_FILTERED[label]


@pytest.mark.parametrize("kernel", [0, 2, 4])
@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
@pytest.mark.parametrize("label", list(_wide().keys()))
def test_filter_across_tiles(product_lib, oracle_lib, label, precision, kernel):
    """Blocks several filter tiles wide and tall (vector tiles of 32 groups along xi, 8 rows,
    chunks of planes), with the OA8, OA4 and SFO11P filters, on every fused-filter kernel (scalar;
    groups of 2 or 4 points): the fused filter against the oracle, FP64 within 1e-13 and the
    compensated form within 1e-6 (one FP32 rounding)."""
    if precision == api.FP64 and kernel == 4:
        pytest.skip("FP64 groups hold 2 points")
    case = _wide()[label]
    p = api.Solver(product_lib, case, precision=precision, filter_kernel=kernel)
    p.apply_filter()
    tol = 1e-13 if precision == api.FP64 else 1e-6
    assert rl2(p.download(0)[0], _oracle_filtered(oracle_lib, label)) <= tol


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
@pytest.mark.parametrize("label", ["curvi3d_136", "sfo11p_3d_72", "pulse2d_520", "filter4_3d_68"])
def test_filter_forms_same_bits(product_lib, oracle_lib, label, precision):
    """The forms of the scalar fused filter (one row per thread on 8-row tiles, two rows per
    thread on 16-row tiles, and for the compensated form on 3-D blocks two points per thread on
    64 x 8 tiles) do the same arithmetic per point: identical bits, within 1e-13 (FP64) or 1e-6
    (compensated) of the oracle, and the same bits again after two RK steps with each form."""
    case = _wide()[label]
    out, steps = [], []
    forms = (1, 2, 3) if precision == api.FP32_COMPENSATED and "3d" in label else (1, 2)
    for form in forms:
        p = api.Solver(product_lib, case, precision=precision, filter_kernel=0, filter_form=form)
        assert p.info().filter_rows == form
        p.apply_filter()
        out.append(p.download(0)[0])
        q = api.Solver(product_lib, case, precision=precision, filter_kernel=0, filter_form=form)
        dt = q.compute_dt()
        q.advance(2, dt)
        steps.append(q.download(0)[0])
    tol = 1e-13 if precision == api.FP64 else 1e-6
    assert rl2(out[0], _oracle_filtered(oracle_lib, label)) <= tol
    for q in range(1, len(forms)):
        np.testing.assert_array_equal(out[q], out[0])
        np.testing.assert_array_equal(steps[q], steps[0])


def test_filter_form_refusals(product_lib):
    """The two-row form takes no block with holes and not the vector kernel's groups; the
    two-point form takes only compensated 3-D blocks without holes."""
    with pytest.raises(api.LeeError, match="filter form"):
        api.Solver(product_lib, cases.curvi3d(n=40, nsteps=1, halfwidth=3.0), precision=api.FP64, filter_form=3)
    with pytest.raises(api.LeeError, match="filter form"):
        api.Solver(product_lib, cases.pulse2d(n=48, nsteps=1), precision=api.FP32_COMPENSATED, filter_form=3)
    with pytest.raises(api.LeeError, match="filter form"):
        api.Solver(product_lib, cases.holes(3, nsteps=1), precision=api.FP32_COMPENSATED, filter_form=3)
    with pytest.raises(api.LeeError, match="filter form"):
        api.Solver(product_lib, cases.holes(2, nsteps=1), filter_form=2)
    with pytest.raises(api.LeeError, match="filter form"):
        api.Solver(product_lib, cases.curvi3d(n=40, nsteps=1, halfwidth=3.0), precision=api.FP32_COMPENSATED,
                   filter_kernel=4, filter_form=2)


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_rho_ratio_follows_the_pre_filter_state(product_lib, oracle_lib, precision):
    """With a sheared mean the right-hand side reads rho'/rho_bar, which the reference
    recomputes after each boundary update and not after the filter: a right-hand side taken
    after a step, or after a filter call, sees the pre-filter state."""
    tol = 1e-12 if precision == api.FP64 else 1e-5
    case = cases.shear2d(nx=48, ny=40, nsteps=3)
    o = api.Solver(oracle_lib, case)
    p = api.Solver(product_lib, case, precision=precision)
    o.apply_filter()
    p.apply_filter()
    assert rl2(p.eval_rhs(0, 0.1), o.eval_rhs(0, 0.1)) <= tol
    dt = o.compute_dt()
    o.advance(case.nsteps, dt)
    p.advance(case.nsteps, dt)
    assert rl2(p.eval_rhs(0, 0.2), o.eval_rhs(0, 0.2)) <= tol


# ---- overset (two blocks, hole cut, fringes, O-grid seam) ---------------------------------

def _overset_golden(name):
    from tests.golden.make_golden import OVERSET_WORKLOADS
    return OVERSET_WORKLOADS[name]()


OVERSET_NAMES = ["cylinder2d_64", "holes2d", "holes3d"]


@pytest.mark.parametrize("name", OVERSET_NAMES)
def test_overset_maps_are_bit_exact(product_lib, name):
    """The receiver and donor indices and the normalised weights the GPU holds equal the
    reference's overset::receiverCells / donorCells, to the last bit."""
    g = load_golden(name)
    case = _overset_golden(name)
    m = api.Solver(product_lib, case).get_overset()
    for b in range(len(case.blocks)):
        sel = m["donor_block"] == b
        np.testing.assert_array_equal(m["donor_l0"][sel], g[f"donor_l0_{b}"])
        np.testing.assert_array_equal(m["weights"][sel], g[f"weights_{b}"])
        np.testing.assert_array_equal(m["recv_l0"][m["recv_block"] == b], g[f"recv_l0_{b}"])


@pytest.mark.parametrize("name", OVERSET_NAMES)
def test_overset_fp64_steps(product_lib, name):
    """holes2d / holes3d: a hole after fluid (no closure, the reference's `last_iblank /=
    BLANKED`), after a receiver (right closure), after a hole (zero), fluid and receivers after a
    hole (left closure), holes at line starts and ends, along every direction; through the
    TMA-staged kernels."""
    g = load_golden(name)
    case = _overset_golden(name)
    nb = len(case.blocks)
    s = api.Solver(product_lib, case)
    # the hole blocks run the TMA-staged kernels, their closure classes from the closure codes
    info = s.info()
    assert info.tma_stage == 1 and info.tma_filter == 1
    dt = float(g["dt"])
    assert abs(s.compute_dt() - dt) <= 1e-14 * dt
    for b in range(nb):
        assert rl2(s.eval_rhs(b, 0.0), g[f"rhs_{b}"]) <= 1e-12
    s.advance(1, dt)
    for b in range(nb):
        assert rl2(s.download(b)[0], g[f"step1_{b}"]) <= 1e-12
    s.advance(int(g["nsteps"]) - 1, dt)
    for b in range(nb):
        assert rl2(s.download(b)[0], g[f"stepn_{b}"]) <= 1e-10


@pytest.mark.parametrize("name", OVERSET_NAMES)
def test_overset_fp32_compensated_steps(product_lib, name):
    g = load_golden(name)
    case = _overset_golden(name)
    s = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    s.advance(int(g["nsteps"]), float(g["dt"]))
    for b in range(len(case.blocks)):
        assert rl2(s.download(b)[0][4], g[f"stepn_{b}"][4]) <= 1e-5


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_overset_larger_vs_oracle(product_lib, oracle_lib, precision, tmp_path):
    """A mid-size cylinder layout (read from its overset file by both sides) against the oracle."""
    case = cases.cylinder2d(nb=160, length=24.0, ntheta=128, nr=40, r_out=3.0, first_cell=0.02, r_cut=1.0,
                            sponge=8, nsteps=60, pulse=(1.6, -0.5, 1e-3, 0.4))
    path = str(tmp_path / "overset.bin")
    case.overset.write(path)
    o = api.Solver(oracle_lib, case, overset_file=path)
    p = api.Solver(product_lib, case, precision=precision, overset_file=path)
    dt = o.compute_dt()
    o.advance(case.nsteps, dt)
    p.advance(case.nsteps, dt)
    for b in range(2):
        yo, yp = o.download(b)[0], p.download(b)[0]
        if precision == api.FP64:
            assert rl2(yp, yo) <= 1e-10
        else:
            assert rl2(yp[4], yo[4]) <= 1e-5


# ---- replayed step graphs ----------------------------------------------------------------

def _graph_cases():
    return {
        "pulse2d": cases.pulse2d(n=96, length=95 * 100.0 / 255.0, sponge=10, nsteps=13),
        "curvi3d_fdo11p": (lambda c: (setattr(c, "fd_scheme", "FDO11P"), setattr(c, "filter_scheme", "SFO11P"),
                                      setattr(c, "filter_strength", 0.2), c)[-1])(cases.curvi3d(n=24, nsteps=7)),
        "shear2d_rk2": (lambda c: (setattr(c, "rk", "RUNGE_KUTTA2"), c)[-1])(cases.shear2d(nx=64, ny=40, nsteps=9)),
        "cylinder_nofilter": (lambda c: (setattr(c, "filter_scheme", "NONE"), c)[-1])(
            _overset_golden("cylinder2d_64")),
        "cylinder": _overset_golden("cylinder2d_64"),
        # stage and update times read from the graph's time table
        "waves2d": cases.waves2d(nx=64, ny=48, nsteps=11),
        "jet3d_rk2": (lambda c: (setattr(c, "rk", "RUNGE_KUTTA2"), c)[-1])(cases.jet3d(n=20, nsteps=7)),
        "axisym2d": cases.axisym2d(nx=64, nr=40, nsteps=9),
        "jet2d_source": cases.jet2d_source(nx=64, ny=48, nsteps=9),
    }


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
@pytest.mark.parametrize("label", list(_graph_cases().keys()))
def test_step_graphs_give_the_same_bits(product_lib, label, precision):
    """lee_advance replaying a captured step graph (with the monopole amplitudes read from a
    device table and buffer roles that rotate) gives the same bits as launching every
    kernel on its own, over step counts that leave a remainder."""
    case = _graph_cases()[label]
    a = api.Solver(product_lib, case, precision=precision)
    b = api.Solver(product_lib, case, precision=precision)
    b.set_graphs(False)
    dt = a.compute_dt()
    for n in (1, case.nsteps, 3):
        a.advance(n, dt)
        b.advance(n, dt)
    for blk in range(len(case.blocks)):
        ya, sa, ta = a.download(blk)
        yb, sb, tb = b.download(blk)
        assert (sa, ta) == (sb, tb)
        np.testing.assert_array_equal(ya, yb)


@pytest.mark.parametrize("args,code", [
    ((api.WAVE_ACOUSTIC, api.WAVEFORM_GAUSSIAN_ROUNDJET, 0, 0.1, 2.0, 1.0), api.LEE_ERR_ARG),
    ((api.WAVE_ENTROPY, api.WAVEFORM_PLANE, 0, 0.1, 2.0, 0.0), api.LEE_ERR_ARG),
    ((api.WAVE_ENTROPY, api.WAVEFORM_HOMOGENEOUS, 0, 1.5, 2.0, 0.0), api.LEE_ERR_ARG),
    ((api.WAVE_ENTROPY, api.WAVEFORM_HOMOGENEOUS, 3, 0.1, 2.0, 0.0), api.LEE_ERR_ARG),
    ((api.WAVE_ENTROPY, api.WAVEFORM_HOMOGENEOUS, 0, 0.1, 0.0, 0.0), api.LEE_ERR_ARG),
    ((api.WAVE_ENTROPY, api.WAVEFORM_GAUSSIAN_ROUNDJET, 0, 0.1, 2.0, 0.0), api.LEE_ERR_ARG),
    ((api.WAVE_ACOUSTIC, api.WAVEFORM_PLANE, 2, 0.1, 2.0, 0.0), api.LEE_ERR_UNSUPPORTED),
])
def test_harmonic_wave_arguments_are_checked(product_lib, args, code):
    """lee_set_harmonic_wave refuses what the reference has no formula for, the amplitude
    range of check_consistency_wave, and an acoustic wave along z in 2-D; a harmonic-wave
    line without a wave stops lee_prepare."""
    case = cases.waves2d(nx=24, ny=20, nsteps=1)
    case.harmonic_wave = None
    with pytest.raises(api.LeeError) as e:
        api.Solver(product_lib, case)
    assert e.value.code == api.LEE_ERR_STATE
    case.harmonic_wave = cases.HarmonicWave("WAVE_ENTROPY", "WAVEFORM_HOMOGENEOUS", 0, 0.1, 2.0)
    s = api.Solver(product_lib, case, upload=False, prepare=False)
    assert product_lib.set_harmonic_wave(s.ctx, *args) == code


def test_harmonic_sponge_blocks_run_the_generic_stage_kernel(product_lib):
    """A block with a harmonic-wave sponge zone runs the stage kernel with the zone loop (the
    TMA stage kernels read one summed strength field); the filter stays TMA-staged."""
    case = cases.waves2d(nx=64, ny=48, nsteps=1)
    s = api.Solver(product_lib, case)
    info = s.info()
    assert info.tma_stage == 0 and info.tma_filter == 1
    case.boundaries = [b for b in case.boundaries if b.kind != "sponge_freund_harmonicwave"]
    assert api.Solver(product_lib, case).info().tma_stage == 1


def test_axisymmetry_arguments_are_checked(product_lib):
    """check_consistency_dimension (src/core/input.cpp:519-535): 2-D and the x axis only."""
    s2 = api.Solver(product_lib, cases.axisym2d(nx=24, nr=16, nsteps=1), upload=False, prepare=False)
    assert product_lib.set_axisymmetric(s2.ctx, 1, 1) == api.LEE_ERR_ARG
    assert product_lib.set_axisymmetric(s2.ctx, 1, 0) == api.LEE_OK
    s3 = api.Solver(product_lib, cases.curvi3d(n=12, nsteps=1), upload=False, prepare=False)
    assert product_lib.set_axisymmetric(s3.ctx, 1, 0) == api.LEE_ERR_ARG
    assert product_lib.set_axisymmetric(s3.ctx, 0, 0) == api.LEE_OK


@pytest.mark.parametrize("label", ["curvi3d_40_sponge", "pulse2d_96", "curvi3d_36_rk2_monopole"])
def test_increment_step_gives_the_same_bits(product_lib, label):
    """The compensated step whose last stage writes the increment alone (the fused filter forms
    y_pre = y_n + increment and its rounding error) gives the bits of the step whose last stage
    writes y_pre and its error, over replayed step graphs and direct launches."""
    case = {
        "curvi3d_40_sponge": lambda: cases.curvi3d(n=40, nsteps=11, halfwidth=3.0, sponge=4),
        "pulse2d_96": lambda: cases.pulse2d(n=96, length=95 * 100.0 / 255.0, sponge=10, nsteps=11),
        "curvi3d_36_rk2_monopole": lambda: (lambda c: (setattr(c, "rk", "RUNGE_KUTTA2"),
                                                       setattr(c, "monopole", (17.0, 18.0, 16.0, 1e-3, 0.6, 2.5, 0.0)),
                                                       c)[-1])(cases.curvi3d(n=36, nsteps=11, halfwidth=3.0, sponge=4)),
    }[label]()
    # on before lee_prepare: the filter's autotuning then keeps the one-row form, which takes the
    # increment
    a = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED, prepare=False)
    assert product_lib.set_increment_step(a.ctx, 1) == api.LEE_OK
    a._chk(product_lib.prepare(a.ctx))
    a.upload(0, case.blocks[0].state)
    b = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    assert a.info().increment_step == 1 and b.info().increment_step == 0
    dt = a.compute_dt()
    for n in (1, case.nsteps, 3):
        a.advance(n, dt)
        b.advance(n, dt)
    ya, sa, ta = a.download(0)
    yb, sb, tb = b.download(0)
    assert (sa, ta) == (sb, tb)
    np.testing.assert_array_equal(ya, yb)
