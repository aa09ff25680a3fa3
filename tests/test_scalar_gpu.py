"""Passive scalars (PHYSICAL_MODEL = LEE_SCALAR) on the GPU against the compiled reference's
golden fixtures (tests/golden/make_golden.py: scalar2d_40x32, scalar3d_14, scalar_cylinder2d_64)
and the CPU oracle.

Tolerances as for the LEE slots: FP64 within 1e-12 relative L2 after one step and 1e-10 after
N steps (all 5 + n slots); the filter within 1e-13; FP32-compensated within 1e-5 relative L2
in p' and in every scalar against the reference.
"""
from __future__ import annotations

import numpy as np
import pytest

from camille_b200 import api, cases
from tests.conftest import golden_case, load_golden
from tests.test_oracle_pin import full_state, overset_case

pytestmark = pytest.mark.gpu
SINGLE = ["scalar2d_40x32", "scalar3d_14"]


def rl2(a, b):
    return api.rel_l2(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("name", SINGLE)
def test_fp64_steps_and_filter(product_lib, name):
    g = load_golden(name)
    case = golden_case(name)
    dt = float(g["dt"])
    s = api.Solver(product_lib, case)
    assert abs(s.compute_dt() - dt) <= 1e-14 * dt
    s.apply_filter()
    assert rl2(full_state(s, 0), g["filter"]) <= 1e-13
    s = api.Solver(product_lib, case)
    s.advance(1, dt)
    y1 = full_state(s, 0)
    assert rl2(y1, g["step1"]) <= 1e-12
    for k in range(case.num_scalars):
        assert rl2(y1[5 + k], g["step1"][5 + k]) <= 1e-12
    s.advance(int(g["nsteps"]) - 1, dt)
    yn = full_state(s, 0)
    assert rl2(yn, g["stepn"]) <= 1e-10
    for k in range(case.num_scalars):
        assert rl2(yn[5 + k], g["stepn"][5 + k]) <= 1e-10


@pytest.mark.parametrize("name", SINGLE)
def test_fp32_compensated_steps(product_lib, name):
    g = load_golden(name)
    case = golden_case(name)
    s = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    s.advance(int(g["nsteps"]), float(g["dt"]))
    y = full_state(s, 0)
    assert rl2(y[4], g["stepn"][4]) <= 1e-5
    for k in range(case.num_scalars):
        assert rl2(y[5 + k], g["stepn"][5 + k]) <= 1e-5


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_scalars_through_overset(product_lib, precision):
    name = "scalar_cylinder2d_64"
    g = load_golden(name)
    case = overset_case(name)
    dt = float(g["dt"])
    s = api.Solver(product_lib, case, precision=precision)
    s.advance(1, dt)
    for b in range(len(case.blocks)):
        y = full_state(s, b)
        if precision == api.FP64:
            assert rl2(y, g[f"step1_{b}"]) <= 1e-12
    s.advance(int(g["nsteps"]) - 1, dt)
    for b in range(len(case.blocks)):
        y = full_state(s, b)
        ref = g[f"stepn_{b}"]
        if precision == api.FP64:
            assert rl2(y, ref) <= 1e-10
        else:
            for v in [4] + [5 + k for k in range(case.num_scalars)]:
                assert rl2(y[v], ref[v]) <= 1e-5, (b, v, rl2(y[v], ref[v]))


def test_larger_block_matches_oracle(product_lib, oracle_lib):
    """Three scalars on a 3-D block of 32^3 (a sponge frame, the sheared wall) through the step
    graphs, FP64 against the oracle over 10 steps, and the replayed graphs give the same bits as
    direct launches."""
    case = cases.with_scalars(cases.wall3d(n=32, nsteps=10, halfwidth=3.0), n=3, seed=31)
    o = api.Solver(oracle_lib, case)
    p = api.Solver(product_lib, case)
    dt = o.compute_dt()
    o.advance(case.nsteps, dt)
    p.advance(case.nsteps, dt)
    assert rl2(full_state(p, 0), full_state(o, 0)) <= 1e-10
    q = api.Solver(product_lib, case)
    product_lib.set_graphs(q.ctx, 0)
    q.advance(case.nsteps, dt)
    np.testing.assert_array_equal(full_state(q, 0), full_state(p, 0))


def test_adjoint_refuses_scalars(product_lib):
    case = golden_case("scalar2d_40x32")
    s = api.Solver(product_lib, case)
    with pytest.raises(api.LeeError, match="scalars"):
        s.apply_adjoint(1, 1e-3)


@pytest.mark.parametrize("label", ["shear2d_rk2_nofilter", "holes2d", "holes3d"])
def test_variants_match_oracle(product_lib, oracle_lib, label):
    """Scalars with RK2 and no filter (the copies that stand in for the filter), and through the
    hand-set hole layouts (closure codes, self-donated receivers, the TMA kernels' hole paths):
    FP64 against the oracle over 6 steps within 1e-10, FP32-compensated within 1e-5."""
    if label == "shear2d_rk2_nofilter":
        base = cases.shear2d(nx=40, ny=32, nsteps=6)
        base.rk, base.filter_scheme = "RUNGE_KUTTA2", "NONE"
    else:
        base = cases.holes(2 if label == "holes2d" else 3, nsteps=6)
    case = cases.with_scalars(base, n=2, seed=41)
    o = api.Solver(oracle_lib, case)
    dt = o.compute_dt()
    o.advance(case.nsteps, dt)
    for prec, tol in ((api.FP64, 1e-10), (api.FP32_COMPENSATED, 1e-5)):
        p = api.Solver(product_lib, case, precision=prec)
        p.advance(case.nsteps, dt)
        for b in range(len(case.blocks)):
            yo, yp = full_state(o, b), full_state(p, b)
            if prec == api.FP64:
                assert rl2(yp, yo) <= tol, (b, rl2(yp, yo))
            else:
                for v in [4, 5, 6]:
                    assert rl2(yp[v], yo[v]) <= tol, (b, v, rl2(yp[v], yo[v]))
