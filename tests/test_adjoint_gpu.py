"""The discrete adjoint (lee_apply_adjoint, lee_adjoint_gradient) on the GPU.

- Dot-product test: <l, M^N x> = <(M^T)^N l, x> for seeded x and l, M the source-free step
  map of lee_advance, within 1e-12 relative in FP64, over several operator combinations.
- The distributed source's forward steps agree with the CPU oracle (FP64, 1e-10).
- Gradient: J(a) is quadratic in the lattice amplitudes a, so (J(a + d) - J(a - d)) / 2 equals
  grad . d up to rounding; checked on 32 seed-drawn directions (central differences of GPU FP64
  objectives), and against the tangent-linear derivative from FP64 oracle objectives,
  J(a + d) - J(a) - J(d) (the forward map is affine in a with zero initial state).
- Checkpoint recomputation replays the microphone traces bit for bit; the FP32-compensated
  gradient agrees with the FP64 one.
- A torch.autograd.Function wrapper (the check harness only) passes gradcheck.
"""
from __future__ import annotations

import copy

import numpy as np
import pytest

from camille_b200 import api, cases

pytestmark = pytest.mark.gpu


def _fields(case, rng):
    out = []
    for blk in case.blocks:
        f = rng.standard_normal(blk.state.shape)
        if case.num_dim == 2:
            f[3] = 0.0
        out.append(f)
    return out


def _dot(a, b, num_dim):
    vs = [0, 1, 2, 4] if num_dim == 2 else [0, 1, 2, 3, 4]
    return float(sum(np.vdot(a[v], b[v]) for v in vs))


def _dot_cases():
    a = cases.adjoint3d(n=24, lattice=5, nmics=12)
    a.distributed = None
    a.microphones = None
    b = cases.pulse2d(n=64, length=63 * 100.0 / 255.0, sponge=10)
    c = cases.pulse2d(n=64, length=63 * 100.0 / 255.0, sponge=0)
    c.fd_scheme, c.filter_scheme, c.filter_strength, c.rk = "FDO11P", "SFO11P", 0.3, "RUNGE_KUTTA2"
    d = cases.curvi3d(n=24, mach=0.3, sponge=4)
    d.filter_order, d.filter_blend = 4, 0.6
    e = cases.curvi3d(n=24, mach=0.4, sponge=0)
    e.filter_scheme = "NONE"
    return {"curvi3d_sponge": a, "pulse2d_sponge": b, "fdo11p_sfo11p_rk2_2d": c, "filter4_blend_3d": d,
            "nofilter_3d": e}


@pytest.mark.parametrize("nsteps", [1, 5])
@pytest.mark.parametrize("label", list(_dot_cases().keys()))
def test_dot_product(product_lib, label, nsteps):
    case = _dot_cases()[label]
    rng = np.random.default_rng(11)
    x = _fields(case, rng)[0]
    lam = _fields(case, rng)[0]
    s = api.Solver(product_lib, case, upload=False)
    dt = s.compute_dt()
    s.upload(0, x)
    s.advance(nsteps, dt)
    mx = s.download(0)[0]
    s.upload(0, lam)
    s.apply_adjoint(nsteps, dt)
    mtl = s.download(0)[0]
    lhs, rhs = _dot(lam, mx, case.num_dim), _dot(mtl, x, case.num_dim)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def _grad_case(n=24, lattice=5, nsteps=40):
    return cases.adjoint3d(n=n, lattice=lattice, nmics=12, nsteps=nsteps)


def _with_amps(case, amps):
    c = copy.deepcopy(case)
    c.distributed.amplitudes = amps
    return c


def test_distributed_source_forward_matches_oracle(product_lib, oracle_lib):
    case = _grad_case()
    o = api.Solver(oracle_lib, case)
    p = api.Solver(product_lib, case)
    dt = o.compute_dt()
    Jo = o.eval_objective(case.nsteps, dt)
    Jp = p.eval_objective(case.nsteps, dt)
    assert api.rel_l2(p.download(0)[0], o.download(0)[0]) <= 1e-10
    assert abs(Jp - Jo) <= 1e-10 * Jo


def test_gradient_central_differences_and_tangent_linear(product_lib, oracle_lib):
    case = _grad_case()
    a0 = case.distributed.amplitudes
    s = api.Solver(product_lib, case)
    dt = s.compute_dt()
    J, g, mism = s.adjoint_gradient(case.nsteps, dt, checkpoint_every=7, recompute=True)
    assert mism == 0
    # J from the gradient call equals a plain forward evaluation
    assert abs(J - api.Solver(product_lib, case).eval_objective(case.nsteps, dt)) <= 1e-13 * J
    rng = np.random.default_rng(32)
    worst = 0.0
    for _ in range(32):
        d = rng.standard_normal(a0.shape) * 1e-3
        jp = api.Solver(product_lib, _with_amps(case, a0 + d)).eval_objective(case.nsteps, dt)
        jm = api.Solver(product_lib, _with_amps(case, a0 - d)).eval_objective(case.nsteps, dt)
        fd = 0.5 * (jp - jm)
        ad = float(np.vdot(g, d))
        worst = max(worst, abs(fd - ad) / max(abs(fd), 1e-300))
    assert worst <= 1e-8, worst
    # tangent-linear derivative along two directions from FP64 oracle objectives
    for _ in range(2):
        d = rng.standard_normal(a0.shape) * 1e-3
        Ja = api.Solver(oracle_lib, case).eval_objective(case.nsteps, dt)
        Jd = api.Solver(oracle_lib, _with_amps(case, d)).eval_objective(case.nsteps, dt)
        Jad = api.Solver(oracle_lib, _with_amps(case, a0 + d)).eval_objective(case.nsteps, dt)
        tl = Jad - Ja - Jd  # = 2 w sum p(a) p(d), the derivative along d
        ad = float(np.vdot(g, d))
        assert abs(tl - ad) <= 1e-8 * abs(tl), (tl, ad)


def test_objective_then_gradient_on_one_context(product_lib):
    """A context that evaluated the objective (and captured its step graph) gives the same J
    from its gradient call, and the recomputed segments replay their traces bit for bit."""
    case = _grad_case(nsteps=36)
    s = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    dt = s.compute_dt()
    s.advance(3, dt)
    s.upload(0, case.blocks[0].state)
    J0 = s.eval_objective(case.nsteps, dt)
    s.upload(0, case.blocks[0].state)
    J, g, mism = s.adjoint_gradient(case.nsteps, dt, checkpoint_every=8, recompute=True)
    assert mism == 0 and J == J0
    s.upload(0, case.blocks[0].state)
    J2, g2, _ = s.adjoint_gradient(case.nsteps, dt, checkpoint_every=8, recompute=False)
    assert J2 == J0
    np.testing.assert_array_equal(g, g2)


def test_recompute_replays_and_precisions_agree(product_lib):
    case = _grad_case(nsteps=30)
    s64 = api.Solver(product_lib, case)
    dt = s64.compute_dt()
    J64, g64, m64 = s64.adjoint_gradient(case.nsteps, dt, checkpoint_every=10, recompute=True)
    s64b = api.Solver(product_lib, case)
    J64b, g64b, _ = s64b.adjoint_gradient(case.nsteps, dt, checkpoint_every=10, recompute=False)
    assert m64 == 0 and J64 == J64b
    np.testing.assert_array_equal(g64, g64b)
    s32 = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    J32, g32, m32 = s32.adjoint_gradient(case.nsteps, dt, checkpoint_every=10, recompute=True)
    assert m32 == 0
    assert abs(J32 - J64) <= 1e-5 * J64
    assert api.rel_l2(g32, g64) <= 1e-4


def test_two_point_filter_forms_give_the_same_gradient(product_lib):
    """With the forward filter in its two-point form the transposed filter of the reverse sweep
    runs the two-point kernel too (plain form, the transposed rows as its classes): its gradient
    agrees with the one-row form's to FP32 rounding, with the same objective (the forward filter's
    bits are the same in both forms) and bit-identical recomputed traces."""
    case = _grad_case(n=32, nsteps=24)
    out = {}
    for form in (1, 3):
        s = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED, filter_form=form)
        assert s.info().filter_rows == form
        dt = s.compute_dt()
        out[form] = s.adjoint_gradient(case.nsteps, dt, checkpoint_every=8, recompute=True)
    (J1, g1, m1), (J3, g3, m3) = out[1], out[3]
    assert m1 == 0 and m3 == 0
    assert J3 == J1
    assert api.rel_l2(g3, g1) <= 1e-6


def test_autograd_function_gradcheck(product_lib):
    import torch

    from tests.lee_autograd import LeeObjective

    case = _grad_case(lattice=3, nsteps=12)
    solver_dt = api.Solver(product_lib, case).compute_dt()
    a = torch.tensor(case.distributed.amplitudes, dtype=torch.float64, requires_grad=True)
    fn = lambda amps: LeeObjective.apply(amps, product_lib, case, solver_dt)  # noqa: E731
    assert torch.autograd.gradcheck(fn, (a,), eps=1e-4, atol=1e-12, rtol=1e-6)
