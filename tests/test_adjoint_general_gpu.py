"""The general discrete adjoint on the GPU (lee_adjoint_gen.cu): every block of a context, holes
and their closure codes, BC lines (Neumann, slip wall, centerline, Dirichlet), harmonic-wave
sponges, overset interpolation (the receiver gather of camille src/overset/overset.cpp:886-974,
transposed), non-uniform mean flow with its rho' term, and the axisymmetric term.

- Dot-product test of the step map's linear part, <lam, S^N(x) - S^N(0)> = <(S^T)^N lam, x>, in
  FP64 within 1e-12 relative (the affine part -- monopoles, harmonic waves -- drops out of the
  difference), on the golden workloads that carry these features, the overset cylinder layout
  among them.
- The FP32 transposed map agrees with the FP64 one.
- Gradient on the overset cylinder layout (distributed source on the background, microphones on
  the O-grid): central differences of FP64 objectives (exact for the quadratic objective),
  checkpoint recomputation replaying the traces bit for bit (rho'/rho_bar restored with them).
"""
from __future__ import annotations

import copy

import numpy as np
import pytest

from camille_b200 import api, cases
from tests.conftest import golden_case

pytestmark = pytest.mark.gpu

DOT_CASES = ["shear2d_40x32", "wall3d_14", "waves2d_40x32", "jet3d_14", "axisym2d_48x32", "cylinder2d_64",
             "holes2d", "holes3d", "curvi3d_16", "holes2d_rk2_nofilter", "cylinder2d_64_filter4_blend"]


def _dot_case(name):
    """A golden workload, or one of two variants: the 2-D hole layout with RK2 and no filter (the
    hole mask then acts alone), and the cylinder with the 4th-order filter blended at 0.6."""
    if name == "holes2d_rk2_nofilter":
        case = golden_case("holes2d")
        case.rk, case.filter_scheme = "RUNGE_KUTTA2", "NONE"
        return case
    if name == "cylinder2d_64_filter4_blend":
        case = golden_case("cylinder2d_64")
        case.filter_order, case.filter_blend = 4, 0.6
        return case
    return golden_case(name)


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
    return float(sum(np.vdot(x[v], y[v]) for x, y in zip(a, b) for v in vs))


def _run(s, case, fields, nsteps, dt):
    for b, f in enumerate(fields):
        s.upload(b, f)
    s.advance(nsteps, dt)
    return [s.download(b)[0] for b in range(len(case.blocks))]


def _adjoint(s, case, lam, nsteps, dt):
    for b, f in enumerate(lam):
        s.upload(b, f)
    s.apply_adjoint(nsteps, dt)
    return [s.download(b)[0] for b in range(len(case.blocks))]


@pytest.mark.parametrize("nsteps", [1, 4])
@pytest.mark.parametrize("name", DOT_CASES)
def test_dot_product(product_lib, name, nsteps):
    case = _dot_case(name)
    rng = np.random.default_rng(17)
    x = _fields(case, rng)
    lam = _fields(case, rng)
    zero = [np.zeros_like(f) for f in x]
    s = api.Solver(product_lib, case, upload=False)
    dt = s.compute_dt()
    sx = _run(s, case, x, nsteps, dt)
    s0 = _run(s, case, zero, nsteps, dt)
    mx = [a - b for a, b in zip(sx, s0)]
    mtl = _adjoint(s, case, lam, nsteps, dt)
    lhs, rhs = _dot(lam, mx, case.num_dim), _dot(mtl, x, case.num_dim)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs, abs(lhs - rhs) / abs(lhs))


def test_fp32_transpose_agrees_with_fp64(product_lib):
    case = golden_case("cylinder2d_64")
    rng = np.random.default_rng(5)
    lam = _fields(case, rng)
    out = {}
    for prec in (api.FP64, api.FP32_COMPENSATED):
        s = api.Solver(product_lib, case, precision=prec, upload=False)
        dt = s.compute_dt()
        out[prec] = _adjoint(s, case, lam, 3, dt)
    for a, b in zip(out[api.FP64], out[api.FP32_COMPENSATED]):
        assert api.rel_l2(b, a) <= 1e-5


def _cylinder_gradient_case(nsteps=120):
    """The cylinder layout from rest (J is then a quadratic form in the amplitudes, so central
    differences are exact up to rounding) with a 4 x 4 lattice source on the background just
    left of the O-grid, and microphones on an O-grid ring that its waves reach within the run."""
    case = copy.deepcopy(golden_case("cylinder2d_64"))
    case.nsteps = nsteps
    case.monopole = None
    for blk in case.blocks:
        blk.state = np.zeros_like(blk.state)
    rng = np.random.default_rng(9)
    amps = rng.normal(0.0, 1e-3, size=(1, 4, 4))
    case.distributed = cases.DistributedSource(0, 0.8 * np.pi, (18.0, 28.0, 0.0), (2.0, 2.0, 1.0), amps)
    nx = case.blocks[1].dims[0]
    ii = np.arange(4, nx - 4, 5)
    case.microphones = cases.Microphones(1, (ii + nx * 8).astype(np.int64), 0.05)
    return case


def _with_amps(case, amps):
    c = copy.deepcopy(case)
    c.distributed.amplitudes = amps
    return c


def test_overset_gradient_central_differences(product_lib):
    case = _cylinder_gradient_case()
    a0 = case.distributed.amplitudes
    s = api.Solver(product_lib, case)
    dt = s.compute_dt()
    J, g, mism = s.adjoint_gradient(case.nsteps, dt, checkpoint_every=25, recompute=True)
    assert mism == 0
    assert abs(J - api.Solver(product_lib, case).eval_objective(case.nsteps, dt)) <= 1e-13 * J
    s2 = api.Solver(product_lib, case)
    J2, g2, _ = s2.adjoint_gradient(case.nsteps, dt, checkpoint_every=25, recompute=False)
    assert J2 == J
    np.testing.assert_array_equal(g, g2)
    assert np.linalg.norm(g) > 0.0
    rng = np.random.default_rng(33)
    worst = 0.0
    for _ in range(6):
        d = rng.standard_normal(a0.shape) * 1e-3
        jp = api.Solver(product_lib, _with_amps(case, a0 + d)).eval_objective(case.nsteps, dt)
        jm = api.Solver(product_lib, _with_amps(case, a0 - d)).eval_objective(case.nsteps, dt)
        fd = 0.5 * (jp - jm)
        ad = float(np.vdot(g, d))
        worst = max(worst, abs(fd - ad) / max(abs(fd), 1e-300))
    assert worst <= 1e-8, worst
