"""Batches of independent 2-D instances (lee_advance_blocks and the batched kernels).

A context holding several Cartesian instances runs one launch per RK stage and one per filter
for the whole batch. Each instance is checked against itself run alone in its own single-block
context (the per-block kernels) and against the CPU oracle, in FP64 within 1e-12 / 1e-10
relative L2; the FP32-compensated batch against the FP64 one-at-a-time runs within 1e-5 in p';
replayed step graphs against direct launches, bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from camille_b200 import api, cases

pytestmark = pytest.mark.gpu


def _batch(nsteps=24):
    return cases.batch2d(count=6, nmin=40, nmax=96, spacing_spread=2.0, nsteps=nsteps, seed=9)


def _alone(lib, case, b, dt, nsteps, precision=api.FP64):
    s = api.Solver(lib, cases.instance(case, b), precision=precision)
    s.advance(nsteps, dt)
    y, step, t = s.download(0)
    s.close()
    return y, step, t


def test_block_time_steps_are_each_blocks_own(product_lib):
    case = _batch()
    s = api.Solver(product_lib, case)
    dts = s.compute_dt_blocks()
    for b in range(len(case.blocks)):
        alone = api.Solver(product_lib, cases.instance(case, b)).compute_dt()
        assert abs(dts[b] - alone) <= 1e-15 * alone
    assert np.unique(dts).size == len(case.blocks)


def test_fp64_batch_matches_each_instance_alone_and_the_oracle(product_lib, oracle_lib):
    case = _batch()
    s = api.Solver(product_lib, case)
    dts = s.compute_dt_blocks()
    s.advance_blocks(case.nsteps, dts)
    for b in range(len(case.blocks)):
        y, step, t = s.download(b)
        ya, stepa, ta = _alone(product_lib, case, b, dts[b], case.nsteps)
        assert step == stepa == case.nsteps and t == ta
        assert api.rel_l2(y, ya) <= 1e-12
        yo, _, _ = _alone(oracle_lib, case, b, dts[b], case.nsteps)
        assert api.rel_l2(y, yo) <= 1e-10


def test_fp32_compensated_batch_vs_fp64_alone(product_lib):
    case = _batch(nsteps=60)
    s = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    dts = s.compute_dt_blocks()
    s.advance_blocks(case.nsteps, dts)
    for b in range(len(case.blocks)):
        y = s.download(b)[0]
        ya = _alone(product_lib, case, b, dts[b], case.nsteps)[0]
        assert api.rel_l2(y[4], ya[4]) <= 1e-5


def test_full_size_batch_stays_finite_and_close(product_lib):
    """The 64-instance workload (5.2M points, the autotuned strip shapes) over 300 steps: the
    compensated batch stays within 1e-5 of the FP64 batch in p'."""
    case = cases.batch2d(nsteps=300)
    a = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    b = api.Solver(product_lib, case, precision=api.FP64)
    assert a.info().batched and b.info().batched
    dts = b.compute_dt_blocks()
    a.advance_blocks(case.nsteps, dts)
    b.advance_blocks(case.nsteps, dts)
    for q in range(0, len(case.blocks), 7):
        ya, yb = a.download(q)[0], b.download(q)[0]
        assert np.isfinite(ya).all()
        assert api.rel_l2(ya[4], yb[4]) <= 1e-5


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_batch_graphs_give_the_same_bits(product_lib, precision):
    case = _batch()
    a = api.Solver(product_lib, case, precision=precision)
    b = api.Solver(product_lib, case, precision=precision)
    b.set_graphs(False)
    dts = a.compute_dt_blocks()
    for n in (1, 7, 3):
        a.advance_blocks(n, dts)
        b.advance_blocks(n, dts)
    for q in range(len(case.blocks)):
        np.testing.assert_array_equal(a.download(q)[0], b.download(q)[0])


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_every_work_item_shape_gives_the_same_bits(product_lib, precision):
    """The strip shapes the autotuner picks from (one or two columns per stage thread, one
    field per filter CTA) change the launch, not the arithmetic of any point."""
    case = _batch(nsteps=5)
    ref = None
    for shape in range(7):
        s = api.Solver(product_lib, case, precision=precision)
        assert product_lib.set_batch_shapes(s.ctx, shape, (shape + 3) % 7) == api.LEE_OK
        dts = s.compute_dt_blocks()
        s.advance_blocks(case.nsteps, dts)
        out = [s.download(b)[0] for b in range(len(case.blocks))]
        s.close()
        if ref is None:
            ref = out
        for a, b in zip(out, ref):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_block_streams_give_the_same_bits(product_lib, precision):
    """Blocks on side streams (the default for several blocks: the two-block overset layout with
    its slip wall, sponges and overset gathers between stages) and on one stream give the same
    bits, replayed in step graphs or launched directly."""
    from tests.golden.make_golden import OVERSET_WORKLOADS
    case = OVERSET_WORKLOADS["cylinder2d_64"]()
    a = api.Solver(product_lib, case, precision=precision)
    b = api.Solver(product_lib, case, precision=precision)
    assert product_lib.set_block_streams(b.ctx, 0) == api.LEE_OK
    dt = a.compute_dt()
    for n in (1, 7, 2):
        a.advance(n, dt)
        b.advance(n, dt)
    for blk in range(2):
        np.testing.assert_array_equal(a.download(blk)[0], b.download(blk)[0])


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_batch_without_batched_kernels_matches_instances(product_lib, precision):
    """lee_set_batching(0): the instances run their own (TMA-staged) kernels side by side, each on
    its own clock; every instance matches the same instance run alone, bit for bit."""
    case = cases.batch2d(count=6, nmin=48, nmax=96, nsteps=9)
    s = api.Solver(product_lib, case, precision=precision, batching=False)
    assert s.info().batched == 0
    dts = s.compute_dt_blocks()
    s.advance_blocks(case.nsteps, dts)
    for b in range(len(case.blocks)):
        alone = api.Solver(product_lib, cases.instance(case, b), precision=precision)
        alone.advance(case.nsteps, float(dts[b]))
        np.testing.assert_array_equal(s.download(b)[0], alone.download(0)[0])


LEE_ERR_TIMEOUT = 8


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_persistent_step_gives_the_same_bits(product_lib, precision):
    """lee_set_batch_persistent: every RK stage and the filter of a batched step in one persistent
    launch (grid barriers between the phases) give the bits of the per-phase launches, for every
    shape it takes, with step graphs and with direct launches, in one launch per step."""
    case = _batch(nsteps=6)
    ref = api.Solver(product_lib, case, precision=precision)
    dts = ref.compute_dt_blocks()
    ref.advance_blocks(case.nsteps, dts)
    want = [ref.download(b)[0] for b in range(len(case.blocks))]
    for shape in range(5):
        for graphs in (True, False):
            s = api.Solver(product_lib, case, precision=precision)
            assert product_lib.set_batch_persistent(s.ctx, shape) == api.LEE_OK
            assert product_lib.set_finite_check(s.ctx, -1) == api.LEE_OK  # (its sentinel is a launch too)
            s.set_graphs(graphs)
            s.advance_blocks(case.nsteps, dts)
            if not graphs:
                assert s.stats().kernel_launches == case.nsteps
            for b in range(len(case.blocks)):
                np.testing.assert_array_equal(s.download(b)[0], want[b])
            s.close()


def test_persistent_step_refusals(product_lib):
    case = _batch(nsteps=1)
    s = api.Solver(product_lib, case)
    assert product_lib.set_batch_persistent(s.ctx, 5) == api.LEE_ERR_ARG  # two columns per stage thread
    assert product_lib.set_batch_persistent(s.ctx, -1) == api.LEE_OK
    one = api.Solver(product_lib, cases.curvi3d(n=16, nsteps=1, halfwidth=2.0))
    assert product_lib.set_batch_persistent(one.ctx, 0) == api.LEE_ERR_STATE  # not batched


@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_persistent_barrier_gives_up_and_the_context_recovers(product_lib, precision):
    """With a wait limit of 0 every grid barrier of the persistent step gives up at once: the call
    reports LEE_ERR_TIMEOUT (every CTA leaves the kernel, none waits), and with the default limit
    restored the same context steps on and matches a fresh context."""
    case = _batch(nsteps=3)
    s = api.Solver(product_lib, case, precision=precision)
    assert product_lib.set_batch_persistent(s.ctx, 0) == api.LEE_OK
    dts = s.compute_dt_blocks()
    s.advance_blocks(1, dts)
    assert product_lib.set_wait_limit(s.ctx, 0.0) == api.LEE_OK
    with pytest.raises(api.LeeError) as e:
        s.advance_blocks(2, dts)
    assert e.value.code == LEE_ERR_TIMEOUT
    assert product_lib.set_wait_limit(s.ctx, -1.0) == api.LEE_OK
    for b in range(len(case.blocks)):
        s.upload(b, case.blocks[b].state)
    s.advance_blocks(case.nsteps, dts)
    ref = api.Solver(product_lib, case, precision=precision)
    ref.advance_blocks(case.nsteps, dts)
    for b in range(len(case.blocks)):
        np.testing.assert_array_equal(s.download(b)[0], ref.download(b)[0])
