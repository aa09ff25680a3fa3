"""Failure detection without a GPU fault.

- The non-finite sentinel (lee_set_finite_check): a NaN uploaded from the host ends lee_advance
  with LEE_ERR_NONFINITE, at the end of the call by default or after the first chunk of the
  chosen interval; the context stays usable.
- The bounded waits of the TMA-staged kernels (lee_set_wait_limit): with a limit of 0 every wait
  gives up at once, the CTA drains its copies in flight and returns, and lee_advance reports
  LEE_ERR_TIMEOUT; with the default limit restored the same
  context advances again and gives the bits of a fresh context.

Nothing here faults, traps or hangs a GPU: the NaN is data, and every wait that gives up is
followed by waits (with the default one-second limit) that end when the copies land.
"""
from __future__ import annotations

import numpy as np
import pytest

from camille_b200 import api, cases

LEE_ERR_NONFINITE, LEE_ERR_TIMEOUT = 6, 8


def _nan_state(case):
    y = case.blocks[0].state.copy()
    y[4].flat[y[4].size // 2 + 7] = np.nan
    return y


def _case():
    return cases.curvi3d(n=40, nsteps=4, halfwidth=3.0, sponge=4)


@pytest.mark.parametrize("lib_name", ["oracle", pytest.param("product", marks=pytest.mark.gpu)])
def test_nonfinite_state_is_reported(lib_name, request):
    lib = request.getfixturevalue("oracle_lib" if lib_name == "oracle" else "product_lib")
    case = cases.curvi3d(n=20, nsteps=3, halfwidth=2.0)
    s = api.Solver(lib, case)
    dt = s.compute_dt()
    s.upload(0, _nan_state(case))
    with pytest.raises(api.LeeError) as e:
        s.advance(3, dt)
    assert e.value.code == LEE_ERR_NONFINITE
    assert not np.all(np.isfinite(s.download(0)[0]))
    # the context stays usable: a finite state advances
    s.upload(0, case.blocks[0].state)
    s.advance(3, dt)
    assert np.all(np.isfinite(s.download(0)[0]))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_nonfinite_check_interval_ends_the_call_early(product_lib, precision):
    case = _case()
    s = api.Solver(product_lib, case, precision=precision)
    dt = s.compute_dt()
    assert product_lib.set_finite_check(s.ctx, 2) == api.LEE_OK
    s.upload(0, _nan_state(case))
    with pytest.raises(api.LeeError) as e:
        s.advance(10, dt)
    assert e.value.code == LEE_ERR_NONFINITE
    assert s.download(0)[1] == 2  # stopped after the first chunk of two steps
    # with the sentinel off the call runs to its end
    assert product_lib.set_finite_check(s.ctx, -1) == api.LEE_OK
    s.upload(0, _nan_state(case))
    s.advance(4, dt)
    assert s.download(0)[1] == 4


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [api.FP64, api.FP32_COMPENSATED])
def test_wait_limit_zero_reports_timeout_and_the_context_recovers(product_lib, precision):
    case = _case()
    s = api.Solver(product_lib, case, precision=precision)
    assert s.info().tma_stage == 1 and s.info().tma_filter == 1
    dt = s.compute_dt()
    s.advance(2, dt)  # captures the step graph with the default limit
    assert product_lib.set_wait_limit(s.ctx, 0.0) == api.LEE_OK
    with pytest.raises(api.LeeError) as e:
        s.advance(2, dt)
    assert e.value.code == LEE_ERR_TIMEOUT
    assert product_lib.set_wait_limit(s.ctx, -1.0) == api.LEE_OK
    s.upload(0, case.blocks[0].state)
    s.advance(3, dt)
    ref = api.Solver(product_lib, case, precision=precision)
    ref.advance(3, dt)
    np.testing.assert_array_equal(s.download(0)[0], ref.download(0)[0])


@pytest.mark.gpu
def test_wait_limit_arguments(product_lib):
    s = api.Solver(product_lib, cases.curvi3d(n=12, nsteps=1), upload=False, prepare=False)
    assert product_lib.set_wait_limit(s.ctx, 11.0) == api.LEE_ERR_ARG
    assert product_lib.set_wait_limit(s.ctx, float("nan")) == api.LEE_ERR_ARG
    assert product_lib.set_finite_check(s.ctx, -2) == api.LEE_ERR_ARG
