"""lee_filter_field_static, the filter entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc -- for instance a host framework that
owns the device memory through its own caching allocator, or a time loop that must not
allocate -- and filters one field that the caller already holds on the device, keeping
its intermediate passes in a scratch array compiled into the library. This test calls it
through the C ABI on device buffers owned by torch and checks its output against
lee_apply_filter (the context-based entry point) on two calls in a row, the second call
reusing the scratch the first one left behind, on a stream of its own, with neither torch's
memory pool nor the device's free memory changing across it. It runs last (file name) so that a
failure here cannot hide the other tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from camille_b200 import api, cases

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative L2, the filter tolerance of tests/test_parity_gpu.py


def _entry():
    dll = C.CDLL(api.PRODUCT_LIB)
    fn = dll.lee_filter_field_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    err = dll.lee_last_error
    err.restype = C.c_char_p
    err.argtypes = [C.c_void_p]
    return fn, err


def _case(label: str):
    if label == "2d":
        case = cases.pulse2d(n=96, length=95 * 100.0 / 255.0, sponge=0)
    else:
        case = cases.curvi3d(n=28, halfwidth=2.0)
    rng = np.random.default_rng(7)
    blk = case.blocks[0]
    blk.state = rng.standard_normal(blk.state.shape) * 1e-3
    if case.num_dim == 2:
        blk.state[3] = 0.0
    return case


def _context_filter(product_lib, case) -> np.ndarray:
    s = api.Solver(product_lib, case)
    s.apply_filter()
    out = s.download(0)[0]
    s.close()
    return out


@pytest.mark.parametrize("label", ["2d", "3d"])
def test_static_filter_matches_context_filter(product_lib, label):
    import torch

    fn, err = _entry()
    case = _case(label)
    ref = _context_filter(product_lib, case)
    blk = case.blocks[0]
    nx, ny, nz = blk.dims
    cfg = api.config_for(case)
    variables = [0, 1, 2, 4] if case.num_dim == 2 else [0, 1, 2, 3, 4]
    side = torch.cuda.Stream()
    # two calls in a row on the shared scratch: the first on torch's current stream, the second on
    # a stream of its own; around the second (the library's kernels and its scratch are loaded by
    # then) neither torch's pool nor the device's free memory may change
    for call, v in enumerate(variables[:2]):
        d_in = torch.from_numpy(np.ascontiguousarray(blk.state[v])).cuda()
        d_out = torch.full_like(d_in, float("nan"))
        strm = torch.cuda.current_stream() if call == 0 else side
        torch.cuda.synchronize()
        reserved, (free, _) = torch.cuda.memory_reserved(), torch.cuda.mem_get_info()
        rc = fn(case.num_dim, cfg.filter_scheme, cfg.filter_order, cfg.filter_strength, cfg.filter_blend,
                nx, ny, nz, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), C.c_void_p(strm.cuda_stream))
        assert rc == 0, err(None).decode()
        strm.synchronize()
        if call == 1:
            assert torch.cuda.memory_reserved() == reserved
            assert torch.cuda.mem_get_info()[0] == free
        got = d_out.cpu().numpy()
        rel = api.rel_l2(got, ref[v])
        assert rel <= TOL, f"call {call}: relative L2 {rel:.3e}"


def test_static_filter_refuses_oversized_fields(product_lib):
    fn, err = _entry()
    case = cases.curvi3d(n=12)
    cfg = api.config_for(case)
    rc = fn(3, cfg.filter_scheme, cfg.filter_order, cfg.filter_strength, cfg.filter_blend,
            128, 128, 65, C.c_void_p(1), C.c_void_p(2), None)
    assert rc == 1  # LEE_ERR_ARG
    assert "exceed the static scratch" in err(None).decode()
