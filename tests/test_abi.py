"""The C ABI: every function declared in include/lee_b200.h is exported by the CUDA
library (and, under the orc_ prefix, by the CPU oracle), and the library refuses to
run without a GPU instead of falling back to the CPU."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

from camille_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions() -> list[str]:
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^[A-Za-z_][\w \*]*?\b(lee_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_header_declares_the_abi():
    names = declared_functions()
    for n in ("lee_create", "lee_destroy", "lee_last_error", "lee_set_block", "lee_set_mean",
              "lee_add_boundary", "lee_prepare", "lee_upload_state", "lee_download_state",
              "lee_compute_dt", "lee_advance", "lee_eval_rhs", "lee_apply_filter", "lee_get_setup"):
        assert n in names


def test_product_exports_every_declared_symbol(product_lib):
    dll = C.CDLL(api.PRODUCT_LIB)
    missing = [n for n in declared_functions() if not hasattr(dll, n)]
    assert not missing, missing


# Entry points that take device pointers: the CPU oracle and the context-based Solver
# binding do not cover them (tests call them through ctypes directly).
DEVICE_ONLY = {"lee_filter_field_static"}


def test_oracle_exports_the_same_abi(oracle_lib):
    missing = [n for n in declared_functions()
               if n not in DEVICE_ONLY and not hasattr(oracle_lib.dll, "orc_" + n[4:])]
    assert not missing, missing


def test_bindings_cover_the_header():
    bound = {"lee_" + n for n in api.SIGNATURES}
    assert set(declared_functions()) - DEVICE_ONLY <= bound


def test_no_cpu_fallback_without_gpu(product_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from camille_b200 import cases
    with pytest.raises(api.LeeError) as e:
        api.Solver(product_lib, cases.pulse2d(n=32, sponge=0))
    assert e.value.code == 7  # LEE_ERR_NODEVICE


@pytest.mark.parametrize("shift", [8, 8 * 50, -8 * 99])
def test_static_filter_refuses_overlapping_ranges(shift):
    """lee_filter_field_static reads stencil neighbours of every input point while its last pass
    writes the output: input and output ranges that share any element are refused with
    LEE_ERR_ARG before any device work (so this needs no GPU)."""
    dll = C.CDLL(api.PRODUCT_LIB)
    fn = dll.lee_filter_field_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    dll.lee_last_error.restype = C.c_char_p
    dll.lee_last_error.argtypes = [C.c_void_p]
    base = 1 << 20
    rc = fn(2, api.FILTER["STANDARD_CENTRAL"], 8, 1.0, 1.0, 10, 10, 1, C.c_void_p(base), C.c_void_p(base + shift),
            None)
    assert rc == api.LEE_ERR_ARG
    assert b"overlap" in dll.lee_last_error(None)
