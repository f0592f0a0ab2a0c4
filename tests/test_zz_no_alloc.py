"""cufsp_vec_sum_noalloc: the vector sum that allocates no device memory (gpu).

Some callers cannot call cudaMalloc or let a library do it for them -- e.g. a runtime that owns all
device memory through its own pool and accounts for every byte.  This entry point keeps its scratch
in a fixed __device__ array of the library, so it must (1) give the same sums as the allocating
cufsp_vec_sum, (2) leave nothing behind that spoils the next call (every call shares the array),
and (3) refuse inputs larger than that array covers.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from cuda_fsp_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_N = 4194304  # CUFSP_NOALLOC_MAX_N


def _sum_alloc(lib, x, stream):
    out = C.c_double()
    _lib.check(lib, lib.cufsp_vec_sum(x.numel(), x.data_ptr(), C.byref(out), stream), "cufsp_vec_sum")
    return out.value


def _sum_noalloc(lib, x, d_out, stream):
    _lib.check(lib, lib.cufsp_vec_sum_noalloc(x.numel(), x.data_ptr(), d_out.data_ptr(), stream),
               "cufsp_vec_sum_noalloc")


def test_noalloc_sum_matches_allocating_sum_on_consecutive_calls(cuda):
    import torch
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda").manual_seed(7)
    # two calls in a row on different inputs and sizes: the shared scratch must not carry state over
    for n, shift in ((MAX_N, 0.25), (1000003, -0.5)):
        x = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - shift
        d_out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        _sum_noalloc(lib, x, d_out, stream)
        torch.cuda.synchronize()
        got = d_out.item()
        ref = _sum_alloc(lib, x, stream)
        # different block shapes add in a different order: agree to a few ulps of sum |x|
        assert abs(got - ref) <= 1e-13 * x.abs().sum().item(), (n, got, ref)
        assert abs(got - x.sum().item()) <= 1e-13 * x.abs().sum().item()
    # a repeat of the same input reproduces the same bits (fixed summation order)
    d2 = torch.zeros(1, dtype=torch.float64, device="cuda")
    _sum_noalloc(lib, x, d2, stream)
    torch.cuda.synchronize()
    assert d2.item() == got


def test_noalloc_sum_small_and_empty(cuda):
    import torch
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    x = torch.tensor([1.5, -2.0, 4.25], dtype=torch.float64, device="cuda")
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda")
    _sum_noalloc(lib, x, d_out, stream)
    torch.cuda.synchronize()
    assert d_out.item() == 3.75
    empty = torch.zeros(0, dtype=torch.float64, device="cuda")
    d_out.fill_(9.0)
    _sum_noalloc(lib, empty, d_out, stream)
    torch.cuda.synchronize()
    assert d_out.item() == 0.0


def test_noalloc_sum_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    lib = _lib.load()
    x = torch.zeros(MAX_N + 1, dtype=torch.float64, device="cuda")
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = lib.cufsp_vec_sum_noalloc(x.numel(), x.data_ptr(), d_out.data_ptr(), None)
    assert _lib.STATUS[st] == "CUFSP_ERR_INVALID_ARG"
    assert b"CUFSP_NOALLOC_MAX_N" in lib.cufsp_last_error()
