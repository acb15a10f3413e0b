"""The allocation-free entry point mofft_execute_fixed_scratch_f32.

It exists for callers that cannot allocate device memory (a host framework
that owns the whole GPU memory budget, or a latency-critical loop that must
not call cudaMalloc / cudaFree).  Its scratch is a static device array shared
by every call, so this file checks, through the C-ABI, two calls in a row
against the plan-based entry point (mofft_execute_f32 on an in-place batched
plan, which uses its own allocated workspace), within the FP32 tolerance the
other tests use (rel-L2 <= 5e-7 * log2 n), plus the size limits.  It is
collected last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import mofft_b200 as m
from tests.conftest import cuda_available, fp32_tol, rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

LIMIT = 1 << 22


def _fixed(lib, x, y, n, batch, direction, stream=None):
    return lib.mofft_execute_fixed_scratch_f32(x.data_ptr(), y.data_ptr(), n, batch,
                                               direction, stream)


def _planned(x, n, batch, direction):
    y = x.clone()
    with m.Plan.create(n, direction, m.IN_PLACE, bits=32, batch=batch) as plan:
        plan.execute(y, y)
    return y


def test_two_calls_match_plan_api():
    import torch
    lib = m.load()
    lib.mofft_execute_fixed_scratch_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_size_t, ctypes.c_size_t,
                                                    ctypes.c_int, ctypes.c_void_p]
    lib.mofft_execute_fixed_scratch_f32.restype = ctypes.c_int
    gen = torch.Generator(device="cuda").manual_seed(21)
    cases = [(1 << 16, 32, m.FORWARD), (1 << 20, 4, m.BACKWARD)]   # second fills the limit
    for n, batch, direction in cases:
        x = torch.view_as_complex(torch.rand((batch, n, 2), generator=gen, device="cuda") * 2 - 1)
        want = _planned(x, n, batch, direction)
        for _ in range(2):                     # two calls in a row reuse the scratch
            y = torch.empty_like(x)
            assert _fixed(lib, x, y, n, batch, direction) == m.Status.SUCCESS
            torch.cuda.synchronize()
            err = rel_l2(y.cpu().numpy(), want.cpu().numpy())
            assert err <= fp32_tol(n), (n, batch, direction, err)
        z = x.clone()                          # in place as well
        assert _fixed(lib, z, z, n, batch, direction) == m.Status.SUCCESS
        torch.cuda.synchronize()
        assert rel_l2(z.cpu().numpy(), want.cpu().numpy()) <= fp32_tol(n)


def test_limits_are_rejected():
    import torch
    lib = m.load()
    lib.mofft_execute_fixed_scratch_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_size_t, ctypes.c_size_t,
                                                    ctypes.c_int, ctypes.c_void_p]
    x = torch.zeros((8, 1 << 20), dtype=torch.complex64, device="cuda")
    # beyond the static array: 8 * 2^20 > 2^22 points
    assert _fixed(lib, x, x, 1 << 20, 8, m.FORWARD) == m.Status.UNSUPPORTED_SIZE
    # a one-pass length needs no scratch
    assert _fixed(lib, x, x, 4096, 2, m.FORWARD) == m.Status.UNSUPPORTED_SIZE
    assert _fixed(lib, x, x, 17 * 4096, 1, m.FORWARD) == m.Status.UNSUPPORTED_SIZE
    assert _fixed(lib, x, x, 1 << 16, 0, m.FORWARD) == m.Status.INVALID_ARGUMENT
    assert _fixed(lib, x, x, 1 << 16, 1, 0) == m.Status.INVALID_ARGUMENT
    host = np.zeros(1 << 16, dtype=np.complex64)
    assert lib.mofft_execute_fixed_scratch_f32(host.ctypes.data, host.ctypes.data, 1 << 16, 1,
                                               m.FORWARD, None) == m.Status.INVALID_ARGUMENT
    assert LIMIT == 1 << 22
