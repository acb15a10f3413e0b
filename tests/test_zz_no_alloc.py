"""The allocation-free entry point mofft_execute_fixed_scratch_f32.

It exists for callers that cannot allocate device memory (a host framework
that owns the whole GPU memory budget, or a latency-critical loop that must
not call cudaMalloc / cudaFree).  Its scratch is a static device array shared
by every call, so this file checks, through the C-ABI, two calls in a row
against the plan-based entry point (mofft_execute_f32 on an in-place batched
plan, which uses its own allocated workspace), within the FP32 tolerance the
other tests use (rel-L2 <= 5e-7 * log2 n), plus the size limits.  It is
collected last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process.  Each result is
also checked against the long-double oracle, on power-of-two lengths and on
two-pass lengths with radix-3, -5 and -7 stages (whose twiddle tables have
odd radices and super-stage tables of uneven size), on the default stream
and on a caller's stream."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import mofft_b200 as m
import oracle
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


def _bind(lib):
    lib.mofft_execute_fixed_scratch_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_size_t, ctypes.c_size_t,
                                                    ctypes.c_int, ctypes.c_void_p]
    lib.mofft_execute_fixed_scratch_f32.restype = ctypes.c_int


def _oracle_rows(x, direction, rows):
    xs = x.cpu().numpy()[rows].astype(np.complex128)
    return oracle.fft_ld(xs, direction)


# (length, batch, direction); 2^20 x 4 fills the static array
CASES = [(1 << 16, 32, m.FORWARD), (1 << 20, 4, m.BACKWARD),
         (3 << 15, 8, m.FORWARD), (3 << 15, 8, m.BACKWARD),
         (5 << 14, 4, m.BACKWARD), (7 << 14, 3, m.FORWARD)]


@pytest.mark.parametrize("n,batch,direction", CASES)
def test_two_calls_match_plan_api_and_oracle(n, batch, direction):
    import torch
    lib = m.load()
    _bind(lib)
    gen = torch.Generator(device="cuda").manual_seed(21 + n % 97)
    x = torch.view_as_complex(torch.rand((batch, n, 2), generator=gen, device="cuda") * 2 - 1)
    want = _planned(x, n, batch, direction).cpu().numpy()
    rows = sorted({0, batch // 2, batch - 1})
    ref = _oracle_rows(x, direction, rows)
    assert rel_l2(want[rows], ref) <= fp32_tol(n)
    for _ in range(2):                     # two calls in a row reuse the scratch
        y = torch.empty_like(x)
        assert _fixed(lib, x, y, n, batch, direction) == m.Status.SUCCESS
        torch.cuda.synchronize()
        got = y.cpu().numpy()
        err = rel_l2(got, want)
        assert err <= fp32_tol(n), (n, batch, direction, err)
        assert rel_l2(got[rows], ref) <= fp32_tol(n), (n, batch, direction)
    z = x.clone()                          # in place as well
    assert _fixed(lib, z, z, n, batch, direction) == m.Status.SUCCESS
    torch.cuda.synchronize()
    assert rel_l2(z.cpu().numpy(), want) <= fp32_tol(n)


def test_caller_stream_and_alternating_lengths():
    """Calls enqueued on a caller's stream, alternating between two lengths
    with different twiddle layouts, so that each call must rewrite what the
    previous one left in the shared array."""
    import torch
    lib = m.load()
    _bind(lib)
    stream = torch.cuda.Stream()
    gen = torch.Generator(device="cuda").manual_seed(5)
    shapes = [(5 << 14, 2), (1 << 16, 4), (5 << 14, 2), (1 << 16, 4)]
    for n, batch in shapes:
        x = torch.view_as_complex(torch.rand((batch, n, 2), generator=gen,
                                             device="cuda") * 2 - 1)
        torch.cuda.synchronize()
        y = torch.empty_like(x)
        with torch.cuda.stream(stream):
            assert lib.mofft_execute_fixed_scratch_f32(x.data_ptr(), y.data_ptr(), n, batch,
                                                       m.FORWARD,
                                                       stream.cuda_stream) == m.Status.SUCCESS
        stream.synchronize()
        ref = _oracle_rows(x, m.FORWARD, list(range(batch)))
        assert rel_l2(y.cpu().numpy(), ref) <= fp32_tol(n), (n, batch)


def test_limits_are_rejected():
    import torch
    lib = m.load()
    _bind(lib)
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
