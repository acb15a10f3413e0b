"""Thread-block-cluster kernels (cluster_*): one transform of 2^14..2^16 FP32
/ 2^14..2^15 FP64 points per cluster of 4-16 CTAs, the four-step transpose
carried by bulk copies between the CTAs' shared memories.  Checked against the
oracle through the C-ABI with explicit kernel plans (the planner runs them
only when a tuned or explicit kernel list names them): both directions, in
and out of place, a distance that leaves gaps, a batch of 2^24 points sampled
across the batch, and the bounded wait for the exchanged tiles (CTA 0 of
every cluster never sends, every wait runs out, the plan reports
MOFFT_INTERNAL_ERROR and then executes normally)."""
from __future__ import annotations

import time

import numpy as np
import pytest

import mofft_b200 as m
import oracle
from tests.conftest import cuda_available, fp32_tol, fp64_tol, rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

CTYPE = {32: np.complex64, 64: np.complex128}


def cluster_kernels():
    return [k for k in m.kernels() if k["name"].startswith("cluster_")]


def tol(n, bits):
    return fp32_tol(n) if bits == 32 else fp64_tol(n)


def test_cluster_kernels_registered():
    names = sorted(k["name"] for k in cluster_kernels())
    assert names == ["cluster_double_128x128_k8", "cluster_double_128x256_k16",
                     "cluster_float_128x128_k4", "cluster_float_128x256_k8",
                     "cluster_float_256x256_k16"]
    for k in cluster_kernels():
        assert k["kind"] == m.KERNEL_ROWS and k["lines"] == 1


@pytest.mark.parametrize("dist_pad", [0, 3])
def test_cluster_kernels_against_oracle(dist_pad):
    import torch
    for k in cluster_kernels():
        n, bits = k["length"], k["precision_bits"]
        batch, dist = 6, n + dist_pad
        buf = oracle.uniform(batch * dist, seed=n + dist_pad, dtype=CTYPE[bits])
        lines = buf.reshape(batch, dist)[:, :n].astype(np.complex128)
        for direction in (m.FORWARD, m.BACKWARD):
            ref = oracle.fft_ld(lines, direction)
            for inplace in (False, True):
                x = torch.from_numpy(buf.copy()).cuda()
                y = x if inplace else torch.full_like(x, 7.0)
                with m.Plan.create(n, direction, m.IN_PLACE if inplace else m.OUT_OF_PLACE,
                                   bits=bits, batch=batch, distance=dist,
                                   kernels=[k["index"]]) as plan:
                    plan.execute(x, y)
                torch.cuda.synchronize()
                got = y.cpu().numpy().reshape(batch, dist)
                err = rel_l2(got[:, :n], ref)
                assert err <= tol(n, bits), (k["name"], direction, inplace, dist, err)
                if dist_pad and not inplace:
                    assert np.all(got[:, n:] == 7.0), k["name"]   # gaps untouched


def test_cluster_kernels_full_batch_sampled():
    """2^24 points per call; rows at both ends and in the middle of the batch
    against the oracle."""
    import torch
    for k in cluster_kernels():
        n, bits = k["length"], k["precision_bits"]
        batch = (1 << 24) // n
        gen = torch.Generator(device="cuda").manual_seed(n + bits)
        x = torch.view_as_complex(
            (torch.rand((batch, n, 2), generator=gen, device="cuda",
                        dtype=torch.float32 if bits == 32 else torch.float64) * 2 - 1)
            .contiguous())
        rows = sorted({0, 1, batch // 2, batch - 1})
        src = x[rows].cpu().numpy().astype(np.complex128)
        ref = oracle.fft_ld(src, m.FORWARD)
        with m.Plan.create(n, m.FORWARD, m.IN_PLACE, bits=bits, batch=batch,
                           kernels=[k["index"]]) as plan:
            plan.execute(x, x)
        torch.cuda.synchronize()
        assert rel_l2(x[rows].cpu().numpy(), ref) <= tol(n, bits), k["name"]


def test_cluster_lost_tiles_report_error_then_recover():
    import torch
    lib = m.load()
    k = next(k for k in cluster_kernels() if k["name"] == "cluster_float_256x256_k16")
    n, batch = k["length"], 8
    x = oracle.uniform(batch * n, seed=5, dtype=np.complex64).reshape(batch, n)
    ref = oracle.fft_ld(x.astype(np.complex128), m.FORWARD)
    d = torch.from_numpy(x).cuda()
    out = torch.zeros_like(d)
    with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=batch,
                       kernels=[k["index"]]) as plan:
        t0 = time.perf_counter()
        st = lib.mofft_plan_check_lost_copy_f32(plan.handle, d.data_ptr(), out.data_ptr())
        waited = time.perf_counter() - t0
        assert st == m.Status.INTERNAL_ERROR
        assert waited < 30.0, waited
        plan.check_status()                       # the error word was cleared
        out.zero_()
        plan.execute(d, out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref) <= fp32_tol(n)
