"""Tensor-core precision forms of the FP32 transform (n = 4096 and 65536).

MOFFT_FORM_TF32X3 and MOFFT_FORM_BF16X3 run the three radix-16 Stockham
stages as DFT-matrix GEMMs on the tcgen05 tensor cores with split operands
(hi + lo, three products, FP32 accumulation).  They are checked against the
long-double oracle on the precision-mix inputs (a third uniform[-1,1), a
third log-uniform magnitudes 1e-3..1e3 with uniform phase, a third single
tones), forward and backward, in place and out of place, through the C-ABI.
n = 65536 runs two column passes of 256-point lines (same GEMMs, 16 lines
per tile, super-stage twiddles between the passes); its bounds are the same
per stage, four stages instead of three.

Tolerance: both forms must meet the FP32 bar of every other FP32 result,
relative L2 error <= 5e-7 * log2 n against the FP64 oracle (6.0e-6 at 4096,
8.0e-6 at 65536), over the batch and over each input class of the mix on its
own.  (TF32X3 operands carry 2 x 11 significant bits, about 3 * 2^-22 per
product; BF16X3 2 x 8 bits, about 3 * 2^-18 per product, which averages to
well under the bar over a transform.)  The CUDA-core FP32 path of the same
plan stays within the same bound and is at least as accurate as TF32X3, which
in turn is more accurate than BF16X3."""
from __future__ import annotations

import numpy as np
import pytest

import mofft_b200 as m
import oracle
from mofft_b200 import workloads
from tests.conftest import cuda_available, fp32_tol, rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

N = 4096
TOL = {m.FORM_TF32X3: fp32_tol(N), m.FORM_BF16X3: fp32_tol(N)}
NAMES = {m.FORM_TF32X3: "tf32x3", m.FORM_BF16X3: "bf16x3"}


def _mix(batch: int, seed: int = 3, n: int = N) -> np.ndarray:
    return workloads.precision_mix(batch * n, n, seed=seed)


def _expected(x: np.ndarray, direction: int) -> np.ndarray:
    return oracle.fft_ld(x.astype(np.complex128), direction)


def _run(x: np.ndarray, direction: int, placement: int, form: int) -> np.ndarray:
    import torch
    batch, n = x.shape
    d = torch.from_numpy(x).cuda()
    out = d if placement == m.IN_PLACE else torch.empty_like(d)
    with m.Plan.create(n, direction, placement, bits=32, batch=batch) as plan:
        plan.set_precision_form(form)
        assert plan.precision_form == form
        plan.execute(d, out)
    return out.cpu().numpy()


@pytest.mark.parametrize("form", [m.FORM_TF32X3, m.FORM_BF16X3])
@pytest.mark.parametrize("direction", [m.FORWARD, m.BACKWARD])
@pytest.mark.parametrize("placement", [m.OUT_OF_PLACE, m.IN_PLACE])
def test_form_matches_oracle(form, direction, placement):
    x = _mix(24)
    want = _expected(x, direction)
    got = _run(x, direction, placement, form)
    err = rel_l2(got, want)
    assert err <= TOL[form], (NAMES[form], direction, placement, err)
    # every input class of the mix within the bound on its own
    third = x.shape[0] // 3
    for lo, hi in ((0, third), (third, 2 * third), (2 * third, x.shape[0])):
        e = rel_l2(got[lo:hi], want[lo:hi])
        assert e <= TOL[form], (NAMES[form], lo, e)


def test_error_ordering_fp32_tf32x3_bf16x3():
    x = _mix(12, seed=9)
    want = _expected(x, m.FORWARD)
    errs = {f: rel_l2(_run(x, m.FORWARD, m.OUT_OF_PLACE, f), want)
            for f in (m.FORM_FP32, m.FORM_TF32X3, m.FORM_BF16X3)}
    print("rel-L2 vs oracle:", {("fp32", "tf32x3", "bf16x3")[f]: f"{e:.3e}"
                                for f, e in errs.items()})
    assert errs[m.FORM_FP32] <= fp32_tol(N)
    assert errs[m.FORM_FP32] <= errs[m.FORM_TF32X3] * 1.5
    assert errs[m.FORM_TF32X3] < errs[m.FORM_BF16X3]


def test_roundtrip_and_repeat_bitwise():
    import torch
    x = _mix(6, seed=4)
    d = torch.from_numpy(x).cuda()
    y1 = torch.empty_like(d)
    y2 = torch.empty_like(d)
    z = torch.empty_like(d)
    with m.Plan.create(N, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=6) as fwd, \
            m.Plan.create(N, m.BACKWARD, m.OUT_OF_PLACE, bits=32, batch=6) as bwd:
        fwd.set_precision_form(m.FORM_TF32X3)
        bwd.set_precision_form(m.FORM_TF32X3)
        fwd.execute(d, y1)
        fwd.execute(d, y2)
        bwd.execute(y1, z)
    assert torch.equal(y1, y2)            # deterministic
    back = z.cpu().numpy() / N
    assert rel_l2(back, x) <= 2 * TOL[m.FORM_TF32X3]


def test_schedule_switch_and_unsupported_length():
    kernels = {k["index"]: k for k in m.kernels()}
    tensor = [k for k in kernels.values() if k["kind"] == m.KERNEL_TENSOR]
    assert sorted(k["name"] for k in tensor) == ["tensor_float_4096_bf16x3_r16x3",
                                                "tensor_float_4096_bf16x3_r64x2",
                                                "tensor_float_4096_tf32x3_r16x3"]
    with m.Plan.create(N, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=4) as plan:
        base = plan.schedule()
        plan.set_precision_form(m.FORM_BF16X3)
        s = plan.schedule()
        assert s["pass_count"] == 1
        assert kernels[s["kernels"][0]]["name"] == "tensor_float_4096_bf16x3_r64x2"
        plan.set_precision_form(m.FORM_FP32)
        assert plan.schedule()["kernels"] == base["kernels"]
    with m.Plan.create(2048, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=4) as plan:
        with pytest.raises(m.MofftError) as e:
            plan.set_precision_form(m.FORM_TF32X3)
        assert e.value.status == m.Status.UNSUPPORTED_SIZE
        assert plan.precision_form == m.FORM_FP32
        plan.execute(*_pair(2048, 4))      # still runs its FP32 schedule


def _pair(n, batch):
    import torch
    x = torch.ones((batch, n), dtype=torch.complex64, device="cuda")
    return x, torch.empty_like(x)


def test_host_buffers_distance_and_stream():
    import torch
    batch, dist = 5, N + 96
    x = np.zeros((batch, dist), dtype=np.complex64)
    x[:, :N] = _mix(batch, seed=8)[:batch]
    want = _expected(x[:, :N], m.BACKWARD)
    y = np.zeros_like(x)
    with m.Plan.create(N, m.BACKWARD, m.OUT_OF_PLACE, bits=32, batch=batch,
                       distance=dist) as plan:
        plan.set_precision_form(m.FORM_TF32X3)
        plan.execute(x, y)                  # host buffers: staged copies
        assert rel_l2(y[:, :N], want) <= TOL[m.FORM_TF32X3]
        d = torch.from_numpy(x).cuda()
        o = torch.zeros_like(d)
        stream = torch.cuda.Stream()
        plan.set_stream(stream.cuda_stream)
        with torch.cuda.stream(stream):
            plan.execute(d, o)              # asynchronous on the attached stream
        plan.check_status()                 # blocking; no wait timed out
        got = o.cpu().numpy()
    assert rel_l2(got[:, :N], want) <= TOL[m.FORM_TF32X3]
    assert not np.any(got[:, N:])           # padding between transforms untouched


def test_form_from_plan_option_flags():
    import ctypes
    import torch
    lib = m.load()
    x = _mix(4, seed=12)
    want = _expected(x, m.FORWARD)
    for bit, form in ((m.PLAN_FORM_TF32X3, m.FORM_TF32X3), (m.PLAN_FORM_BF16X3, m.FORM_BF16X3)):
        h = ctypes.c_void_p()
        opts = m.PlanOptions(m.PLANNER_PRETUNED, bit, 0, 0)
        diag = m.Diagnostics()
        st = lib.mofft_plan_create_batched_f32(ctypes.byref(h), N, 4, 0, m.FORWARD,
                                               m.OUT_OF_PLACE, ctypes.byref(opts),
                                               ctypes.byref(diag))
        assert st == m.Status.SUCCESS
        plan = m.Plan(h.value, 32)
        assert plan.precision_form == form
        d = torch.from_numpy(x).cuda()
        out = torch.empty_like(d)
        plan.execute(d, out)
        plan.destroy()
        assert rel_l2(out.cpu().numpy(), want) <= TOL[form]
    # a length without a tensor-core kernel
    h = ctypes.c_void_p()
    opts = m.PlanOptions(m.PLANNER_PRETUNED, m.PLAN_FORM_TF32X3, 0, 0)
    st = lib.mofft_plan_create_with_options_f32(ctypes.byref(h), 2048, m.FORWARD,
                                                m.OUT_OF_PLACE, ctypes.byref(opts), None)
    assert st == m.Status.UNSUPPORTED_SIZE and h.value is None


N2 = 65536
TOL2 = {m.FORM_TF32X3: fp32_tol(N2), m.FORM_BF16X3: fp32_tol(N2)}


@pytest.mark.parametrize("form", [m.FORM_TF32X3, m.FORM_BF16X3])
@pytest.mark.parametrize("direction", [m.FORWARD, m.BACKWARD])
@pytest.mark.parametrize("placement", [m.OUT_OF_PLACE, m.IN_PLACE])
def test_form_65536_matches_oracle(form, direction, placement):
    x = _mix(6, seed=5, n=N2)
    want = _expected(x, direction)
    got = _run(x, direction, placement, form)
    err = rel_l2(got, want)
    assert err <= TOL2[form], (NAMES[form], direction, placement, err)
    for lo, hi in ((0, 2), (2, 4), (4, 6)):   # each input class of the mix
        assert rel_l2(got[lo:hi], want[lo:hi]) <= TOL2[form]


def test_form_65536_schedule_and_error_ordering():
    kernels = {k["index"]: k for k in m.kernels()}
    with m.Plan.create(N2, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=2) as plan:
        plan.set_precision_form(m.FORM_TF32X3)
        s = plan.schedule()
        assert s["pass_count"] == 2
        assert [kernels[k]["name"] for k in s["kernels"]] == \
            ["tensor_cols_float_256_tf32x3_c16"] * 2
    x = _mix(3, seed=6, n=N2)
    want = _expected(x, m.FORWARD)
    errs = {f: rel_l2(_run(x, m.FORWARD, m.OUT_OF_PLACE, f), want)
            for f in (m.FORM_FP32, m.FORM_TF32X3, m.FORM_BF16X3)}
    print("n=65536 rel-L2 vs oracle:", {("fp32", "tf32x3", "bf16x3")[f]: f"{e:.3e}"
                                        for f, e in errs.items()})
    assert errs[m.FORM_FP32] <= fp32_tol(N2)
    assert errs[m.FORM_TF32X3] < errs[m.FORM_BF16X3]


@pytest.mark.parametrize("n", [N, N2])
def test_precision_config_full_size_sampled(n):
    """The precision-form workload at its full size, 2^27 points (n = 4096,
    batch 32768; n = 65536, batch 2048) of the precision mix, out of place:
    the CUDA-core form and both tensor-core forms, 72 rows spread over the
    batch (every input class, the last CTAs) against the long-double oracle."""
    import torch
    points = 1 << 27
    batch = points // n
    x = workloads.precision_mix(points, n, seed=11)
    rows = sorted(set(np.linspace(0, batch - 1, 64).astype(int).tolist()) |
                  set(range(batch - 8, batch)))
    want = _expected(x[rows], m.FORWARD)
    d = torch.from_numpy(x).cuda()
    del x
    out = torch.empty_like(d)
    errs = {}
    for form in (m.FORM_FP32, m.FORM_TF32X3, m.FORM_BF16X3):
        with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=batch) as plan:
            plan.set_precision_form(form)
            plan.execute(d, out)
        torch.cuda.synchronize()
        got = out[rows].cpu().numpy()
        errs[form] = rel_l2(got, want)
        assert errs[form] <= fp32_tol(n), (n, form, errs[form])
    print(f"n={n} 2^27 points rel-L2:", {("fp32", "tf32x3", "bf16x3")[f]: f"{e:.3e}"
                                           for f, e in errs.items()})


@pytest.mark.parametrize("form", [m.FORM_TF32X3, m.FORM_BF16X3])
def test_lost_copy_times_out_and_plan_stays_usable(form):
    """The tensor-core kernels bound every wait: a launch whose first wait
    can never be satisfied (radix-16 kernel: the input copies are never
    issued; radix-64 kernel: the first GEMM is never issued) ends in
    MOFFT_INTERNAL_ERROR after about a second (no GPU fault, TMEM released),
    and the same plan then executes correctly on the same context."""
    import ctypes
    import time
    import torch
    lib = m.load()
    x = _mix(8, seed=21)
    want = _expected(x, m.FORWARD)
    d = torch.from_numpy(x).cuda()
    out = torch.empty_like(d)
    with m.Plan.create(N, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=8) as plan:
        assert lib.mofft_plan_check_lost_copy_f32(plan.handle, d.data_ptr(), out.data_ptr()) \
            == m.Status.INVALID_ARGUMENT          # CUDA-core schedule: nothing to check
        plan.set_precision_form(form)
        t0 = time.perf_counter()
        st = lib.mofft_plan_check_lost_copy_f32(plan.handle, d.data_ptr(), out.data_ptr())
        waited = time.perf_counter() - t0
        assert st == m.Status.INTERNAL_ERROR
        assert waited < 30.0, waited
        plan.check_status()                       # the error word was cleared
        plan.execute(d, out)
    assert rel_l2(out.cpu().numpy(), want) <= TOL[form]
