"""Planner and recipe API on the GPU, mirroring the reference's
tests/test_planning.c and tests/test_plan_recipe.c, through the C-ABI."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import mofft_b200 as m
import oracle
from tests.conftest import cuda_available, max_abs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

TEST_N = 30
CTYPE = {32: np.complex64, 64: np.complex128}
SUF = {32: "f32", 64: "f64"}


def fn(name, bits):
    return getattr(m.load(), f"mofft_{name}_{SUF[bits]}")


def planning_input(n, bits):
    """tests/test_planning.c:11-23."""
    i = np.arange(n, dtype=np.float64)
    x = (np.sin(i * 0.31) + (i % 5) * 0.07) + 1j * (np.cos(i * 0.23) - (i % 7) * 0.03)
    return x.astype(CTYPE[bits])


def execute(plan_handle, bits, x, inplace):
    if inplace:
        y = x.copy()
        st = fn("execute", bits)(plan_handle, y.ctypes.data, y.ctypes.data)
    else:
        y = np.empty_like(x)
        st = fn("execute", bits)(plan_handle, x.ctypes.data, y.ctypes.data)
    assert st == 0
    return y


def tol(bits, n):
    """tests/test_planning.c:63, :78."""
    return 2e-4 * n if bits == 32 else 2e-11 * n


def test_measured_planner():
    """test_measured_planner (tests/test_planning.c:85-151)."""
    opts = m.PlanOptions(m.PLANNER_MEASURE, 0, 4, 3)
    for direction in (m.FORWARD, m.BACKWARD):
        for placement in (m.OUT_OF_PLACE, m.IN_PLACE):
            for bits in (32, 64):
                h = ctypes.c_void_p()
                d = m.Diagnostics()
                st = fn("plan_create_with_options", bits)(ctypes.byref(h), TEST_N, direction,
                                                          placement, ctypes.byref(opts),
                                                          ctypes.byref(d))
                assert st == 0
                assert d.measured == 1 and 1 <= d.candidates_measured <= 4
                assert d.kernel_bank < d.kernel_bank_count == 4
                assert d.selected_median_seconds > 0 and d.planning_seconds > 0
                assert d.length == TEST_N and d.precision_bits == bits
                assert int(np.prod(d.radix_list())) == TEST_N
                r = m.MeasureReport()
                assert fn("plan_get_measure_report", bits)(h, ctypes.byref(r)) == 0
                assert r.candidates == d.candidates_measured
                assert 1 <= r.winner_model_rank <= r.candidates
                assert 1 <= r.model_first_measured_rank <= r.candidates
                assert r.winner_seconds == d.selected_median_seconds
                assert r.winner_model_seconds > 0
                x = planning_input(TEST_N, bits)
                y = execute(h, bits, x, placement == m.IN_PLACE)
                ref = oracle.dft_ld(x.astype(np.complex128), direction)
                assert max_abs(y, ref) <= tol(bits, TEST_N)
                fn("plan_destroy", bits)(h)
    # a plan that was not measured has no report
    with m.Plan.create(64, m.FORWARD, bits=32) as p:
        with pytest.raises(m.MofftError):
            p.measure_report()


def test_measured_plan_of_a_large_batch():
    """MEASURE on a batch of 2^26 points (n = 4096 FP32, batch 16384): the
    candidates are timed on a bounded batch of 2^25 points, the model ranks
    them first, the report says how the model's order compared, and the plan
    runs the whole batch correctly."""
    import torch
    n, batch = 4096, 16384
    with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=batch,
                       mode=m.PLANNER_MEASURE, candidate_limit=6, timing_samples=3) as plan:
        r = plan.measure_report()
        print("measure report n=4096 batch=16384:", r)
        assert 1 <= r["winner_model_rank"] <= r["candidates"] <= 6
        assert r["winner_seconds"] > 0 and r["winner_model_seconds"] > 0
        x = oracle.uniform(n * batch, seed=3, dtype=np.complex64).reshape(batch, n)
        d = torch.from_numpy(x).cuda()
        y = torch.empty_like(d)
        plan.execute(d, y)
        torch.cuda.synchronize()
        rows = [0, 5000, batch - 1]
        ref = oracle.fft_ld(x[rows].astype(np.complex128), -1)
        got = y[rows].cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 5e-7 * 12


def test_large_measured_plan_keeps_input():
    """test_large_measured_plan (tests/test_planning.c:153-209): FP64 n=262144,
    the caller's input is not modified by planning and the plan runs finite."""
    n = 262144
    i = np.arange(n)
    x = ((i % 101) - 50) / 101.0 + 1j * (((i % 67) - 33) / 67.0)
    orig = x.copy()
    opts = m.PlanOptions(m.PLANNER_MEASURE, 0, 4, 3)
    h = ctypes.c_void_p()
    d = m.Diagnostics()
    assert fn("plan_create_with_options", 64)(ctypes.byref(h), n, m.FORWARD, m.OUT_OF_PLACE,
                                             ctypes.byref(opts), ctypes.byref(d)) == 0
    assert d.measured and 1 <= d.candidates_measured <= 4 and d.selected_median_seconds > 0
    assert np.array_equal(x, orig)
    y = execute(h, 64, x, False)
    assert np.all(np.isfinite(y))
    assert oracle.rel_l2(y, oracle.fft_ld(x, -1)) <= 2e-15 * np.log2(n)
    fn("plan_destroy", 64)(h)


def test_pretuned_strict_and_bound_api():
    """test_pretuned_and_bound_api (tests/test_planning.c:211-252)."""
    opts = m.PlanOptions(0, 0, 0, 0)
    h = ctypes.c_void_p()
    d = m.Diagnostics()
    assert fn("plan_create_with_options", 32)(ctypes.byref(h), TEST_N, m.FORWARD,
                                             m.OUT_OF_PLACE, ctypes.byref(opts),
                                             ctypes.byref(d)) == 0
    assert not d.measured and d.radix_count > 0 and d.kernel_bank_count > 0
    assert d.kernel_bank == 0 and d.used_model_fallback == 1 and d.used_wisdom == 0
    fn("plan_destroy", 32)(h)
    strict = m.PlanOptions(0, m.PLAN_STRICT_WISDOM, 0, 0)
    h2 = ctypes.c_void_p(1)
    assert fn("plan_create_with_options", 32)(ctypes.byref(h2), 17, m.FORWARD, m.OUT_OF_PLACE,
                                             ctypes.byref(strict), None) == \
        m.Status.WISDOM_NOT_FOUND
    assert h2.value is None
    x = planning_input(TEST_N, 32)
    y = np.empty_like(x)
    plan = fn("plan_dft_1d", 32)(TEST_N, x.ctypes.data, y.ctypes.data, m.FORWARD, 0)
    assert plan
    assert fn("execute_plan", 32)(plan) == 0
    assert max_abs(y, oracle.dft_ld(x.astype(np.complex128), -1)) <= tol(32, TEST_N)
    fn("plan_destroy", 32)(plan)
    # bound-array flags: MEASURE works, MEASURE|WISDOM_ONLY is refused
    plan = fn("plan_dft_1d", 32)(TEST_N, x.ctypes.data, y.ctypes.data, m.FORWARD, 1)
    assert plan
    assert fn("execute_plan", 32)(plan) == 0
    fn("plan_destroy", 32)(plan)
    assert not fn("plan_dft_1d", 32)(TEST_N, x.ctypes.data, y.ctypes.data, m.FORWARD, 3)
    # in place follows input == output
    z = x[:16].astype(np.complex128).copy()
    plan = fn("plan_dft_1d", 64)(16, z.ctypes.data, z.ctypes.data, m.BACKWARD, 0)
    assert plan
    assert fn("execute_plan", 64)(plan) == 0
    assert max_abs(z, oracle.dft_ld(x[:16].astype(np.complex128), 1)) <= tol(64, 16)
    fn("plan_destroy", 64)(plan)


def test_each_kernel_bank():
    """test_each_compiled_bank (tests/test_planning.c:254-302): chain {3, 10}."""
    radices = (ctypes.c_int * 2)(3, 10)
    for bank in (0, 1, 2, 3):   # default codelets, like-terms, even-odd, vector-reuse
        for direction in (m.FORWARD, m.BACKWARD):
            for bits in (32, 64):
                h = ctypes.c_void_p()
                assert fn("plan_create_with_radices", bits)(ctypes.byref(h), TEST_N, direction,
                                                            m.OUT_OF_PLACE, radices, 2) == 0
                assert fn("plan_set_kernel_bank", bits)(h, bank) == 0
                b = ctypes.c_uint()
                assert fn("plan_get_kernel_bank", bits)(h, ctypes.byref(b)) == 0 and b.value == bank
                assert fn("plan_set_kernel_bank", bits)(h, 4) == m.Status.INVALID_ARGUMENT
                x = planning_input(TEST_N, bits)
                y = execute(h, bits, x, False)
                assert max_abs(y, oracle.dft_ld(x.astype(np.complex128), direction)) <= \
                    tol(bits, TEST_N)
                fn("plan_destroy", bits)(h)


def test_single_stage_radix64_in_place():
    """test_single_stage_in_place (tests/test_planning.c:304-355)."""
    radix = (ctypes.c_int * 1)(64)
    for bank in (0, 1, 2, 3):
        for direction in (m.FORWARD, m.BACKWARD):
            for bits in (32, 64):
                h = ctypes.c_void_p()
                assert fn("plan_create_with_radices", bits)(ctypes.byref(h), 64, direction,
                                                            m.IN_PLACE, radix, 1) == 0
                assert fn("plan_set_kernel_bank", bits)(h, bank) == 0
                x = planning_input(64, bits)
                y = execute(h, bits, x, True)
                assert max_abs(y, oracle.dft_ld(x.astype(np.complex128), direction)) <= \
                    tol(bits, 64)
                # placement must match input == output
                other = np.empty_like(x)
                assert fn("execute", bits)(h, x.ctypes.data, other.ctypes.data) == \
                    m.Status.INVALID_ARGUMENT
                fn("plan_destroy", bits)(h)


# ------------------------------------------------------------- recipes

def recipe_input(n, bits):
    """tests/test_plan_recipe.c:93-96."""
    i = np.arange(n, dtype=np.float64)
    x = (0.2 + np.sin(i * 7 + 3) * 0.7) + 1j * (np.cos(i * 5 + 1) * 0.4 - 0.1)
    return x.astype(CTYPE[bits])


def relative_scale_error(a, b):
    """max |a-b| / (1 + |b|) (tests/test_plan_recipe.c:52-65)."""
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.max(np.abs(a - b) / (1 + np.abs(b))))


def export(h, bits):
    req = ctypes.c_size_t()
    assert fn("plan_export", bits)(h, None, 0, ctypes.byref(req)) == 0 and req.value >= 2
    small = ctypes.create_string_buffer(b"x", 1)
    req2 = ctypes.c_size_t()
    assert fn("plan_export", bits)(h, small, 1, ctypes.byref(req2)) == m.Status.BUFFER_TOO_SMALL
    assert req2.value == req.value and small.raw[:1] == b"x"
    buf = ctypes.create_string_buffer(req.value)
    assert fn("plan_export", bits)(h, buf, req.value, ctypes.byref(req2)) == 0
    raw = buf.raw[: req.value]
    assert raw[-1:] == b"\0" and raw[-2:-1] == b"\n" and m.build_id().encode() in raw
    return raw


@pytest.mark.parametrize("bank", [0, 1, 2, 3])
def test_recipe_replay(bank):
    """check_recipe_case (tests/test_plan_recipe.c:82-191) for n = 64 {4,4,4}
    and 96 {3,4,8}, both directions and placements, both precisions, plus the
    single-stage radix-64 in-place plan."""
    cases = [(64, [4, 4, 4]), (96, [3, 4, 8]), (64, [64])]
    for n, radices in cases:
        for direction in (m.FORWARD, m.BACKWARD):
            for placement in ((m.IN_PLACE,) if len(radices) == 1 else
                              (m.OUT_OF_PLACE, m.IN_PLACE)):
                for bits, eps in ((32, 2e-5), (64, 2e-10)):
                    arr = (ctypes.c_int * len(radices))(*radices)
                    h = ctypes.c_void_p()
                    assert fn("plan_create_with_radices", bits)(ctypes.byref(h), n, direction,
                                                                placement, arr,
                                                                len(radices)) == 0
                    assert fn("plan_set_kernel_bank", bits)(h, bank) == 0
                    mask = bank % 4 if len(radices) > 1 else 0
                    assert fn("plan_set_blocked_transpose_mask", bits)(h, mask) == 0
                    assert fn("plan_set_direct_input", bits)(h, bank & 1) == 0
                    layout = 1 if bank & 2 else 0
                    assert fn("plan_set_stage_layout", bits)(h, layout) == 0
                    raw = export(h, bits)
                    imp = ctypes.c_void_p()
                    d = m.Diagnostics()
                    assert fn("plan_import", bits)(ctypes.byref(imp), raw, len(raw),
                                                   ctypes.byref(d)) == 0
                    assert d.used_wisdom == 1 and d.measured == 0
                    assert d.candidates_measured == 0 and d.planning_seconds == 0.0
                    assert d.selected_median_seconds == 0.0 and d.length == n
                    assert d.precision_bits == bits and d.direction == direction
                    assert d.placement == placement and d.radix_count == len(radices)
                    assert d.kernel_bank == bank and d.blocked_transpose_mask == mask
                    assert d.direct_input == (bank & 1) and d.stage_layout == layout
                    assert d.radix_list() == radices
                    x = recipe_input(n, bits)
                    inplace = placement == m.IN_PLACE
                    a = execute(h, bits, x, inplace)
                    b = execute(imp, bits, x, inplace)
                    ref = oracle.dft_ld(x.astype(np.complex128), direction)
                    assert relative_scale_error(a, ref) <= eps
                    assert relative_scale_error(b, ref) <= eps
                    assert relative_scale_error(b, a) <= eps
                    # same schedule
                    sa, sb = m.Schedule(), m.Schedule()
                    fn("plan_get_schedule", bits)(h, ctypes.byref(sa))
                    fn("plan_get_schedule", bits)(imp, ctypes.byref(sb))
                    assert list(sa.kernels[:sa.pass_count]) == list(sb.kernels[:sb.pass_count])
                    fn("plan_destroy", bits)(h)
                    fn("plan_destroy", bits)(imp)


def test_recipe_rejections():
    """test_rejections (tests/test_plan_recipe.c:196-241)."""
    radices = (ctypes.c_int * 3)(4, 4, 4)
    h = ctypes.c_void_p()
    assert fn("plan_create_with_radices", 32)(ctypes.byref(h), 64, m.FORWARD, m.OUT_OF_PLACE,
                                              radices, 3) == 0
    raw = bytearray(export(h, 32))
    fn("plan_destroy", 32)(h)
    size = len(raw)

    def bad(data, length, expected, bits=32):
        out = ctypes.c_void_p(1)
        st = fn("plan_import", bits)(ctypes.byref(out), bytes(data), length, None)
        assert st == expected and out.value is None

    bad(raw, size - 1, m.Status.INVALID_ARGUMENT)
    bad(raw, size - 2, m.Status.INVALID_ARGUMENT)
    x = bytearray(raw)
    x[0:1] = b"X"
    bad(x, size, m.Status.INCOMPATIBLE_RECIPE)
    off = len("MOFFT_PLAN_V1 ")
    x = bytearray(raw)
    x[off] = ord("1") if raw[off] == ord("0") else ord("0")
    bad(x, size, m.Status.INCOMPATIBLE_RECIPE)
    fam = off + 65
    x = bytearray(raw)
    x[fam] = ord("1") if raw[fam] == ord("0") else ord("0")
    bad(x, size, m.Status.INCOMPATIBLE_RECIPE)
    bad(raw, size, m.Status.INCOMPATIBLE_RECIPE, bits=64)
    bad(raw + b"x\0", size + 2, m.Status.INVALID_ARGUMENT)


def test_bound_array_measure_equals_pretuned_result():
    """MEASURE and PRETUNED plans of the same length agree."""
    n = 4096
    x = oracle.uniform(n, seed=4).astype(np.complex64)
    y1 = np.empty_like(x)
    y2 = np.empty_like(x)
    p1 = fn("plan_dft_1d", 32)(n, x.ctypes.data, y1.ctypes.data, m.FORWARD, 0)
    p2 = fn("plan_dft_1d", 32)(n, x.ctypes.data, y2.ctypes.data, m.FORWARD, 1)
    assert p1 and p2
    assert fn("execute_plan", 32)(p1) == 0 and fn("execute_plan", 32)(p2) == 0
    ref = oracle.fft_ld(x.astype(np.complex128), -1)
    assert oracle.rel_l2(y1, ref) <= 5e-7 * 12 and oracle.rel_l2(y2, ref) <= 5e-7 * 12
    fn("plan_destroy", 32)(p1)
    fn("plan_destroy", 32)(p2)


def test_tuned_three_pass_only_where_a_workspace_exists_anyway():
    """FP64 n = 2^20: the compiled wisdom holds a three-pass schedule.  In
    place (which needs a batch-sized workspace in any case) the plan uses it;
    out of place the plan keeps the two-pass model schedule, which needs no
    workspace, so tuning never costs memory."""
    n = 1 << 20
    with m.Plan.create(n, m.FORWARD, m.IN_PLACE, bits=64, batch=2) as p:
        s = p.schedule()
        assert s["pass_count"] == 3 and s["workspace_bytes"] > 0
    with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=64, batch=2) as p:
        s = p.schedule()
        assert s["pass_count"] == 2 and s["workspace_bytes"] == 0
