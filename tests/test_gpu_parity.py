"""GPU parity: libmofft.so (sm_100a kernels, through the C-ABI) against the
oracle and the reference's own test cases.  Mirrors tests/test_fft.c,
tests/test_binary_banks.c and tests/test_planning.c of the reference, plus the
batched workloads (n=1024 x 4096 forward/backward, the power-of-two / 3*2^k /
5*2^k sweep) with the rel-L2 bounds 5e-7*log2(n) (FP32) and 2e-15*log2(n)
(FP64)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import mofft_b200 as m
import oracle
from tests.conftest import (DBL_EPS, FLT_EPS, cuda_available, fp32_tol, fp64_tol, max_abs,
                            rel_l2, three_mode_expected, three_mode_input)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

CTYPE = {32: np.complex64, 64: np.complex128}


def run_host(x: np.ndarray, direction: int, *, bits: int, inplace: bool = False,
             radices=None, bank: int = 0, kernels=None) -> np.ndarray:
    """Execute through the C-ABI with host (numpy) buffers."""
    x = np.ascontiguousarray(x, dtype=CTYPE[bits])
    n = x.shape[-1]
    batch = x.size // n
    with m.Plan.create(n, direction, m.IN_PLACE if inplace else m.OUT_OF_PLACE, bits=bits,
                       batch=batch, radices=radices, kernels=kernels) as plan:
        if bank:
            plan.set_kernel_bank(bank)
        if inplace:
            y = x.copy()
            plan.execute(y, y)
        else:
            y = np.empty_like(x)
            plan.execute(x, y)
    return y


def oracle_ref(x: np.ndarray, direction: int) -> np.ndarray:
    n = x.shape[-1]
    if n <= (1 << 20):
        return oracle.fft_ld(x, direction)
    return oracle.fft_port(np.asarray(x, np.complex128), direction, threads=8)


# ---------------------------------------------------------------- test_fft.c

FFT_SIZES = (2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32, 45, 64, 144, 225, 256)


@pytest.mark.parametrize("n", FFT_SIZES)
def test_reference_sizes_against_golden(n, golden_transforms):
    """tests/test_fft.c:489-573: every size x direction x placement, FP32 and
    FP64, max-abs tolerance 32*FLT_EPS*n / 96*DBL_EPS*n vs the direct DFT."""
    for d in (-1, 1):
        x = golden_transforms[f"fft_{n}_{d}_in"]
        want = golden_transforms[f"fft_{n}_{d}_out"]
        for inplace in (False, True):
            y32 = run_host(x.astype(np.complex64), d, bits=32, inplace=inplace)
            y64 = run_host(x, d, bits=64, inplace=inplace)
            assert max_abs(y32, want.astype(np.complex64)) <= 32 * FLT_EPS * n, (n, d, inplace)
            assert max_abs(y64, want) <= 96 * DBL_EPS * n, (n, d, inplace)


def test_unsupported_length():
    lib = m.load()
    h = ctypes.c_void_p(1)
    assert lib.mofft_plan_create_f32(ctypes.byref(h), 17, m.FORWARD,
                                     m.OUT_OF_PLACE) == m.Status.UNSUPPORTED_SIZE
    assert h.value is None
    assert lib.mofft_plan_create_f64(ctypes.byref(h), 1, m.FORWARD,
                                     m.OUT_OF_PLACE) == m.Status.UNSUPPORTED_SIZE


@pytest.mark.parametrize("n", [256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536, 131072,
                               262144, 144, 169, 196, 225, 1728, 2197, 2744, 3375, 20736,
                               28561, 38416, 50625, 248832, 371293, 537824, 759375])
def test_extended_sizes_plan_and_match(n):
    """tests/test_fft.c:577-587 creates plans for these; here they also run
    against the oracle (one transform each, both precisions)."""
    x = oracle.uniform(n, seed=n, dtype=np.complex128)
    ref = oracle_ref(x, -1)
    assert rel_l2(run_host(x, -1, bits=32), ref) <= fp32_tol(n)
    assert rel_l2(run_host(x, -1, bits=64), ref) <= fp64_tol(n)


@pytest.mark.parametrize("n", [169, 196, 1024, 1728, 2197, 38416, 248832])
def test_roundtrip(n):
    """tests/test_fft.c:101-145: bwd(fwd(x))/n == x within 128*FLT_EPS*log2 n
    (FP32) and 512*DBL_EPS*log2 n (FP64)."""
    i = np.arange(n, dtype=np.float64)
    x = (np.sin(i * .017) + (i % 17) * .003) + 1j * (np.cos(i * .013) - (i % 13) * .002)
    for bits, tol in ((32, 128 * FLT_EPS), (64, 512 * DBL_EPS)):
        y = run_host(x, -1, bits=bits)
        z = run_host(y, 1, bits=bits) / n
        assert max_abs(z, x.astype(CTYPE[bits])) <= tol * max(1.0, np.log2(n)), bits


def test_specific_radix_chain():
    """tests/test_fft.c:147-195: chain {32, 8} agrees with the default plan."""
    n = 256
    i = np.arange(n)
    x = np.sin(.03 * i) + 1j * np.cos(.02 * i)
    for bits, tol in ((32, 64 * FLT_EPS * n), (64, 256 * DBL_EPS * n)):
        a = run_host(x, -1, bits=bits)
        b = run_host(x, -1, bits=bits, radices=[32, 8])
        assert max_abs(a, b) <= tol


RADICES = (2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32, 64)


@pytest.mark.parametrize("radix", RADICES)
def test_two_level_chains_every_radix(radix):
    """tests/test_fft.c:197-251 ({2, R}) and :408-487 ({13, R, 2}, forward vs
    the DFT and backward round trip) for every radix of the reference."""
    for chain in ([2, radix], [13, radix, 2]):
        n = int(np.prod(chain))
        i = np.arange(n)
        x = (np.sin(.13 * i) + .01 * (i % 3)) + 1j * (np.cos(.07 * i) - .02 * (i % 5))
        ref = oracle.dft_ld(x, -1)
        for bits, tol in ((32, 64 * FLT_EPS * n), (64, 256 * DBL_EPS * n)):
            for bank in (0, 1, 2, 3):
                y = run_host(x, -1, bits=bits, radices=chain, bank=bank)
                assert max_abs(y, ref) <= tol, (chain, bits, bank)
                z = run_host(y, 1, bits=bits, radices=chain, bank=bank) / n
                assert max_abs(z, x) <= (128 * FLT_EPS if bits == 32 else 512 * DBL_EPS) * \
                    radix * np.log2(n), (chain, bits, bank)


def test_layout_knobs_do_not_change_results():
    """tests/test_fft.c:253-406: blocked vs linear transposes are bit-identical
    and the SECTION layout matches TRANSPOSE; on the GPU these knobs keep the
    same device schedule, so the results are identical."""
    n = 4096
    i = np.arange(n)
    x = np.sin(.017 * i) + 1j * np.cos(.013 * i)
    for bits in (32, 64):
        for chain in ([16, 16, 16], [8, 16, 32], [8, 8, 64], [4, 4, 16, 16], [4] * 6):
            base = run_host(x, -1, bits=bits, radices=chain)
            lib = m.load()
            s = "f32" if bits == 32 else "f64"
            with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=bits, radices=chain) as p:
                assert getattr(lib, f"mofft_plan_set_direct_input_{s}")(p.handle, 0) == 0
                assert getattr(lib, f"mofft_plan_set_blocked_transpose_mask_{s}")(
                    p.handle, 1) == 0
                assert getattr(lib, f"mofft_plan_set_stage_layout_{s}")(p.handle, 1) == 0
                assert getattr(lib, f"mofft_plan_set_transpose_strategy_{s}")(p.handle, 1) == 0
                assert getattr(lib, f"mofft_plan_set_blocked_transpose_mask_{s}")(
                    p.handle, 1 << 10) == m.Status.INVALID_ARGUMENT
                y = np.empty_like(base)
                p.execute(np.ascontiguousarray(x, CTYPE[bits]), y)
            assert np.array_equal(y, base), (bits, chain)


# ------------------------------------------------------ test_binary_banks.c

BANK_SIZES = (121, 169, 196, 225, 256, 1024, 1728, 2197, 2744, 3375, 20736, 28561, 38416,
              50625, 65536, 248832, 262144, 371293, 537824, 759375)


@pytest.mark.parametrize("n", BANK_SIZES)
def test_three_mode_spectral_oracle(n):
    """tests/test_binary_banks.c: the analytic three-mode spectrum, every
    kernel bank, both signs and placements, tolerance 5e-5 / 2e-11."""
    x = three_mode_input(n)
    for bank in (0, 1, 2, 3):
        for sign in (-1, 1):
            want = three_mode_expected(n, sign)
            for inplace in (False, True):
                for bits, tol in ((32, 5e-5), (64, 2e-11)):
                    y = run_host(x, sign, bits=bits, inplace=inplace, bank=bank) / n
                    assert max_abs(y, want) <= tol, (bank, sign, inplace, bits)


@pytest.mark.parametrize("radix", RADICES)
def test_three_mode_single_and_double_radix(radix):
    """tests/test_binary_banks.c:65-73: chains {R} and {R, 2}."""
    for chain in ([radix], [radix, 2]):
        n = int(np.prod(chain))
        x = three_mode_input(n)
        for sign in (-1, 1):
            want = three_mode_expected(n, sign)
            for bank in (0, 1, 2, 3):
                for bits, tol in ((32, 5e-5), (64, 2e-11)):
                    y = run_host(x, sign, bits=bits, radices=chain, bank=bank) / n
                    assert max_abs(y, want) <= tol, (chain, sign, bank, bits)


# ------------------------------------------------------------ batched paths

def test_c1_forward_backward_device_buffers():
    """n=1024, batch=4096, out-of-place, uniform[-1,1) from seed 0: forward vs
    the oracle for every transform and backward(forward(x))/n vs x, with
    device (torch) buffers through the C-ABI."""
    import torch
    n, batch = 1024, 4096
    x = oracle.uniform(n * batch, seed=0, dtype=np.complex64).reshape(batch, n)
    ref = oracle.fft_ld(x.astype(np.complex128), -1)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty_like(dx)
    dz = torch.empty_like(dx)
    with m.Plan.create(n, m.FORWARD, bits=32, batch=batch) as f, \
            m.Plan.create(n, m.BACKWARD, bits=32, batch=batch) as b:
        f.execute(dx, dy)
        b.execute(dy, dz)
    torch.cuda.synchronize()
    y = dy.cpu().numpy()
    z = dz.cpu().numpy() / n
    assert rel_l2(y, ref) <= fp32_tol(n)
    per = np.linalg.norm(y - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert per.max() <= fp32_tol(n)
    assert rel_l2(z, x) <= fp32_tol(n)


def _sweep_case(n: int, bits: int, batch: int, direction: int, inplace: bool):
    x = oracle.uniform(n * batch, seed=n, dtype=CTYPE[bits]).reshape(batch, n)
    y = run_host(x, direction, bits=bits, inplace=inplace)
    rows = sorted({0, batch // 2, batch - 1})
    ref = np.stack([oracle_ref(x[r].astype(np.complex128), direction) for r in rows])
    err = rel_l2(y[rows], ref)
    assert err <= (fp32_tol(n) if bits == 32 else fp64_tol(n)), (n, bits, err)


SWEEP_POW2 = [2 ** e for e in range(4, 25)]
SWEEP_MIXED = [3 * 2 ** e for e in range(4, 19, 2)] + [5 * 2 ** e for e in range(4, 18, 2)]


@pytest.mark.parametrize("n", SWEEP_POW2 + SWEEP_MIXED)
def test_sweep_in_place_sampled(n):
    """The plain-method sweep (in place, both precisions, both directions) on
    a reduced batch; three transforms per call are checked against the
    oracle."""
    for bits in (32, 64):
        batch = max(1, min(64, (1 << 22) // n))
        for direction in (-1, 1):
            _sweep_case(n, bits, batch, direction, inplace=True)
    _sweep_case(n, 32, max(1, min(8, (1 << 20) // n)), -1, inplace=False)


def test_bench_config_rows_across_the_batch():
    """The default benchmark workload itself: n = 4096, batch 16384 (2^26
    points), in place, PRETUNED, device buffers, both directions.  Rows spread
    over the whole batch, and every row of the last 32 (the last CTAs of the
    launch), are checked against the long-double oracle."""
    import torch
    n, batch = 4096, 16384
    x = oracle.uniform(n * batch, seed=n, dtype=np.complex64).reshape(batch, n)
    rows = sorted(set(np.linspace(0, batch - 1, 64).astype(int).tolist()) |
                  set(range(batch - 32, batch)))
    d = torch.from_numpy(x).cuda()
    for direction in (m.FORWARD, m.BACKWARD):
        y = d.clone()
        with m.Plan.create(n, direction, m.IN_PLACE, bits=32, batch=batch) as plan:
            plan.execute(y, y)
        torch.cuda.synchronize()
        got = y[rows].cpu().numpy()
        ref = oracle.fft_ld(x[rows].astype(np.complex128), direction)
        assert rel_l2(got, ref) <= fp32_tol(n), direction
        per = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert per.max() <= fp32_tol(n), (direction, int(np.argmax(per)))


def test_every_specialised_kernel():
    """Each compiled one-pass kernel (every variant, selected by registry
    index) against the oracle, both directions, in and out of place, odd
    batch to exercise tail CTAs."""
    ks = [k for k in m.kernels() if k["kind"] == m.KERNEL_ROWS]
    for k in ks:
        n = k["length"]
        batch = 7
        x = oracle.uniform(n * batch, seed=99, dtype=CTYPE[k["precision_bits"]]).reshape(batch, n)
        tol = fp32_tol(n) if k["precision_bits"] == 32 else fp64_tol(n)
        for direction in (-1, 1):
            ref = oracle.fft_ld(x.astype(np.complex128), direction)
            for inplace in (False, True):
                y = run_host(x, direction, bits=k["precision_bits"], kernels=[k["index"]],
                             inplace=inplace)
                assert rel_l2(y, ref) <= tol, (k["name"], direction, inplace)


PREFETCH_KERNEL = "rows_float_16384_t512_b1_sfalse_dxp"


def test_prefetching_kernel_many_lines_per_cta():
    """The persistent kernel that bulk-copies each CTA's next line while it
    transforms the current one, with more lines than resident CTAs (every CTA
    runs 2-3 lines), both directions, in and out of place.  With an odd
    distance every other line start is not 16-byte aligned: those lines are
    loaded directly and the copies of the aligned ones still pair with their
    waits."""
    import torch
    k = next(k for k in m.kernels() if k["name"] == PREFETCH_KERNEL)
    n, batch = k["length"], 300
    for dist in (n, n + 1):
        buf = oracle.uniform(batch * dist, seed=dist, dtype=np.complex64)
        x = torch.from_numpy(buf).cuda()
        lines = buf.reshape(batch, dist)[:, :n].astype(np.complex128)
        for direction in (-1, 1):
            ref = oracle_ref(lines, direction)
            for inplace in (False, True):
                with m.Plan.create(n, direction, m.IN_PLACE if inplace else m.OUT_OF_PLACE,
                                   bits=32, batch=batch, distance=dist,
                                   kernels=[k["index"]]) as plan:
                    y = x.clone() if inplace else torch.zeros_like(x)
                    plan.execute(y if inplace else x, y)
                    plan.check_status()
                out = y.cpu().numpy().reshape(batch, dist)
                assert rel_l2(out[:, :n], ref) <= fp32_tol(n), (dist, direction, inplace)
                if dist > n and not inplace:
                    assert np.all(out[:, n:] == 0)      # gaps untouched


def test_prefetching_kernel_lost_copy_keeps_output():
    """Failure check of the prefetching kernel: no CTA's first line copy is
    issued, so every bounded wait runs out (about a second, no GPU fault).
    The plan reports MOFFT_INTERNAL_ERROR once, the CTAs load those lines
    themselves so the output is still the forward transform, and the plan
    then executes normally on the same context."""
    import time
    import torch
    lib = m.load()
    k = next(k for k in m.kernels() if k["name"] == PREFETCH_KERNEL)
    n, batch = k["length"], 300
    x = oracle.uniform(batch * n, seed=12, dtype=np.complex64).reshape(batch, n)
    ref = oracle_ref(x.astype(np.complex128), -1)
    d = torch.from_numpy(x).cuda()
    out = torch.zeros_like(d)
    with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=batch,
                       kernels=[k["index"]]) as plan:
        t0 = time.perf_counter()
        st = lib.mofft_plan_check_lost_copy_f32(plan.handle, d.data_ptr(), out.data_ptr())
        waited = time.perf_counter() - t0
        assert st == m.Status.INTERNAL_ERROR
        assert waited < 30.0, waited
        assert rel_l2(out.cpu().numpy(), ref) <= fp32_tol(n)
        plan.check_status()                       # the error word was cleared
        out.zero_()
        plan.execute(d, out)
    assert rel_l2(out.cpu().numpy(), ref) <= fp32_tol(n)


def test_batch_distance_and_stream():
    """distance > length leaves the gaps untouched; an attached stream makes
    execute asynchronous on that stream."""
    import torch
    n, batch, dist = 256, 33, 300
    buf = oracle.uniform(batch * dist, seed=5, dtype=np.complex64)
    x = torch.from_numpy(buf).cuda()
    y = torch.full_like(x, 7 + 7j)
    lib = m.load()
    h = ctypes.c_void_p()
    opts = m.PlanOptions(0, 0, 0, 0)
    assert lib.mofft_plan_create_batched_f32(ctypes.byref(h), n, batch, dist, m.FORWARD,
                                             m.OUT_OF_PLACE, ctypes.byref(opts), None) == 0
    plan = m.Plan(h.value, 32)
    s = torch.cuda.Stream()
    plan.set_stream(s.cuda_stream)
    with torch.cuda.stream(s):
        plan.execute(x, y)
    s.synchronize()
    out = y.cpu().numpy().reshape(batch, dist)
    assert np.all(out[:, n:] == np.complex64(7 + 7j))
    ref = oracle.fft_ld(buf.reshape(batch, dist)[:, :n].astype(np.complex128), -1)
    assert rel_l2(out[:, :n], ref) <= fp32_tol(n)
    plan.destroy()


def test_torch_convenience_matches_oracle():
    import torch
    x = torch.from_numpy(oracle.uniform(64 * 512, seed=1, dtype=np.complex128)).reshape(64, 512)
    y = m.fft(x.cuda(), m.FORWARD)
    torch.cuda.synchronize()
    assert rel_l2(y.cpu().numpy(), oracle.fft_ld(x.numpy(), -1)) <= fp64_tol(512)


def _cols_partners(k, ks):
    """Two-pass schedules (kernel indices) that run column kernel k, once as
    the first pass and once as the second where some partner allows it."""
    out = []
    same = [p for p in ks if p["precision_bits"] == k["precision_bits"]]
    for first in (True, False):
        for p in sorted(same, key=lambda q: q["length"]):
            pair = [k, p] if first else [p, k]
            n = pair[0]["length"] * pair[1]["length"]
            if n > (1 << 20):
                continue
            try:
                with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=k["precision_bits"],
                                   kernels=[q["index"] for q in pair]):
                    pass
            except m.MofftError:
                continue
            out.append((n, [q["index"] for q in pair]))
            break
    return out


def test_every_column_kernel():
    """Each compiled column-pass kernel (every variant, selected by registry
    index) inside two-pass plans -- as the first pass and as the second --
    against the oracle, both directions, odd batch."""
    ks = [k for k in m.kernels() if k["kind"] == m.KERNEL_COLS]
    missing = []
    for k in ks:
        cases = _cols_partners(k, ks)
        if not cases:
            missing.append(k["name"])
            continue
        for n, kernels in cases:
            batch = 3
            x = oracle.uniform(n * batch, seed=n, dtype=CTYPE[k["precision_bits"]]).reshape(batch, n)
            tol = fp32_tol(n) if k["precision_bits"] == 32 else fp64_tol(n)
            for direction in (-1, 1):
                y = run_host(x, direction, bits=k["precision_bits"], kernels=kernels)
                ref = oracle.fft_ld(x.astype(np.complex128), direction)
                assert rel_l2(y, ref) <= tol, (k["name"], n, kernels)
    assert not missing, missing
