"""The oracle (CPU restatement of the reference transform) pinned to the
reference's own codelet evaluator, its C tests' direct-DFT cases, its analytic
three-mode test, a long double direct DFT and numpy's pocketfft."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tests.conftest import (DBL_EPS, FLT_EPS, max_abs, rel_l2, three_mode_expected,
                            three_mode_input)

RADICES = (2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32, 64)


def test_codelet_golden_vectors(golden_codelets):
    """Single-stage oracle == reference evaluate_pattern for every radix and
    rewrite family (tolerance of compiler/mofft_compiler/validate.py:160)."""
    checked = 0
    for key in golden_codelets.files:
        if not key.endswith("_in"):
            continue
        stem = key[:-3]
        radix = int(stem.split("_")[0][1:])
        sign = -1 if "_forward_" in stem else 1
        x = golden_codelets[key]
        want = golden_codelets[stem + "_out"]
        got = oracle.fft_ld(x, sign, factors=[radix])
        assert max_abs(got, want) <= 192 * DBL_EPS * radix, stem
        checked += 1
    assert checked >= 2 * len(RADICES) * 2


def test_transform_golden_vectors(golden_transforms):
    """Sizes and inputs of tests/test_fft.c:489-573, tolerance 96*DBL_EPS*n."""
    keys = [k for k in golden_transforms.files if k.startswith("fft_") and k.endswith("_in")]
    assert len(keys) == 42
    for key in keys:
        _, n, d, _ = key.split("_")
        n, d = int(n), int(d)
        x = golden_transforms[key]
        want = golden_transforms[key.replace("_in", "_out")]
        got = oracle.fft_ld(x, d)
        assert max_abs(got, want) <= 96 * DBL_EPS * n, (n, d)


def test_planning_and_recipe_golden_vectors(golden_transforms):
    for prefix in ("planning_30", "recipe_64", "recipe_96"):
        for d in (-1, 1):
            x = golden_transforms[f"{prefix}_{d}_in"]
            want = golden_transforms[f"{prefix}_{d}_out"]
            n = len(x)
            assert max_abs(oracle.fft_ld(x, d), want) <= 2e-11 * n


@pytest.mark.parametrize("n", [121, 169, 196, 225, 256, 1024, 1728, 2197, 2744, 3375,
                               20736, 28561])
def test_three_mode_known_answer(n):
    """tests/test_binary_banks.c: X/n has 0.25 at 0, 1 at +-3 and 0.5 at -+5."""
    x = three_mode_input(n)
    for sign in (-1, 1):
        got = oracle.fft_ld(x, sign) / n
        assert max_abs(got, three_mode_expected(n, sign)) <= 2e-11


@pytest.mark.parametrize("n", [2, 3, 5, 7, 11, 13, 30, 60, 96, 144, 225, 256, 1000, 1024])
def test_matches_direct_dft_and_numpy(n):
    x = oracle.uniform(n, seed=n, dtype=np.complex128)
    for sign in (-1, 1):
        got = oracle.fft_ld(x, sign)
        direct = oracle.dft_ld(x, sign)
        ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
        assert rel_l2(got, direct) <= 1e-17 * n + 4e-16
        assert rel_l2(got, ref) <= 5e-15


def test_explicit_chains_agree():
    """tests/test_fft.c:147-195: an explicit {32, 8} chain equals the default."""
    x = oracle.uniform(256, seed=3, dtype=np.complex128)
    a = oracle.fft_ld(x, -1)
    b = oracle.fft_ld(x, -1, factors=[32, 8])
    c = oracle.fft_ld(x, -1, factors=[2, 4, 2, 16])
    assert max_abs(a, b) <= 64 * DBL_EPS * 256
    assert max_abs(a, c) <= 64 * DBL_EPS * 256


def test_unsupported_lengths():
    with pytest.raises(ValueError):
        oracle.plan_factors(17)
    with pytest.raises(ValueError):
        oracle.plan_factors(1)
    assert np.prod(oracle.plan_factors(759375)) == 759375


@pytest.mark.parametrize("n", [1024, 4096, 3 * 1024, 5 * 512])
def test_port_precision(n):
    """The float/double ports (the timed CPU baseline) meet the FP32/FP64
    tolerances against the long double oracle."""
    x = oracle.uniform(4 * n, seed=11, dtype=np.complex128).reshape(4, n)
    ref = oracle.fft_ld(x, -1)
    y32 = oracle.fft_port(x.astype(np.complex64), -1, threads=2)
    y64 = oracle.fft_port(x, -1, threads=2)
    assert rel_l2(y32, ref) <= 5e-7 * np.log2(n)
    assert rel_l2(y64, ref) <= 2e-15 * np.log2(n)


def test_roundtrip_fixture(golden_transforms):
    for n in (169, 196):
        x = golden_transforms[f"roundtrip_{n}_in"]
        y = oracle.fft_ld(x, -1)
        assert max_abs(y, golden_transforms[f"roundtrip_{n}_fwd"]) <= 96 * DBL_EPS * n
        z = oracle.fft_ld(y, 1) / n
        assert max_abs(z, x) <= 512 * DBL_EPS * np.log2(n)


def test_uniform_generator_is_seeded():
    a = oracle.uniform(1000, 7)
    b = oracle.uniform(1000, 7)
    c = oracle.uniform(1000, 8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.real.min() >= -1 and a.real.max() < 1
    assert abs(a.real.mean()) < 0.1 and abs(a.imag.mean()) < 0.1
    assert FLT_EPS > 0
