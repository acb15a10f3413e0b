"""Shared test setup: repository imports, the `gpu` marker, helpers."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"
FLT_EPS = float(np.finfo(np.float32).eps)
DBL_EPS = float(np.finfo(np.float64).eps)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden_codelets():
    return np.load(GOLDEN / "codelets.npz")


@pytest.fixture(scope="session")
def golden_transforms():
    return np.load(GOLDEN / "transforms.npz")


def max_abs(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a, np.complex128) - np.asarray(b, np.complex128))))


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d else 1.0))


def fp32_tol(n: int) -> float:
    """Relative L2 bound for FP32 results: 5e-7 * log2(n)."""
    return 5e-7 * max(1.0, np.log2(n))


def fp64_tol(n: int) -> float:
    """Relative L2 bound for FP64 results: 2e-15 * log2(n)."""
    return 2e-15 * max(1.0, np.log2(n))


def three_mode_input(n: int) -> np.ndarray:
    """tests/test_binary_banks.c:17-21: x_j = 0.25 + e^{2 pi i 3j/n} + 0.5 e^{-2 pi i 5j/n}."""
    j = np.arange(n, dtype=np.float64)
    a = 2 * np.pi * 3 * j / n
    b = 2 * np.pi * 5 * j / n
    return (0.25 + np.cos(a) + 0.5 * np.cos(b)) + 1j * (np.sin(a) - 0.5 * np.sin(b))


def three_mode_expected(n: int, sign: int) -> np.ndarray:
    """Spectrum / n of three_mode_input (tests/test_binary_banks.c:33-37)."""
    e = np.zeros(n, dtype=np.complex128)
    e[0] += 0.25
    e[(3 % n) if sign < 0 else (n - 3 % n) % n] += 1.0
    e[((n - 5 % n) % n) if sign < 0 else (5 % n)] += 0.5
    return e
