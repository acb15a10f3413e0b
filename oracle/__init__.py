"""ORACLE -- test infrastructure only.

Python binding of ``oracle/liboracle.so``, the CPU restatement of the
reference transform (see ``oracle.c`` for what it restates and where).  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
it, always as the checker or as the timed CPU baseline, never as the product.

Parity is pinned by ``tests/test_oracle.py`` against the golden fixtures in
``tests/golden/`` (the reference's own codelet evaluator and its C tests'
input formulas, generated by ``tests/golden/make_golden.py``), the
reference's analytic three-mode test, a direct DFT and numpy's pocketfft.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
LIB_PATH = _DIR / "liboracle.so"
_lib = None
_P = ctypes.c_void_p
_SZ = ctypes.c_size_t


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} missing: run `python -m mofft_b200.build`")
        lib = ctypes.CDLL(str(LIB_PATH))
        lib.oracle_plan_factors.argtypes = [_SZ, ctypes.POINTER(ctypes.c_int)]
        lib.oracle_plan_factors.restype = ctypes.c_int
        for name in ("oracle_fft_ld_batch", "oracle_fft_f32_batch", "oracle_fft_f64_batch"):
            fn = getattr(lib, name)
            fn.argtypes = [_P, _P, _SZ, _SZ, _SZ, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                           ctypes.c_int, ctypes.c_int]
            fn.restype = ctypes.c_int
        lib.oracle_dft_ld.argtypes = [_P, _P, _SZ, ctypes.c_int]
        lib.oracle_dft_ld.restype = ctypes.c_int
        lib.oracle_fill_uniform_f64.argtypes = [_P, _SZ, ctypes.c_uint64]
        lib.oracle_fill_uniform_f32.argtypes = [_P, _SZ, ctypes.c_uint64]
        _lib = lib
    return _lib


def plan_factors(n: int) -> list[int]:
    f = (ctypes.c_int * 64)()
    d = load().oracle_plan_factors(n, f)
    if d <= 0:
        raise ValueError(f"unsupported length {n}")
    return list(f[:d])


def _factor_args(factors):
    if factors is None:
        return None, 0
    arr = (ctypes.c_int * len(factors))(*factors)
    return arr, len(factors)


def fft_ld(x: np.ndarray, direction: int = -1, factors=None, threads: int = 0) -> np.ndarray:
    """long double oracle of shape (..., n) complex input; returns complex128."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    n = x.shape[-1]
    batch = x.size // n
    out = np.empty_like(x)
    f, d = _factor_args(factors)
    threads = threads or min(os.cpu_count() or 1, max(1, batch))
    r = load().oracle_fft_ld_batch(x.ctypes.data, out.ctypes.data, n, batch, n, direction, f, d,
                                   threads)
    if r <= 0:
        raise ValueError(f"oracle failed ({r}) for n={n}")
    return out


def fft_port(x: np.ndarray, direction: int = -1, factors=None, threads: int = 1) -> np.ndarray:
    """Reference-precision port (complex64 -> FP32 arithmetic, complex128 -> FP64)."""
    if x.dtype == np.complex64:
        fn = load().oracle_fft_f32_batch
    elif x.dtype == np.complex128:
        fn = load().oracle_fft_f64_batch
    else:
        raise TypeError("complex64 or complex128 required")
    x = np.ascontiguousarray(x)
    n = x.shape[-1]
    out = np.empty_like(x)
    f, d = _factor_args(factors)
    r = fn(x.ctypes.data, out.ctypes.data, n, x.size // n, n, direction, f, d, threads)
    if r <= 0:
        raise ValueError(f"port failed ({r}) for n={n}")
    return out


def dft_ld(x: np.ndarray, direction: int = -1) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    if load().oracle_dft_ld(x.ctypes.data, out.ctypes.data, x.shape[-1], direction) != 0:
        raise ValueError("dft failed")
    return out


def uniform(points: int, seed: int, dtype=np.complex64) -> np.ndarray:
    """splitmix64 uniform[-1,1) complex values, real then imaginary per point."""
    if dtype == np.complex64:
        out = np.empty(points, dtype=np.complex64)
        load().oracle_fill_uniform_f32(out.ctypes.data, points, seed)
    else:
        out = np.empty(points, dtype=np.complex128)
        load().oracle_fill_uniform_f64(out.ctypes.data, points, seed)
    return out


def rel_l2(y: np.ndarray, ref: np.ndarray) -> float:
    y = y.astype(np.complex128).ravel()
    ref = ref.astype(np.complex128).ravel()
    den = np.linalg.norm(ref)
    return float(np.linalg.norm(y - ref) / (den if den > 0 else 1.0))
