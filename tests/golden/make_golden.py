"""Generate the golden fixtures that pin the oracle and the codelets.

Run once in a checkout that has the reference at /root/reference:

    python tests/golden/make_golden.py /root/reference

Fixtures (written next to this script):

codelets.npz
    For every radix of the reference (2..16, 32, 64), both directions and
    every algebraic rewrite pattern the reference defines for that radix
    (compiler/mofft_compiler/rewrites.py:25-41), seeded inputs and the outputs
    of the reference's own evaluator ``evaluate_pattern``
    (compiler/mofft_compiler/rewrites.py:43-95), imported from the reference
    checkout.  Inputs follow tests/test_compiler.py:37-49 (random.Random(8137),
    uniform parts in [-1, 1)).

transforms.npz
    Whole-transform cases built from the reference's C tests: the input
    formulas of tests/test_fft.c:17-18 (sizes of tests/test_fft.c:490-491),
    tests/test_planning.c:11-23 (n = 30), tests/test_plan_recipe.c:93-96
    (n = 64, 96) and tests/test_fft.c:111-112 (roundtrip inputs), each with the
    expected output computed exactly as those tests compute their reference:
    a direct DFT in double with angle = dir*2*pi*j*k/n
    (tests/test_fft.c:20-26).
"""
from __future__ import annotations

import math
import random
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
RADICES = (2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32, 64)


def direct_dft_like_reference_tests(x: np.ndarray, direction: int) -> np.ndarray:
    """tests/test_fft.c:20-26: double accumulation, cos/sin of the full angle."""
    n = len(x)
    out = np.zeros(n, dtype=np.complex128)
    for k in range(n):
        rr = 0.0
        ii = 0.0
        for j in range(n):
            angle = direction * 2.0 * math.pi * j * k / n
            c, s = math.cos(angle), math.sin(angle)
            rr += x[j].real * c - x[j].imag * s
            ii += x[j].real * s + x[j].imag * c
        out[k] = complex(rr, ii)
    return out


def codelets(reference: Path) -> dict:
    sys.path.insert(0, str(reference / "compiler"))
    from mofft_compiler.rewrites import algebraic_patterns, evaluate_pattern
    data = {}
    rng = random.Random(8137)
    for radix in RADICES:
        for direction in ("forward", "backward"):
            for pattern in algebraic_patterns(radix):
                values = [complex(rng.uniform(-1, 1), rng.uniform(-1, 1)) for _ in range(radix)]
                outputs = evaluate_pattern(values, direction, pattern)
                key = f"r{radix}_{direction}_{pattern.value}"
                data[key + "_in"] = np.array(values, dtype=np.complex128)
                data[key + "_out"] = np.array(outputs, dtype=np.complex128)
    return data


def transforms() -> dict:
    data = {}
    sizes = (2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32, 45, 64, 144, 225, 256)
    for n in sizes:
        i = np.arange(n, dtype=np.float64)
        x = (np.sin(i * 0.17) + (i % 7) * 0.03) + 1j * (np.cos(i * 0.11) - (i % 5) * 0.02)
        for d in (-1, 1):
            data[f"fft_{n}_{d}_in"] = x
            data[f"fft_{n}_{d}_out"] = direct_dft_like_reference_tests(x, d)
    n = 30
    i = np.arange(n, dtype=np.float64)
    x = (np.sin(i * 0.31) + (i % 5) * 0.07) + 1j * (np.cos(i * 0.23) - (i % 7) * 0.03)
    for d in (-1, 1):
        data[f"planning_{n}_{d}_in"] = x
        data[f"planning_{n}_{d}_out"] = direct_dft_like_reference_tests(x, d)
    for n in (64, 96):
        i = np.arange(n, dtype=np.float64)
        x = (0.2 + np.sin(i * 7 + 3) * 0.7) + 1j * (np.cos(i * 5 + 1) * 0.4 - 0.1)
        for d in (-1, 1):
            data[f"recipe_{n}_{d}_in"] = x
            data[f"recipe_{n}_{d}_out"] = direct_dft_like_reference_tests(x, d)
    for n in (169, 196):
        i = np.arange(n, dtype=np.float64)
        x = (np.sin(i * 0.017) + (i % 17) * 0.003) + 1j * (np.cos(i * 0.013) - (i % 13) * 0.002)
        data[f"roundtrip_{n}_in"] = x
        data[f"roundtrip_{n}_fwd"] = direct_dft_like_reference_tests(x, -1)
    return data


def main(argv: list[str]) -> int:
    reference = Path(argv[1]) if len(argv) > 1 else Path("/root/reference")
    np.savez_compressed(HERE / "codelets.npz", **codelets(reference))
    np.savez_compressed(HERE / "transforms.npz", **transforms())
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
