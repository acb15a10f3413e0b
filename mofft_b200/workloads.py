"""Seeded synthetic workloads of the benchmark configurations.

ragged_spec      512 transforms, n uniform over {2^6..2^16} U {3*2^k, k=5..13}
                 (values spaced evenly in log2 n), batch uniform in 1..64,
                 direction forward/backward with probability 1/2, seed 7.
serving_stream   requests with Poisson arrivals: n Zipf(s=1.1) over the powers
                 of two 2^8..2^20, batch uniform in 1..256, 80 % FP32 /
                 20 % FP64, direction +-1, seeded.
precision_mix    FP32 inputs that are a 1/3 mix of uniform[-1,1), log-uniform
                 magnitudes 1e-3..1e3 with uniform phase, and unit-amplitude
                 single tones at random bins.
"""
from __future__ import annotations

import numpy as np

RAGGED_LENGTHS = sorted([2 ** e for e in range(6, 17)] + [3 * 2 ** k for k in range(5, 14)])
SERVING_LENGTHS = [2 ** e for e in range(8, 21)]


def ragged_spec(count: int = 512, seed: int = 7, max_batch: int = 64,
                lengths=None) -> list[tuple[int, int, int]]:
    """[(n, batch, direction)] of the ragged-batching workload."""
    rng = np.random.default_rng(seed)
    lengths = RAGGED_LENGTHS if lengths is None else lengths
    n = rng.choice(lengths, size=count)
    batch = rng.integers(1, max_batch + 1, size=count)
    direction = np.where(rng.random(count) < 0.5, -1, 1)
    return [(int(a), int(b), int(c)) for a, b, c in zip(n, batch, direction)]


def serving_stream(count: int, rate_per_s: float, seed: int = 11,
                   max_batch: int = 256) -> list[dict]:
    """Requests sorted by arrival time (seconds from 0)."""
    rng = np.random.default_rng(seed)
    ranks = np.arange(1, len(SERVING_LENGTHS) + 1, dtype=np.float64)
    weights = ranks ** -1.1
    weights /= weights.sum()
    idx = rng.choice(len(SERVING_LENGTHS), size=count, p=weights)
    batch = rng.integers(1, max_batch + 1, size=count)
    bits = np.where(rng.random(count) < 0.8, 32, 64)
    direction = np.where(rng.random(count) < 0.5, -1, 1)
    arrivals = np.cumsum(rng.exponential(1.0 / rate_per_s, size=count))
    return [{"n": SERVING_LENGTHS[i], "batch": int(b), "bits": int(p), "direction": int(d),
             "arrival": float(t)}
            for i, b, p, d, t in zip(idx, batch, bits, direction, arrivals)]


def precision_mix(points: int, n: int, seed: int = 3) -> np.ndarray:
    """complex64 array of `points` values, (points // n) transforms of n."""
    rng = np.random.default_rng(seed)
    batch = points // n
    out = np.empty((batch, n), dtype=np.complex64)
    third = batch // 3
    u = rng.uniform(-1, 1, size=(third, n, 2))
    out[:third] = (u[..., 0] + 1j * u[..., 1]).astype(np.complex64)
    m = batch - third
    half = third + (m // 2)
    mag = 10.0 ** rng.uniform(-3, 3, size=(half - third, n))
    ph = rng.uniform(0, 2 * np.pi, size=(half - third, n))
    out[third:half] = (mag * np.exp(1j * ph)).astype(np.complex64)
    bins = rng.integers(0, n, size=batch - half)
    j = np.arange(n)
    out[half:] = np.exp(2j * np.pi * np.outer(bins, j) / n).astype(np.complex64)
    return out


def precision_mix_device(points: int, n: int, seed: int = 3, device: str = "cuda"):
    """The precision mix generated on the GPU with torch (same three classes
    and proportions as precision_mix, a different random stream): a
    (points // n, n) complex64 tensor."""
    import math

    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    batch = points // n
    out = torch.empty((batch, n), dtype=torch.complex64, device=device)
    third = batch // 3
    half = third + (batch - third) // 2
    u = torch.rand((third, n, 2), generator=g, device=device) * 2 - 1
    out[:third] = torch.view_as_complex(u.contiguous())
    del u
    mag = 10.0 ** (torch.rand((half - third, n), generator=g, device=device,
                              dtype=torch.float64) * 6 - 3)
    ph = torch.rand((half - third, n), generator=g, device=device,
                    dtype=torch.float64) * (2 * math.pi)
    out[third:half] = torch.polar(mag, ph).to(torch.complex64)
    del mag, ph
    bins = torch.randint(0, n, (batch - half, 1), generator=g, device=device)
    j = torch.arange(n, device=device).unsqueeze(0)
    turns = ((bins * j) % n).to(torch.float64) / n   # exact reduction of bin * j / n
    out[half:] = torch.polar(torch.ones_like(turns), turns * (2 * math.pi)).to(torch.complex64)
    return out
