"""Serving loop (include/mofft_serve.h): results of a request mix against
the oracle, each result bit-identical alone and in the mix, coalescing into
fewer launches than requests, host and device buffers, admission cap."""
from __future__ import annotations

import numpy as np
import pytest

import mofft_b200 as m
import oracle
from tests.conftest import cuda_available, fp32_tol, fp64_tol, rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _tensor(batch, n, bits, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    dt = torch.float32 if bits == 32 else torch.float64
    return torch.view_as_complex(torch.rand((batch, n, 2), generator=g, device="cuda",
                                            dtype=dt) * 2 - 1)


def test_mix_matches_oracle_host_and_device():
    import torch
    srv = m.Server(streams=4)
    reqs = []
    rng = np.random.default_rng(0)
    for k in range(48):
        n = int(2 ** rng.integers(8, 21))
        bits = 32 if k % 5 else 64
        batch = int(rng.integers(1, 4))
        d = -1 if k % 2 else 1
        x = _tensor(batch, n, bits, k)
        if k % 3 == 0:      # host (pinned) buffers
            hx = x.cpu().pin_memory()
            hy = torch.empty_like(hx).pin_memory()
            t = srv.submit(n, batch, d, bits, hx.data_ptr(), hy.data_ptr())
            reqs.append((t, x, hy, d, n, bits, hx))     # inputs must outlive the request
        elif k % 3 == 1:    # device, in place
            y = x.clone()
            t = srv.submit(n, batch, d, bits, y.data_ptr(), y.data_ptr())
            reqs.append((t, x, y, d, n, bits, None))
        else:               # device, out of place
            y = torch.empty_like(x)
            t = srv.submit(n, batch, d, bits, x.data_ptr(), y.data_ptr())
            reqs.append((t, x, y, d, n, bits, None))
    for t, x, y, d, n, bits, _ in reqs:
        st, lat = srv.wait(t)
        assert st == 0 and lat > 0
        torch.cuda.synchronize()
        got = y.cpu().numpy()
        ref = oracle.fft_ld(x.cpu().numpy().astype(np.complex128), d)
        tol = fp32_tol(n) if bits == 32 else fp64_tol(n)
        assert rel_l2(got, ref) <= tol, (n, bits, d)
        for b in range(got.shape[0]):   # every transform of the request
            assert rel_l2(got[b], ref[b]) <= tol, (n, bits, d, b)
    stats = srv.stats()
    assert stats["completed"] == 48 and stats["failed"] == 0
    srv.destroy()


@pytest.mark.parametrize("n", [1024, 65536])
def test_alone_equals_mix_and_coalesces(n):
    import torch
    x = _tensor(3, n, 32, 7)
    alone_out = torch.empty_like(x)
    srv = m.Server(streams=2)
    st, _ = srv.wait(srv.submit(n, 3, -1, 32, x.data_ptr(), alone_out.data_ptr()))
    assert st == 0
    srv.destroy()
    # the same request in a mix of 64 same-length requests submitted together
    srv = m.Server(streams=1)
    others = [(_tensor(2, n, 32, 100 + k), None) for k in range(64)]
    outs = [torch.empty_like(o) for o, _ in others]
    tickets = []
    for k, ((o, _), out) in enumerate(zip(others, outs)):
        if k == 20:
            mix_out = torch.empty_like(x)
            tickets.append(srv.submit(n, 3, -1, 32, x.data_ptr(), mix_out.data_ptr()))
        tickets.append(srv.submit(n, 2, -1, 32, o.data_ptr(), out.data_ptr()))
    for t in tickets:
        assert srv.wait(t)[0] == 0
    torch.cuda.synchronize()
    assert torch.equal(alone_out, mix_out)
    stats = srv.stats()
    assert stats["launches"] < len(tickets)       # requests were coalesced
    srv.destroy()


def test_alone_equals_mix_mixed_lengths_and_precisions():
    """Each request of a stream that mixes lengths (one-pass and two-pass),
    precisions, directions and host / device buffers gives bit-identical
    results alone (the only request on the server) and in the mix, where
    same-shape requests are coalesced into pointer-table launches and groups
    of different shapes overlap on several streams."""
    import torch
    shapes = [(256, 32, -1), (1024, 64, 1), (4096, 32, -1), (65536, 32, -1),
              (1 << 20, 32, 1), (512, 64, -1), (16384, 64, 1), (3 * 1024, 32, 1)]
    probes = []
    for k, (n, bits, d) in enumerate(shapes):
        batch = 1 + k % 3
        probes.append((n, bits, d, batch, _tensor(batch, n, bits, 500 + k), k % 4 == 3))

    def submit(srv, n, bits, d, batch, x, host, keep):
        if host:
            hx = x.cpu().pin_memory()
            hy = torch.empty_like(hx).pin_memory()
            keep.append(hx)
            return srv.submit(n, batch, d, bits, hx.data_ptr(), hy.data_ptr()), hy
        y = torch.empty_like(x)
        return srv.submit(n, batch, d, bits, x.data_ptr(), y.data_ptr()), y

    alone = []
    srv = m.Server(streams=2)
    keep = []
    for n, bits, d, batch, x, host in probes:
        t, y = submit(srv, n, bits, d, batch, x, host, keep)
        assert srv.wait(t)[0] == 0
        torch.cuda.synchronize()
        alone.append(y.cpu().clone())
    srv.destroy()

    srv = m.Server(streams=4)
    tickets, mixed = [], {}
    fillers = []
    for rep in range(3):
        for k, (n, bits, d, batch, x, host) in enumerate(probes):
            if rep == 1:
                mixed[k] = submit(srv, n, bits, d, batch, x, host, keep)
                tickets.append(mixed[k][0])
            fb = 1 + (rep + k) % 4
            fx = _tensor(fb, n, bits, 900 + 10 * rep + k)
            t, fy = submit(srv, n, bits, d, fb, fx, False, keep)
            fillers.append((fx, fy))
            tickets.append(t)
    for t in tickets:
        assert srv.wait(t)[0] == 0
    torch.cuda.synchronize()
    for k, (n, bits, d, batch, x, host) in enumerate(probes):
        got = mixed[k][1].cpu()
        assert torch.equal(got, alone[k]), (n, bits, d, host)
        ref = oracle.fft_ld(x.cpu().numpy().astype(np.complex128), d)
        tol = fp32_tol(n) if bits == 32 else fp64_tol(n)
        assert rel_l2(got.numpy(), ref) <= tol, (n, bits, d)
    assert srv.stats()["launches"] < len(tickets)
    srv.destroy()


def test_admission_cap():
    import torch
    n, batch = 4096, 64
    x = _tensor(batch, n, 32, 3)
    y = torch.empty_like(x)
    payload = 2 * batch * n * 8
    srv = m.Server(hbm_budget_bytes=payload)        # room for exactly one request
    small = [srv.submit(n, batch, -1, 32, x.data_ptr(), y.data_ptr()) for _ in range(4)]
    for t in small:
        assert srv.wait(t)[0] == 0
    big = _tensor(2 * batch, n, 32, 4)
    t = srv.submit(n, 2 * batch, -1, 32, big.data_ptr(), big.data_ptr())
    assert srv.wait(t)[0] == m.Status.ALLOCATION_FAILURE
    assert srv.stats()["peak_admitted_bytes"] <= payload
    with pytest.raises(m.MofftError):
        srv.submit(17 * 16, 1, -1, 32, x.data_ptr(), y.data_ptr())
    srv.destroy()


def test_lengths_on_runtime_stage_kernels():
    """A length without a specialised kernel (7 * 64 = 448, 11 * 1024 = 11264)
    runs on the runtime-stage kernels, which take no pointer tables: several
    such requests waiting together still complete correctly (one plain
    launch each), on host and on device buffers."""
    import torch
    srv = m.Server(streams=2)
    reqs = []
    for k, (n, bits) in enumerate([(448, 32), (448, 32), (11264, 64), (11264, 64), (448, 64)]):
        x = _tensor(3, n, bits, 100 + k)
        if k % 2:
            hx = x.cpu().pin_memory()
            hy = torch.empty_like(hx).pin_memory()
            reqs.append((srv.submit(n, 3, -1, bits, hx.data_ptr(), hy.data_ptr()), x, hy, n,
                         bits, hx))
        else:
            y = torch.empty_like(x)
            reqs.append((srv.submit(n, 3, -1, bits, x.data_ptr(), y.data_ptr()), x, y, n,
                         bits, None))
    for t, x, y, n, bits, _ in reqs:
        st, _lat = srv.wait(t)
        assert st == 0, (n, bits)
        torch.cuda.synchronize()
        ref = oracle.fft_ld(x.cpu().numpy().astype(np.complex128), -1)
        assert rel_l2(y.cpu().numpy(), ref) <= (fp32_tol(n) if bits == 32 else fp64_tol(n))
    srv.destroy()
