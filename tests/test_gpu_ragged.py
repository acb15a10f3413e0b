"""Ragged batches in one CUDA graph (one-pass lengths as tiles of one
persistent launch over a work-descriptor queue, longer ones as tuned groups
through pointer tables; or every item in the persistent launch): every item
against the oracle, bit-identical repeats, each item the same alone and in
the mix, and the per-item comparison path."""
from __future__ import annotations

import numpy as np
import pytest

import mofft_b200 as m
import oracle
from mofft_b200 import workloads
from tests.conftest import cuda_available, fp32_tol, rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def make_items(spec, seed=0, inplace=lambda k: False):
    """(source, output, direction, pristine input) per item; in-place items
    have source is output."""
    import torch
    gen = torch.Generator(device="cuda").manual_seed(seed)
    items = []
    for k, (n, batch, direction) in enumerate(spec):
        x = torch.view_as_complex(torch.rand((batch, n, 2), generator=gen, device="cuda") * 2 - 1)
        if inplace(k):
            y = x.clone()
            items.append((y, y, direction, x))
        else:
            items.append((x, torch.empty_like(x), direction, x.clone()))
    return items


@pytest.mark.parametrize("single_launch", [False, True])
def test_ragged_matches_oracle_and_repeats(single_launch):
    import torch
    # every length of the workload at least once, small batches
    spec = [(n, 1 + (k % 5), -1 if k % 2 else 1) for k, n in enumerate(workloads.RAGGED_LENGTHS)]
    spec += workloads.ragged_spec(count=24, seed=5, max_batch=6)
    items = make_items(spec, inplace=lambda k: k % 3 == 1)
    plan = m.RaggedPlan([(a, b, d) for a, b, d, _ in items], single_launch=single_launch)
    tiles, grid = plan.info()
    assert tiles > 0 and grid > 0
    before = m.launch_count()
    plan.execute()
    launches = m.launch_count() - before
    # one persistent launch, plus one launch per pass of every tuned group
    assert launches == 1 if single_launch else launches > 1
    torch.cuda.synchronize()
    assert plan.status() == 0
    first = [b.clone() for _, b, _, _ in items]
    for (src, out, direction, orig), got in zip(items, first):
        x = orig.cpu().numpy()
        ref = oracle.fft_ld(x.astype(np.complex128), direction)
        n = x.shape[-1]
        assert rel_l2(got.cpu().numpy(), ref) <= fp32_tol(n), (n, direction)
    # repeat (graph replay): restore in-place inputs, results bit-identical
    for src, out, direction, orig in items:
        if src.data_ptr() == out.data_ptr():
            out.copy_(orig)
    plan.execute()
    torch.cuda.synchronize()
    assert plan.status() == 0
    for (_, out, _, _), got in zip(items, first):
        assert torch.equal(out, got)
    plan.destroy()


def test_item_alone_equals_item_in_mix():
    import torch
    spec = workloads.ragged_spec(count=40, seed=9, max_batch=4)
    items = make_items(spec, seed=1)
    mix = m.RaggedPlan([(a, b, d) for a, b, d, _ in items])
    mix.execute()
    torch.cuda.synchronize()
    assert mix.status() == 0
    for k in (0, 7, 19, 39):
        _, y_mix, direction, x = items[k]
        y_alone = torch.empty_like(x)
        alone = m.RaggedPlan([(x, y_alone, direction)])
        alone.execute()
        torch.cuda.synchronize()
        assert alone.status() == 0
        assert torch.equal(y_alone, y_mix), spec[k]
        alone.destroy()
    mix.destroy()


def test_per_item_path_agrees():
    import torch
    spec = workloads.ragged_spec(count=32, seed=3, max_batch=4)
    items = make_items(spec, seed=2)
    plan = m.RaggedPlan([(a, b, d) for a, b, d, _ in items])
    plan.execute()
    torch.cuda.synchronize()
    ragged = [b.clone() for _, b, _, _ in items]
    plan.execute_per_item()
    torch.cuda.synchronize()
    for (_, out, _, _), r in zip(items, ragged):
        n = out.shape[-1]
        assert rel_l2(out.cpu().numpy(), r.cpu().numpy()) <= fp32_tol(n)
    plan.destroy()


def test_unsupported_length_rejected():
    import torch
    x = torch.zeros((1, 17 * 16), dtype=torch.complex64, device="cuda")
    with pytest.raises(m.MofftError):
        m.RaggedPlan([(x, x, -1)])


def test_lost_dependency_times_out_and_context_stays_usable():
    """A second-pass tile whose first-pass tiles never signal gives up after
    its bounded wait: the plan's status turns to an error, no GPU fault, and
    the next execute of the same plan runs normally and is correct."""
    import time
    import torch
    spec = [(16384, 1, -1), (256, 3, 1)]            # one two-pass item, one one-pass item
    items = make_items(spec, seed=11)
    plan = m.RaggedPlan([(a, b, d) for a, b, d, _ in items], single_launch=True)
    stream = torch.cuda.Stream()
    t0 = time.perf_counter()
    plan.check_lost_dependency(stream.cuda_stream)
    stream.synchronize()
    waited = time.perf_counter() - t0
    assert plan.status() == m.Status.INTERNAL_ERROR
    assert waited < 30.0, waited                       # bounded: about a second per tile
    plan.execute(stream.cuda_stream)
    stream.synchronize()
    assert plan.status() == m.Status.SUCCESS
    for (src, out, d, x) in items:
        n = x.shape[-1]
        ref = oracle.fft_ld(x.cpu().numpy().astype(np.complex128), d)
        assert rel_l2(out.cpu().numpy(), ref) <= fp32_tol(n), n
    plan.destroy()


def test_long_items_run_as_tuned_groups():
    """Without two-pass tiles the persistent queue has no waits: the lost-
    dependency run reports success, and the long items (in place and out of
    place, both directions) still match the oracle."""
    import torch
    spec = [(65536, 3, -1), (65536, 2, 1), (24576, 2, -1), (256, 3, 1), (32768, 1, 1)]
    items = make_items(spec, seed=4, inplace=lambda k: k in (1, 2))
    plan = m.RaggedPlan([(a, b, d) for a, b, d, _ in items])
    plan.check_lost_dependency()
    torch.cuda.synchronize()
    assert plan.status() == m.Status.SUCCESS
    plan.execute()
    torch.cuda.synchronize()
    assert plan.status() == m.Status.SUCCESS
    for (src, out, d, x) in items:
        n = x.shape[-1]
        ref = oracle.fft_ld(x.cpu().numpy().astype(np.complex128), d)
        assert rel_l2(out.cpu().numpy(), ref) <= fp32_tol(n), n
    plan.destroy()
