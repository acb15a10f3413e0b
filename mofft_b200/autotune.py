"""GPU autotuner: MEASURE-planner search over the plain-method sweep, written
as plan wisdom.

The B200 counterpart of the reference's retune pipeline
(tools/retune_native.py:25-136 driving tools/plan_search.cpp:514-639 and
tools/compile_wisdom.py): for every length of the sweep (powers of two
2^4..2^24, 3*2^k and 5*2^k) and both precisions, a batched MEASURE plan
(candidate radix chains x pass splits x kernel instances x kernel banks,
timed with CUDA events on the GPU) picks the fastest schedule; the winning
stage chain and kernel instance names go to
mofft_b200/wisdom/b200_wisdom.json, which compile_wisdom.py turns into the
device plan cache that PRETUNED plans consult.

Run on the GPU:  python -m mofft_b200.autotune [--out path] [--formal]
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import sys
from pathlib import Path

import mofft_b200 as m

SWEEP = sorted([2 ** e for e in range(4, 25)] + [3 * 2 ** e for e in range(4, 19)] +
               [5 * 2 ** e for e in range(4, 18)])


def tune_one(n: int, bits: int, points: int, candidates: int, samples: int) -> dict:
    lib = m.load()
    batch = max(1, points // n)
    h = ctypes.c_void_p()
    diag = m.Diagnostics()
    opts = m.PlanOptions(m.PLANNER_MEASURE, 0, candidates, samples)
    fn = getattr(lib, f"mofft_plan_create_batched_f{bits}")
    m.check(fn(ctypes.byref(h), n, batch, 0, m.FORWARD, m.IN_PLACE, ctypes.byref(opts),
               ctypes.byref(diag)), f"measure n={n} bits={bits}")
    plan = m.Plan(h.value, bits)
    sched = plan.schedule()
    names = {k["index"]: k["name"] for k in m.kernels()}
    plan.destroy()
    chain = list(reversed(diag.radix_list()))
    secs = diag.selected_median_seconds
    flops = 5.0 * n * (n.bit_length() - 1 if n & (n - 1) == 0 else __import__("math").log2(n))
    return {"length": n, "precision_bits": bits, "chain": chain,
            "kernels": [names[k] for k in sched["kernels"]] if diag.kernel_bank == 0 else [],
            "kernel_bank": diag.kernel_bank, "batch": batch,
            "candidates_measured": diag.candidates_measured,
            "median_seconds": secs, "gflops": round(flops * batch / secs / 1e9, 1)}


def main(argv: list[str]) -> int:
    p = argparse.ArgumentParser()
    p.add_argument("--out", default=str(Path(__file__).resolve().parent / "wisdom" /
                                        "b200_wisdom.json"))
    p.add_argument("--candidates", type=int, default=32)
    p.add_argument("--samples", type=int, default=5)
    p.add_argument("--formal", action="store_true",
                   help="mark the wisdom formal (tuned on an otherwise idle B200)")
    p.add_argument("--lengths", type=int, nargs="*")
    args = p.parse_args(argv[1:])
    import torch
    dev = torch.cuda.get_device_name(0)
    entries = []
    for bits in (32, 64):
        points = (1 << 25) if bits == 32 else (1 << 24)
        for n in (args.lengths or SWEEP):
            e = tune_one(n, bits, points, args.candidates, args.samples)
            entries.append(e)
            print(json.dumps(e), flush=True)
    out = {"source": f"mofft_b200.autotune on {dev}, "
                     f"{datetime.datetime.now(datetime.timezone.utc).date()}",
           "formal": bool(args.formal), "entries": entries}
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    Path(args.out).write_text(json.dumps(out, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
