"""libmofft.so checks that need no GPU: it loads, exports every entry point
the headers declare, keeps the reference's status strings / version / build ID
format, validates arguments before touching a device, reproduces the
reference's cost-model byte accounting, and plans every supported length."""
from __future__ import annotations

import ctypes
import math
import re

import numpy as np
import pytest

import mofft_b200 as m
from tests.conftest import ROOT, cuda_available

INF = float("inf")
DBL_MAX = np.finfo(np.float64).max


def declared_functions() -> set[str]:
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        for match in re.finditer(r"\b(mofft_[a-z0-9_]+)\s*\(", text):
            names.add(match.group(1))
    return names


def test_every_declared_symbol_is_exported():
    lib = m.load()
    declared = declared_functions()
    assert len(declared) >= 55
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    for n in m.exported_names():
        assert n in declared, n
    # nothing beyond the declared API is exported
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(m.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert exported == declared, sorted(exported ^ declared)


def test_status_strings_version_build_id():
    want = ["success", "invalid argument", "unsupported size", "allocation failure",
            "unsupported hardware", "internal error", "compiled wisdom not found",
            "incompatible plan recipe", "output buffer too small"]
    for i, s in enumerate(want):
        assert m.status_string(i) == s
    assert m.status_string(99) == "unknown status"
    assert m.load().mofft_version().decode() == "0.4.0"
    bid = m.build_id()
    assert re.fullmatch(r"[0-9a-f]{64}", bid)
    assert (ROOT / "mofft_b200" / "lib" / "BUILD_ID").read_text().strip() == bid


def test_options_validation_before_hardware():
    lib = m.load()
    h = ctypes.c_void_p(1)
    diag = m.Diagnostics()
    bad = [m.PlanOptions(m.PLANNER_MEASURE, 1, 0, 0),     # MEASURE with flags
           m.PlanOptions(7, 0, 0, 0),                     # bad mode
           m.PlanOptions(0, 4, 0, 0),                     # unknown flag
           m.PlanOptions(0, m.PLAN_FORM_TF32X3 | m.PLAN_FORM_BF16X3, 0, 0),  # two forms
           m.PlanOptions(m.PLANNER_MEASURE, m.PLAN_FORM_TF32X3, 0, 0),      # MEASURE + form
           m.PlanOptions(m.PLANNER_MEASURE, 0, 65, 0),    # > 64 candidates
           m.PlanOptions(m.PLANNER_MEASURE, 0, 0, 32)]    # > 31 samples
    for opts in bad:
        st = lib.mofft_plan_create_with_options_f32(ctypes.byref(h), 64, m.FORWARD,
                                                     m.OUT_OF_PLACE, ctypes.byref(opts),
                                                     ctypes.byref(diag))
        assert st == m.Status.INVALID_ARGUMENT
        assert h.value is None
    # a precision form is an FP32 option
    form = m.PlanOptions(0, m.PLAN_FORM_BF16X3, 0, 0)
    st = lib.mofft_plan_create_with_options_f64(ctypes.byref(h), 4096, m.FORWARD,
                                                 m.OUT_OF_PLACE, ctypes.byref(form),
                                                 ctypes.byref(diag))
    assert st == m.Status.INVALID_ARGUMENT and h.value is None
    st = lib.mofft_plan_create_f32(None, 64, m.FORWARD, m.OUT_OF_PLACE)
    assert st == m.Status.INVALID_ARGUMENT
    st = lib.mofft_plan_create_f64(ctypes.byref(h), 64, 0, m.OUT_OF_PLACE)
    assert st == m.Status.INVALID_ARGUMENT
    st = lib.mofft_plan_create_f64(ctypes.byref(h), 64, m.FORWARD, 5)
    assert st == m.Status.INVALID_ARGUMENT
    bad_radices = (ctypes.c_int * 2)(17, 16)
    st = lib.mofft_plan_create_with_radices_f32(ctypes.byref(h), 256, m.FORWARD,
                                                 m.OUT_OF_PLACE, bad_radices, 2)
    assert st == m.Status.INVALID_ARGUMENT
    buf = (ctypes.c_float * 8)()
    assert lib.mofft_plan_dft_1d_f32(4, buf, buf, m.FORWARD, 3) is None
    assert lib.mofft_plan_dft_1d_f32(4, None, buf, m.FORWARD, 0) is None
    assert lib.mofft_execute_f32(None, buf, buf) == m.Status.INVALID_ARGUMENT
    assert lib.mofft_execute_plan_f64(None) == m.Status.INVALID_ARGUMENT
    lib.mofft_plan_destroy_f32(None)


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU path")
def test_no_gpu_reports_unsupported_hardware():
    lib = m.load()
    h = ctypes.c_void_p()
    assert lib.mofft_plan_create_f32(ctypes.byref(h), 64, m.FORWARD,
                                     m.OUT_OF_PLACE) == m.Status.UNSUPPORTED_HARDWARE
    assert h.value is None
    with pytest.raises(m.MofftError):
        m.Plan.create(64)


def test_recipe_rejections_without_device():
    lib = m.load()
    bid = m.build_id()
    good = f"MOFFT_PLAN_V1 {bid} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 3 4 4 4\n"
    for f in (lib.mofft_plan_import_f32, lib.mofft_plan_import_f64):
        h = ctypes.c_void_p(1)
        raw = good.encode() + b"\0"
        # truncated: missing NUL / missing newline
        assert f(ctypes.byref(h), raw, len(raw) - 1, None) == m.Status.INVALID_ARGUMENT
        assert h.value is None
        assert f(ctypes.byref(h), raw, len(raw) - 2, None) == m.Status.INVALID_ARGUMENT
        bad = ("X" + good[1:]).encode() + b"\0"
        assert f(ctypes.byref(h), bad, len(bad), None) == m.Status.INCOMPATIBLE_RECIPE
        flip = good.replace(bid, ("1" if bid[0] == "0" else "0") + bid[1:]).encode() + b"\0"
        assert f(ctypes.byref(h), flip, len(flip), None) == m.Status.INCOMPATIBLE_RECIPE
        trailing = raw + b"x\0"
        assert f(ctypes.byref(h), trailing, len(trailing), None) == m.Status.INVALID_ARGUMENT
        spaced = good.replace(" 4 4 4", "  4 4 4").encode() + b"\0"
        assert f(ctypes.byref(h), spaced, len(spaced), None) == m.Status.INCOMPATIBLE_RECIPE
    # precision mismatch is checked before the device family
    h = ctypes.c_void_p(1)
    raw = good.encode() + b"\0"
    assert lib.mofft_plan_import_f64(ctypes.byref(h), raw, len(raw), None) == \
        m.Status.INCOMPATIBLE_RECIPE


def test_recipe_status_per_malformed_field():
    """One malformed field at a time, and the precedence between kinds of
    failure, as the reference's recipe parser ranks them
    (src/mofft.c:1760-1842, tests/test_plan_recipe.c:196-241).  A valid
    recipe needs the device family, so these cases stop short of it."""
    lib = m.load()
    bid = m.build_id()
    head = f"MOFFT_PLAN_V1 {bid}"
    INV, INC = m.Status.INVALID_ARGUMENT, m.Status.INCOMPATIBLE_RECIPE
    cases = [
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 3 4 4 4 4", INV),  # depth/count
        (f"{head} 0a00094 f32 64 -1 0 0 0000000000000000 1 0 3 4 4 4", INV),  # family width
        (f"{head} 0a00009g f32 64 -1 0 0 0000000000000000 1 0 3 4 4 4", INV),  # family digit
        (f"{head} 0a000094 f32 64 -1 0 0 000000000000000 1 0 3 4 4 4", INV),  # mask width
        (f"{head} 0a000094 f32 6x -1 0 0 0000000000000000 1 0 3 4 4 4", INV),  # length digit
        (f"{head} 0a000094 f32 64 2 0 0 0000000000000000 1 0 3 4 4 4", INV),  # direction
        (f"{head} 0a000094 f32 64 -1 2 0 0000000000000000 1 0 3 4 4 4", INV),  # placement
        (f"{head} 0a000094 f32 64 -1 0 4 0000000000000000 1 0 3 4 4 4", INV),  # bank
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000004 1 0 3 4 4 4", INV),  # mask bit
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 2 0 3 4 4 4", INV),  # direct input
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 2 3 4 4 4", INV),  # layout
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 0 64", INV),  # depth 0
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 3 4 4 5", INV),  # chain
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 3 4 4 2", INV),  # product
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 3 4 1 16", INV),  # radix 1
        (f"{head} 0a000094 f32 1 -1 0 0 0000000000000000 1 0 1 1", INV),  # length 1
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0", INC),  # too few fields
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 3 4  4 4", INC),  # blank pair
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 3 4 4 4 ", INV),  # trailing blank
        (f"{head} 0a000094 f32 64 -1 0 0 0000000000000000 1 0 64" + " 2" * 77, INC),  # fields
        (f"{head} 0a000094 f16 64 -1 0 0 0000000000000000 1 0 3 4 4 4", INC),  # precision
        # the precision tag outranks value failures, syntax outranks the tag
        (f"{head} 0a000094 f64 64 -1 0 0 0000000000000000 1 0 3 4 4 x", INC),
        (f"{head} 0a000094 f64 64 3 0 0 0000000000000000 1 0 3 4 4 4", INC),
        (f"{head} 0a000094 f64 6x -1 0 0 0000000000000000 1 0 3 4 4 4", INV),
        # the magic and build id outrank every field check
        (f"MOFFT_PLAN_V2 {bid} 0a00094 f64 64 -1 0 0 0000000000000000 1 0 3 4 4 4", INC),
        ("\tMOFFT", INV),  # character set
    ]
    for text, expected in cases:
        raw = text.encode() + b"\n\0"
        h = ctypes.c_void_p(1)
        st = lib.mofft_plan_import_f32(ctypes.byref(h), raw, len(raw), None)
        assert st == expected, (text, st)
        assert h.value is None
    big = b"MOFFT_PLAN_V1" + b" 2" * 600 + b"\n\0"  # beyond the 1024-byte limit
    h = ctypes.c_void_p(1)
    assert lib.mofft_plan_import_f32(ctypes.byref(h), big, len(big), None) == INV


def _arr(values):
    return (ctypes.c_int * len(values))(*values)


def test_cost_model_reference_accounting():
    """tests/test_fft.c:493-560 of the reference, same byte values."""
    lib = m.load()
    small = lib.mofft_estimated_stage_cost(8, 64, 0, 4096, 512)
    large = lib.mofft_estimated_stage_cost(8, 64, 0, 262144, 32768)
    assert math.isfinite(small) and math.isfinite(large) and large > small
    assert lib.mofft_estimated_stage_cost(8, 16, 0, 4096, 512) == DBL_MAX
    r = _arr([8, 8, 8, 8])
    materialized = lib.mofft_estimated_plan_cost(4096, 64, r, 4, 0, 0)
    blocked = lib.mofft_estimated_plan_cost(4096, 64, r, 4, 7, 0)
    direct = lib.mofft_estimated_plan_cost(4096, 64, r, 4, 0, 1)
    section = lib.mofft_estimated_plan_cost_with_layout(4096, 64, r, 4, 0, 0, 1)
    sd, ld, bd = m.CostBreakdown(), m.CostBreakdown(), m.CostBreakdown()
    assert lib.mofft_estimated_plan_cost_breakdown_with_layout(4096, 64, r, 4, 0, 0, 1,
                                                               ctypes.byref(sd)) == 0
    assert lib.mofft_estimated_plan_cost_breakdown_with_layout(4096, 64, r, 4, 0, 0, 0,
                                                               ctypes.byref(ld)) == 0
    assert lib.mofft_estimated_plan_cost_breakdown_with_layout(4096, 64, r, 4, 7, 0, 0,
                                                               ctypes.byref(bd)) == 0
    for v in (materialized, blocked, direct, section):
        assert math.isfinite(v)
    assert sd.logical_read_bytes == 336896 and sd.logical_write_bytes == 262144
    assert sd.transferred_read_bytes == 336896 and sd.transferred_write_bytes == 262144
    assert sd.peak_working_set_bytes == 196608 and sd.layout_cost == 0.0
    assert ld.logical_read_bytes == 533504 and ld.logical_write_bytes == 458752
    assert ld.transferred_read_bytes == 992256 and ld.transferred_write_bytes == 458752
    assert bd.transferred_read_bytes == 533504
    assert ld.layout_cost > 0.0
    assert abs(sd.total_cost - section) <= 1e-12
    assert abs(ld.total_cost - materialized) <= 1e-12
    assert lib.mofft_estimated_plan_cost(4096, 64, r, 3, 0, 1) == DBL_MAX
    assert lib.mofft_estimated_plan_cost_breakdown_with_layout(4096, 64, r, 4, 0, 0, 1,
                                                               None) == 1
    assert lib.mofft_estimated_plan_cost_with_layout(4096, 64, r, 4, 0, 0, 99) == DBL_MAX
    assert lib.mofft_estimated_radix_cost(17, 32, 1) == DBL_MAX
    assert 0 < lib.mofft_estimated_radix_cost(16, 32, 1) < lib.mofft_estimated_radix_cost(16, 32, 0)


def test_kernel_registry_is_consistent():
    ks = m.kernels()
    generic = [k for k in ks if k["kind"] == m.KERNEL_GENERIC]
    assert sorted(set((k["precision_bits"], k["max_radix"]) for k in generic)) == \
        [(32, 16), (32, 64), (64, 16), (64, 64)]
    # one runtime-stage kernel per precision, width and kernel bank (0
    # default codelets; 1-3 like-terms, even-odd, vector-reuse families)
    assert sorted(k["name"] for k in generic) == sorted(
        f"generic_{t}{w}{f}" for t in ("float", "double") for w in ("", "_wide")
        for f in ("", "_lt", "_eo", "_vr"))
    for k in ks:
        if k["kind"] == m.KERNEL_GENERIC:
            continue
        assert int(np.prod(k["radices"])) == k["length"], k
        assert k["threads"] <= 1024 and k["threads"] % 32 == 0 or k["threads"] < 32 or \
            k["threads"] % 8 == 0
    for bits in (32, 64):
        lengths = [2 ** e for e in range(1, 14 if bits == 32 else 13)] + \
            [3 * 2 ** e for e in range(4, 13)] + [5 * 2 ** e for e in range(4, 12)]
        for n in lengths:
            assert any(k["kind"] == m.KERNEL_ROWS and k["length"] == n and
                       k["precision_bits"] == bits for k in ks), (bits, n)


def test_explicit_kernel_plans_validate_before_hardware():
    lib = m.load()
    ks = m.kernels()
    rows = {(k["precision_bits"], k["length"]): k["index"] for k in ks
            if k["kind"] == m.KERNEL_ROWS}
    cols = [k for k in ks if k["kind"] == m.KERNEL_COLS and k["precision_bits"] == 32]
    h = ctypes.c_void_p(1)

    def make(bits, n, idx):
        arr = (ctypes.c_int * len(idx))(*idx)
        fn = getattr(lib, f"mofft_plan_create_batched_with_kernels_f{bits}")
        return fn(ctypes.byref(h), n, 4, 0, m.FORWARD, m.OUT_OF_PLACE, arr, len(idx))

    assert make(32, 4096, [rows[(64, 4096)]]) == m.Status.INVALID_ARGUMENT   # precision
    assert make(32, 2048, [rows[(32, 4096)]]) == m.Status.INVALID_ARGUMENT   # length
    assert make(32, 4096, [cols[0]["index"]]) == m.Status.INVALID_ARGUMENT   # one COLS pass
    assert make(32, 4096, [-1]) == m.Status.INVALID_ARGUMENT
    assert h.value is None
    if not cuda_available():
        assert make(32, 4096, [rows[(32, 4096)]]) == m.Status.UNSUPPORTED_HARDWARE


def test_tensor_forms_registered_and_never_planned():
    ks = m.kernels()
    tensor = sorted((k["name"], k["length"], k["radices"], k["precision_bits"])
                    for k in ks if k["kind"] == m.KERNEL_TENSOR)
    assert tensor == [("tensor_float_4096_bf16x3_r16x3", 4096, [16, 16, 16], 32),
                      ("tensor_float_4096_bf16x3_r64x2", 4096, [64, 64], 32),
                      ("tensor_float_4096_tf32x3_r16x3", 4096, [16, 16, 16], 32)]
    cols = sorted((k["name"], k["length"], k["lines"], k["radices"])
                  for k in ks if k["kind"] == m.KERNEL_TENSOR_COLS)
    assert cols == [("tensor_cols_float_256_bf16x3_c16", 256, 16, [16, 16]),
                    ("tensor_cols_float_256_tf32x3_c16", 256, 16, [16, 16])]
    # the planner keeps FP32 (CUDA-core) kernels unless a form is requested
    for bits in (32, 64):
        s = m.schedule_preview(4096, bits)
        assert all(ks[k]["kind"] not in (m.KERNEL_TENSOR, m.KERNEL_TENSOR_COLS)
                   for k in s["kernels"])
    s = m.schedule_preview(65536, 32)
    assert all(ks[k]["kind"] == m.KERNEL_COLS for k in s["kernels"])


def test_wisdom_names_compiled_kernels():
    """Every kernel instance the committed wisdom names is in the compiled
    registry with that entry's precision, and the named kernels multiply out
    to the entry's length with its radix chain (a tuned schedule that names a
    removed or renamed instance would silently fall back to the model)."""
    import json
    from pathlib import Path
    wisdom = json.loads((Path(m.__file__).parent / "wisdom" / "b200_wisdom.json").read_text())
    ks = {k["name"]: k for k in m.kernels()}
    for e in wisdom["entries"]:
        assert int(np.prod(e["chain"])) == e["length"], e
        if e["kernel_bank"] != 0:
            continue
        assert e["kernels"], e
        total = 1
        for name in e["kernels"]:
            assert name in ks, (e["length"], e["precision_bits"], name)
            assert ks[name]["precision_bits"] == e["precision_bits"], name
            total *= ks[name]["length"]
        assert total == e["length"], e


def test_prefetching_kernel_registered():
    """The persistent prefetching one-pass kernel: one line per CTA step,
    512 threads, chain (32, 32, 16) for FP32 16384, and the compiled wisdom
    selects it for that length."""
    import json
    from pathlib import Path
    ks = [k for k in m.kernels() if k["name"] == "rows_float_16384_t512_b1_sfalse_dxp"]
    assert len(ks) == 1
    k = ks[0]
    assert (k["kind"], k["precision_bits"], k["length"], k["lines"], k["threads"],
            k["radices"]) == (m.KERNEL_ROWS, 32, 16384, 1, 512, [32, 32, 16])
    wisdom = json.loads((Path(m.__file__).parent / "wisdom" / "b200_wisdom.json").read_text())
    e = [e for e in wisdom["entries"] if e["length"] == 16384 and e["precision_bits"] == 32]
    assert e and e[0]["kernels"] == [k["name"]]


def test_mixed_lengths_use_specialised_kernels():
    """3*2^k and 5*2^k lengths of the plain-method sweep run on specialised
    kernels (no runtime-stage kernel), single pass up to 12288 / 10240."""
    ks = {k["index"]: k for k in m.kernels()}
    for bits in (32, 64):
        for n in [3 * 2 ** e for e in range(4, 19)] + [5 * 2 ** e for e in range(4, 18)]:
            s = m.schedule_preview(n, bits)
            kinds = [ks[k]["kind"] for k in s["kernels"]]
            assert m.KERNEL_GENERIC not in kinds, (bits, n, s)
            if n <= 12288:
                assert s["pass_count"] == 1, (bits, n, s)


SWEEP = [2 ** e for e in range(1, 25)] + [3 * 2 ** e for e in range(4, 19)] + \
        [5 * 2 ** e for e in range(4, 18)] + [30, 45, 144, 169, 196, 225, 1728, 2197, 2744,
                                               3375, 20736, 28561, 38416, 50625, 248832,
                                               371293, 537824, 759375]


@pytest.mark.parametrize("bits", [32, 64])
def test_planner_covers_every_length(bits):
    """Every length of the sweep (powers of two to 2^24, 3*2^k / 5*2^k up to
    ~2^20, and the reference's extended sizes) gets a schedule whose passes
    multiply to the length, with single-pass lengths in one kernel."""
    ks = {k["index"]: k for k in m.kernels()}
    for n in SWEEP:
        s = m.schedule_preview(n, bits)
        assert int(np.prod(s["lengths"])) == n
        assert int(np.prod(s["radices"])) == n
        limit = 16384 if bits == 32 else 8192
        if n <= limit and (n & (n - 1)) == 0:
            assert s["pass_count"] == 1
            assert ks[s["kernels"][0]]["kind"] == m.KERNEL_ROWS
        assert s["pass_count"] <= 3
        for smem in s["smem_bytes"]:
            assert smem <= 227 * 1024
    with pytest.raises(m.MofftError):
        m.schedule_preview(17, bits)


def test_planner_power_of_two_pass_counts():
    """Pass counts of the model's schedules: ceil(log2 n / 14) for FP32 and
    ceil(log2 n / 13) for FP64, up to 2^24 / 2^22 (one CTA holds 2^14 FP32 /
    2^13 FP64 points; the thread-block cluster kernels, which hold up to 2^16
    / 2^15, run only when a tuned or explicit kernel list names them)."""
    for e in range(1, 25):
        assert m.schedule_preview(2 ** e, 32)["pass_count"] == math.ceil(e / 14), e
    for e in range(1, 23):
        assert m.schedule_preview(2 ** e, 64)["pass_count"] == math.ceil(e / 13), e
    ks = {k["index"]: k for k in m.kernels()}
    for n, bits in ((16384, 32), (32768, 32), (65536, 32), (16384, 64), (32768, 64)):
        s = m.schedule_preview(n, bits)
        assert not any(ks[k]["name"].startswith("cluster_") for k in s["kernels"]), (n, bits)


def test_explicit_radices_are_honoured():
    s = m.schedule_preview(256, 32, radices=[32, 8])
    assert s["radices"] == [32, 8] and s["pass_count"] == 1
    s = m.schedule_preview(4096, 32, radices=[16, 16, 16])
    assert s["radices"] == [16, 16, 16]
    s = m.schedule_preview(64, 64, radices=[64])
    assert s["radices"] == [64]
    with pytest.raises(m.MofftError):
        m.schedule_preview(256, 32, radices=[17, 16])
    g = m.schedule_preview(4096, 32, bank=1)
    ks = {k["index"]: k for k in m.kernels()}
    assert all(ks[k]["kind"] == m.KERNEL_GENERIC for k in g["kernels"])
    for bank, suffix in ((1, "_lt"), (2, "_eo"), (3, "_vr")):
        g = m.schedule_preview(96, 64, bank=bank)
        assert [ks[k]["name"] for k in g["kernels"]] == [f"generic_double{suffix}"], bank
    with pytest.raises(m.MofftError):
        m.schedule_preview(96, 64, bank=4)


def _schedule_candidates(n, bits, ks):
    """The MEASURE planner's candidate shapes: every one-pass kernel of the
    length, every pair of column kernels, every triple of 64..512-point column
    kernels (mofft_measure.c, enumerate)."""
    import itertools
    out = [[k["index"]] for k in ks if k["kind"] == m.KERNEL_ROWS and
           k["precision_bits"] == bits and k["length"] == n]
    cols = [k for k in ks if k["kind"] == m.KERNEL_COLS and k["precision_bits"] == bits]
    out += [[a["index"], b["index"]] for a, b in itertools.product(cols, cols)
            if a["length"] * b["length"] == n]
    narrow = [k for k in cols if 64 <= k["length"] <= 512]
    out += [[a["index"], b["index"], c["index"]]
            for a, b, c in itertools.product(narrow, narrow, narrow)
            if a["length"] * b["length"] * c["length"] == n]
    return out


def test_model_ranks_the_tuned_schedules():
    """The device-time model is the planner's prior: for most lengths of the
    compiled wisdom, the schedule the autotuner measured fastest is among the
    model's two best candidates, and the model's time for it is within a
    factor of two of the measured one."""
    import json
    ks = m.kernels()
    byname = {k["name"]: k for k in ks}
    entries = json.loads((ROOT / "mofft_b200" / "wisdom" / "b200_wisdom.json").read_text())
    top2 = total = 0
    for e in entries["entries"]:
        n, bits, batch = e["length"], e["precision_bits"], e["batch"]
        win = [byname[x]["index"] for x in e["kernels"]]
        t_win = m.model_seconds(n, win, bits, batch)
        assert math.isfinite(t_win), e["kernels"]
        assert 0.5 <= t_win / e["median_seconds"] <= 2.0, (n, bits, t_win, e["median_seconds"])
        times = [m.model_seconds(n, c, bits, batch) for c in _schedule_candidates(n, bits, ks)]
        rank = 1 + sum(1 for t in times if math.isfinite(t) and t < t_win * (1 - 1e-9))
        top2 += rank <= 2
        total += 1
    print(f"tuned schedule among the model's two best: {top2}/{total}")
    assert total >= 90 and top2 >= 0.6 * total
    assert m.model_seconds(4096, [byname["cols_float_64_t4_c32"]["index"]], 32, 1) == INF
