"""MoFFT on NVIDIA B200: Python bindings of the C-ABI library ``libmofft.so``.

The library exports the reference's ``include/mofft.h`` API (plans, execute,
recipes, cost model) plus the batched/stream extensions of
``include/mofft_b200.h``.  This module binds those symbols with ctypes and adds
small conveniences for numpy (host buffers, staged through the GPU by the
library) and torch (device buffers, executed in place on the GPU).

There is no CPU fallback: if the shared library or a CUDA device is missing,
plan creation raises ``MofftError``.
"""
from __future__ import annotations

import ctypes
import enum
import os
from pathlib import Path
from typing import Optional, Sequence

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "lib" / "libmofft.so"


class Status(enum.IntEnum):
    SUCCESS = 0
    INVALID_ARGUMENT = 1
    UNSUPPORTED_SIZE = 2
    ALLOCATION_FAILURE = 3
    UNSUPPORTED_HARDWARE = 4
    INTERNAL_ERROR = 5
    WISDOM_NOT_FOUND = 6
    INCOMPATIBLE_RECIPE = 7
    BUFFER_TOO_SMALL = 8


FORWARD = -1
BACKWARD = 1
OUT_OF_PLACE = 0
IN_PLACE = 1
PLANNER_PRETUNED = 0
PLANNER_MEASURE = 1

# precision forms of FP32 plans (mofft_precision_form)
FORM_FP32 = 0
FORM_TF32X3 = 1
FORM_BF16X3 = 2
PLAN_FORM_TF32X3 = 1 << 8    # mofft_plan_options.flags bits
PLAN_FORM_BF16X3 = 1 << 9
PLAN_STRICT_WISDOM = 1
FLAG_PRETUNED = 0
FLAG_MEASURE = 1
FLAG_WISDOM_ONLY = 2
STAGE_LAYOUT_TRANSPOSE = 0
STAGE_LAYOUT_SECTION = 1
TRANSPOSE_LINEAR = 0
TRANSPOSE_BLOCKED = 1
MAX_PLAN_DEPTH = 64
KERNEL_ROWS, KERNEL_COLS, KERNEL_GENERIC, KERNEL_TENSOR, KERNEL_TENSOR_COLS = 0, 1, 2, 3, 4


class MofftError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = Status(status) if status in Status._value2member_map_ else status
        name = self.status.name if isinstance(self.status, Status) else str(status)
        super().__init__(f"{what}: {name}" if what else name)


class PlanOptions(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("flags", ctypes.c_uint32),
                ("candidate_limit", ctypes.c_size_t), ("timing_samples", ctypes.c_uint32)]


class Diagnostics(ctypes.Structure):
    _fields_ = [("measured", ctypes.c_int), ("used_wisdom", ctypes.c_int),
                ("used_model_fallback", ctypes.c_int),
                ("candidates_measured", ctypes.c_size_t),
                ("radix_count", ctypes.c_size_t),
                ("radices", ctypes.c_int * MAX_PLAN_DEPTH),
                ("kernel_bank", ctypes.c_uint), ("kernel_bank_count", ctypes.c_uint),
                ("blocked_transpose_mask", ctypes.c_uint64),
                ("direct_input", ctypes.c_int), ("stage_layout", ctypes.c_int),
                ("planning_seconds", ctypes.c_double),
                ("selected_median_seconds", ctypes.c_double),
                ("length", ctypes.c_size_t), ("precision_bits", ctypes.c_int),
                ("direction", ctypes.c_int), ("placement", ctypes.c_int)]

    def radix_list(self) -> list[int]:
        return list(self.radices[: self.radix_count])


class CostBreakdown(ctypes.Structure):
    _fields_ = [("kernel_cost", ctypes.c_double), ("memory_cost", ctypes.c_double),
                ("layout_cost", ctypes.c_double), ("total_cost", ctypes.c_double),
                ("logical_read_bytes", ctypes.c_size_t),
                ("logical_write_bytes", ctypes.c_size_t),
                ("transferred_read_bytes", ctypes.c_size_t),
                ("transferred_write_bytes", ctypes.c_size_t),
                ("peak_working_set_bytes", ctypes.c_size_t)]


class Schedule(ctypes.Structure):
    _fields_ = [("pass_count", ctypes.c_int), ("lengths", ctypes.c_int * 4),
                ("kernels", ctypes.c_int * 4), ("smem_bytes", ctypes.c_size_t * 4),
                ("workspace_bytes", ctypes.c_size_t), ("twiddle_bytes", ctypes.c_size_t)]


class RaggedItem(ctypes.Structure):
    _fields_ = [("length", ctypes.c_size_t), ("batch", ctypes.c_size_t),
                ("direction", ctypes.c_int), ("input", ctypes.c_void_p),
                ("output", ctypes.c_void_p)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("streams", ctypes.c_int),
                ("max_group_points", ctypes.c_size_t)]


class Request(ctypes.Structure):
    _fields_ = [("length", ctypes.c_size_t), ("batch", ctypes.c_size_t),
                ("direction", ctypes.c_int), ("precision_bits", ctypes.c_int),
                ("input", ctypes.c_void_p), ("output", ctypes.c_void_p)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("peak_admitted_bytes", ctypes.c_size_t)]


_P = ctypes.c_void_p
_SZ = ctypes.c_size_t
_I = ctypes.c_int
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64

# (name, restype, argtypes) for every exported entry point; the f32/f64 twins
# are expanded below.
class MeasureReport(ctypes.Structure):
    """mofft_measure_report: the MEASURE planner's model order vs its timings."""
    _fields_ = [("candidates", ctypes.c_size_t), ("winner_model_rank", ctypes.c_size_t),
                ("model_first_measured_rank", ctypes.c_size_t),
                ("winner_seconds", ctypes.c_double), ("winner_model_seconds", ctypes.c_double)]


_TYPED = [
    ("mofft_plan_create_{s}", _I, [ctypes.POINTER(_P), _SZ, _I, _I]),
    ("mofft_plan_get_measure_report_{s}", _I, [_P, ctypes.POINTER(MeasureReport)]),
    ("mofft_plan_create_with_options_{s}", _I,
     [ctypes.POINTER(_P), _SZ, _I, _I, ctypes.POINTER(PlanOptions), ctypes.POINTER(Diagnostics)]),
    ("mofft_plan_dft_1d_{s}", _P, [_SZ, _P, _P, _I, _U32]),
    ("mofft_execute_plan_{s}", _I, [_P]),
    ("mofft_plan_create_with_radices_{s}", _I,
     [ctypes.POINTER(_P), _SZ, _I, _I, ctypes.POINTER(_I), _SZ]),
    ("mofft_plan_set_transpose_strategy_{s}", _I, [_P, _I]),
    ("mofft_plan_set_blocked_transpose_mask_{s}", _I, [_P, _U64]),
    ("mofft_plan_set_direct_input_{s}", _I, [_P, _I]),
    ("mofft_plan_set_stage_layout_{s}", _I, [_P, _I]),
    ("mofft_plan_set_kernel_bank_{s}", _I, [_P, ctypes.c_uint]),
    ("mofft_plan_get_kernel_bank_{s}", _I, [_P, ctypes.POINTER(ctypes.c_uint)]),
    ("mofft_plan_export_{s}", _I, [_P, ctypes.c_char_p, _SZ, ctypes.POINTER(_SZ)]),
    ("mofft_plan_import_{s}", _I, [ctypes.POINTER(_P), ctypes.c_char_p, _SZ,
                                   ctypes.POINTER(Diagnostics)]),
    ("mofft_execute_{s}", _I, [_P, _P, _P]),
    ("mofft_plan_destroy_{s}", None, [_P]),
    ("mofft_plan_create_batched_{s}", _I,
     [ctypes.POINTER(_P), _SZ, _SZ, _SZ, _I, _I, ctypes.POINTER(PlanOptions),
      ctypes.POINTER(Diagnostics)]),
    ("mofft_plan_create_batched_with_radices_{s}", _I,
     [ctypes.POINTER(_P), _SZ, _SZ, _SZ, _I, _I, ctypes.POINTER(_I), _SZ]),
    ("mofft_plan_create_batched_with_kernels_{s}", _I,
     [ctypes.POINTER(_P), _SZ, _SZ, _SZ, _I, _I, ctypes.POINTER(_I), _SZ]),
    ("mofft_plan_set_stream_{s}", _I, [_P, _P]),
    ("mofft_plan_get_batch_{s}", _I, [_P, ctypes.POINTER(_SZ), ctypes.POINTER(_SZ)]),
    ("mofft_plan_get_schedule_{s}", _I, [_P, ctypes.POINTER(Schedule)]),
]
_PLAIN = [
    ("mofft_plan_options_init", None, [ctypes.POINTER(PlanOptions)]),
    ("mofft_build_id", ctypes.c_char_p, []),
    ("mofft_estimated_radix_cost", ctypes.c_double, [_I, _I, _I]),
    ("mofft_estimated_stage_cost", ctypes.c_double, [_I, _I, _I, _SZ, _SZ]),
    ("mofft_estimated_plan_cost", ctypes.c_double,
     [_SZ, _I, ctypes.POINTER(_I), _SZ, _U64, _I]),
    ("mofft_estimated_plan_cost_with_layout", ctypes.c_double,
     [_SZ, _I, ctypes.POINTER(_I), _SZ, _U64, _I, _I]),
    ("mofft_estimated_plan_cost_breakdown_with_layout", _I,
     [_SZ, _I, ctypes.POINTER(_I), _SZ, _U64, _I, _I, ctypes.POINTER(CostBreakdown)]),
    ("mofft_wisdom_is_formal", _I, []),
    ("mofft_wisdom_source", ctypes.c_char_p, []),
    ("mofft_status_string", ctypes.c_char_p, [_I]),
    ("mofft_version", ctypes.c_char_p, []),
    ("mofft_kernel_count", _I, []),
    ("mofft_kernel_info", _I, [_I, ctypes.c_char_p, _SZ, ctypes.POINTER(_I),
                               ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I),
                               ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    ("mofft_launch_count", _U64, []),
    ("mofft_execute_fixed_scratch_f32", _I, [_P, _P, _SZ, _SZ, _I, _P]),
    ("mofft_plan_set_precision_form_f32", _I, [_P, _I]),
    ("mofft_plan_get_precision_form_f32", _I, [_P, ctypes.POINTER(_I)]),
    ("mofft_plan_check_f32", _I, [_P]),
    ("mofft_plan_check_lost_copy_f32", _I, [_P, _P, _P]),
    ("mofft_ragged_plan_create_f32", _I, [ctypes.POINTER(_P), ctypes.POINTER(RaggedItem), _SZ]),
    ("mofft_ragged_plan_create_single_launch_f32", _I,
     [ctypes.POINTER(_P), ctypes.POINTER(RaggedItem), _SZ]),
    ("mofft_ragged_execute", _I, [_P, _P]),
    ("mofft_ragged_execute_per_item", _I, [_P, _P]),
    ("mofft_ragged_status", _I, [_P]),
    ("mofft_ragged_check_lost_dependency", _I, [_P, _P]),
    ("mofft_ragged_plan_info", _I, [_P, ctypes.POINTER(_SZ), ctypes.POINTER(_I)]),
    ("mofft_ragged_plan_destroy", None, [_P]),
    ("mofft_server_create", _I, [ctypes.POINTER(_P), ctypes.POINTER(ServerOptions)]),
    ("mofft_server_submit", _I, [_P, ctypes.POINTER(Request), ctypes.POINTER(_U64)]),
    ("mofft_server_wait", _I, [_P, _U64, ctypes.POINTER(ctypes.c_double)]),
    ("mofft_server_drain", _I, [_P]),
    ("mofft_server_get_stats", _I, [_P, ctypes.POINTER(ServerStats)]),
    ("mofft_server_destroy", None, [_P]),
    ("mofft_schedule_preview", _I, [_I, _SZ, ctypes.POINTER(_I), _SZ, ctypes.c_uint,
                                    ctypes.POINTER(Schedule), ctypes.POINTER(_I),
                                    ctypes.POINTER(_SZ)]),
    ("mofft_schedule_model_seconds", ctypes.c_double, [_I, _SZ, _SZ, ctypes.POINTER(_I), _SZ]),
]


def exported_names() -> list[str]:
    """Every entry point the library binds (both precisions expanded)."""
    names = [n.format(s=s) for n, _, _ in _TYPED for s in ("f32", "f64")]
    return names + [n for n, _, _ in _PLAIN]


_lib: Optional[ctypes.CDLL] = None


def load(path: Optional[os.PathLike] = None) -> ctypes.CDLL:
    """Load libmofft.so (raises FileNotFoundError if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: run `python -m mofft_b200.build`")
    lib = ctypes.CDLL(str(p))
    for name, res, args in _TYPED:
        for s in ("f32", "f64"):
            fn = getattr(lib, name.format(s=s))
            fn.restype = res
            fn.argtypes = args
    for name, res, args in _PLAIN:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int, what: str = "") -> None:
    if status != Status.SUCCESS:
        raise MofftError(status, what)


def status_string(status: int) -> str:
    return load().mofft_status_string(status).decode()


def build_id() -> str:
    return load().mofft_build_id().decode()


def launch_count() -> int:
    return int(load().mofft_launch_count())


def kernels() -> list[dict]:
    """The compiled kernel registry."""
    lib = load()
    out = []
    for i in range(lib.mofft_kernel_count()):
        name = ctypes.create_string_buffer(96)
        vals = [ctypes.c_int() for _ in range(6)]
        rad = (ctypes.c_int * 8)()
        lib.mofft_kernel_info(i, name, 96, *[ctypes.byref(v) for v in vals], rad)
        bits, kind, length, lines, threads, count = (v.value for v in vals)
        out.append({"index": i, "name": name.value.decode(), "precision_bits": bits,
                    "kind": kind, "length": length, "lines": lines, "threads": threads,
                    "radices": list(rad[:count]),
                    # generic kernels record the largest radix they run
                    "max_radix": rad[0] if kind == KERNEL_GENERIC else max(rad[:count])})
    return out


def schedule_preview(length: int, bits: int = 32, radices: Optional[Sequence[int]] = None,
                     bank: int = 0) -> dict:
    """Planner decision for a length without a GPU: passes and radix chain."""
    lib = load()
    s = Schedule()
    chain = (ctypes.c_int * 64)()
    count = ctypes.c_size_t()
    arr = _int_array(radices) if radices else None
    st = lib.mofft_schedule_preview(bits, length, arr, len(radices) if radices else 0, bank,
                                    ctypes.byref(s), chain, ctypes.byref(count))
    check(st, f"schedule_preview length={length}")
    n = s.pass_count
    return {"pass_count": n, "lengths": list(s.lengths[:n]), "kernels": list(s.kernels[:n]),
            "smem_bytes": list(s.smem_bytes[:n]), "radices": list(chain[: count.value])}


def model_seconds(length: int, kernels: Sequence[int], bits: int = 32, batch: int = 1) -> float:
    """Device-time model of the schedule running `kernels` (one registry index
    per pass) over `batch` transforms; inf when they do not form one."""
    arr = _int_array(kernels)
    t = load().mofft_schedule_model_seconds(bits, length, batch, arr, len(kernels))
    return float("inf") if t >= 1e300 else float(t)


def _int_array(values: Sequence[int]):
    arr = (ctypes.c_int * max(1, len(values)))(*values)
    return arr


def _pointer_of(buf) -> int:
    """Address of a numpy array or torch tensor (contiguous, complex)."""
    if hasattr(buf, "data_ptr"):
        return int(buf.data_ptr())
    if hasattr(buf, "ctypes"):
        return int(buf.ctypes.data)
    raise TypeError(f"unsupported buffer type {type(buf)!r}")


class Plan:
    """A MoFFT plan (one precision, direction, placement, batch)."""

    def __init__(self, handle: int, bits: int):
        self._h = ctypes.c_void_p(handle)
        self.bits = bits
        self._s = "f32" if bits == 32 else "f64"
        self._lib = load()

    def _fn(self, name: str):
        return getattr(self._lib, f"mofft_{name}_{self._s}")

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @classmethod
    def create(cls, length: int, direction: int = FORWARD, placement: int = OUT_OF_PLACE,
               *, bits: int = 32, batch: int = 1, distance: int = 0,
               mode: int = PLANNER_PRETUNED, flags: int = 0, candidate_limit: int = 0,
               timing_samples: int = 0, radices: Optional[Sequence[int]] = None,
               kernels: Optional[Sequence[int]] = None,
               diagnostics: Optional[Diagnostics] = None) -> "Plan":
        lib = load()
        s = "f32" if bits == 32 else "f64"
        h = ctypes.c_void_p()
        if kernels is not None:
            arr = _int_array(kernels)
            st = getattr(lib, f"mofft_plan_create_batched_with_kernels_{s}")(
                ctypes.byref(h), length, batch, distance, direction, placement, arr,
                len(kernels))
        elif radices is not None:
            arr = _int_array(radices)
            st = getattr(lib, f"mofft_plan_create_batched_with_radices_{s}")(
                ctypes.byref(h), length, batch, distance, direction, placement, arr,
                len(radices))
        else:
            opts = PlanOptions(mode, flags, candidate_limit, timing_samples)
            diag = diagnostics if diagnostics is not None else Diagnostics()
            st = getattr(lib, f"mofft_plan_create_batched_{s}")(
                ctypes.byref(h), length, batch, distance, direction, placement,
                ctypes.byref(opts), ctypes.byref(diag))
        check(st, f"plan length={length} bits={bits}")
        return cls(h.value, bits)

    def execute(self, inp, out=None) -> None:
        """Run on numpy arrays (host) or torch tensors (device)."""
        if out is None:
            out = inp
        check(self._fn("execute")(self._h, _pointer_of(inp), _pointer_of(out)), "execute")

    def execute_ptr(self, in_ptr: int, out_ptr: int) -> int:
        return self._fn("execute")(self._h, in_ptr, out_ptr)

    def set_stream(self, stream_handle: Optional[int]) -> None:
        check(self._fn("plan_set_stream")(self._h, stream_handle or None), "set_stream")

    def set_kernel_bank(self, bank: int) -> None:
        check(self._fn("plan_set_kernel_bank")(self._h, bank), "set_kernel_bank")

    def set_precision_form(self, form: int) -> None:
        """FP32 plans: FORM_FP32 (CUDA cores) or a tensor-core form."""
        if self.bits != 32:
            raise MofftError(1, "precision forms apply to FP32 plans")
        check(self._lib.mofft_plan_set_precision_form_f32(self._h, form), "set_precision_form")

    @property
    def precision_form(self) -> int:
        if self.bits != 32:
            return FORM_FP32
        v = ctypes.c_int()
        check(self._lib.mofft_plan_get_precision_form_f32(self._h, ctypes.byref(v)),
              "get_precision_form")
        return v.value

    def check_status(self) -> None:
        """Blocking: raises if a kernel of this plan that bounds its waits (tensor-core,
        prefetching one-pass) recorded a wait that ran out."""
        if self.bits == 32:
            check(self._lib.mofft_plan_check_f32(self._h), "check")

    def measure_report(self) -> dict:
        """How a MEASURE plan's model order compared with its timings."""
        r = MeasureReport()
        check(self._fn("plan_get_measure_report")(self._h, ctypes.byref(r)), "measure report")
        return {f: getattr(r, f) for f, _ in MeasureReport._fields_}

    def schedule(self) -> dict:
        s = Schedule()
        check(self._fn("plan_get_schedule")(self._h, ctypes.byref(s)), "schedule")
        n = s.pass_count
        return {"pass_count": n, "lengths": list(s.lengths[:n]), "kernels": list(s.kernels[:n]),
                "smem_bytes": list(s.smem_bytes[:n]), "workspace_bytes": s.workspace_bytes,
                "twiddle_bytes": s.twiddle_bytes}

    def export(self) -> bytes:
        req = ctypes.c_size_t()
        check(self._fn("plan_export")(self._h, None, 0, ctypes.byref(req)), "export size")
        buf = ctypes.create_string_buffer(req.value)
        check(self._fn("plan_export")(self._h, buf, req.value, ctypes.byref(req)), "export")
        return buf.raw[: req.value]

    def destroy(self) -> None:
        if self._h and self._h.value:
            self._fn("plan_destroy")(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()


class RaggedPlan:
    """Many FP32 transforms of different lengths in one CUDA graph: the
    one-pass lengths as tiles of one persistent launch, the longer ones as
    tuned groups per (length, direction).  `single_launch` puts every item
    into the persistent launch.

    `items` is a list of (input_tensor, output_tensor, direction) with
    complex64 CUDA tensors of shape (batch, n); input is output for in place."""

    def __init__(self, items, single_launch: bool = False):
        self._lib = load()
        arr = (RaggedItem * len(items))()
        self._keep = []
        for k, (x, y, direction) in enumerate(items):
            n = x.shape[-1]
            arr[k] = RaggedItem(n, x.numel() // n, direction, x.data_ptr(), y.data_ptr())
            self._keep.append((x, y))
        h = ctypes.c_void_p()
        create = (self._lib.mofft_ragged_plan_create_single_launch_f32 if single_launch
                  else self._lib.mofft_ragged_plan_create_f32)
        check(create(ctypes.byref(h), arr, len(items)), "ragged plan")
        self._h = h

    def execute(self, stream: Optional[int] = None) -> None:
        check(self._lib.mofft_ragged_execute(self._h, stream), "ragged execute")

    def execute_per_item(self, stream: Optional[int] = None) -> None:
        check(self._lib.mofft_ragged_execute_per_item(self._h, stream), "per-item execute")

    def status(self) -> int:
        return self._lib.mofft_ragged_status(self._h)

    def check_lost_dependency(self, stream: Optional[int] = None) -> None:
        """One run in which no second-pass dependency can be met (timeout path)."""
        check(self._lib.mofft_ragged_check_lost_dependency(self._h, stream),
              "ragged lost-dependency check")

    def info(self) -> tuple[int, int]:
        tiles = ctypes.c_size_t()
        grid = ctypes.c_int()
        check(self._lib.mofft_ragged_plan_info(self._h, ctypes.byref(tiles), ctypes.byref(grid)),
              "ragged info")
        return tiles.value, grid.value

    def destroy(self) -> None:
        if self._h and self._h.value:
            self._lib.mofft_ragged_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Server:
    """Continuous-batching request engine (include/mofft_serve.h)."""

    def __init__(self, hbm_budget_bytes: int = 0, streams: int = 0, max_group_points: int = 0):
        self._lib = load()
        h = ctypes.c_void_p()
        opts = ServerOptions(hbm_budget_bytes, streams, max_group_points)
        check(self._lib.mofft_server_create(ctypes.byref(h), ctypes.byref(opts)), "server")
        self._h = h

    def submit(self, length: int, batch: int, direction: int, bits: int, input_ptr: int,
               output_ptr: int) -> int:
        req = Request(length, batch, direction, bits, input_ptr, output_ptr)
        ticket = ctypes.c_uint64()
        check(self._lib.mofft_server_submit(self._h, ctypes.byref(req), ctypes.byref(ticket)),
              "submit")
        return ticket.value

    def wait(self, ticket: int) -> tuple[int, float]:
        lat = ctypes.c_double()
        st = self._lib.mofft_server_wait(self._h, ticket, ctypes.byref(lat))
        return st, lat.value

    def drain(self) -> None:
        check(self._lib.mofft_server_drain(self._h), "drain")

    def stats(self) -> dict:
        s = ServerStats()
        check(self._lib.mofft_server_get_stats(self._h, ctypes.byref(s)), "stats")
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def destroy(self) -> None:
        if self._h and self._h.value:
            self._lib.mofft_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def fft(x, direction: int = FORWARD, *, inplace: bool = False):
    """Batched transform of a torch tensor of shape (..., n), complex64 or
    complex128, on its CUDA device.  Returns the output tensor."""
    import torch
    if not x.is_cuda:
        raise ValueError("fft() takes a CUDA tensor; use Plan for host arrays")
    if x.dtype not in (torch.complex64, torch.complex128):
        raise TypeError("complex64 or complex128 tensor required")
    x = x.contiguous()
    n = x.shape[-1]
    batch = x.numel() // n
    bits = 32 if x.dtype == torch.complex64 else 64
    out = x if inplace else torch.empty_like(x)
    plan = _plan_cache_get(n, batch, direction, inplace, bits, x.device.index or 0)
    plan.set_stream(torch.cuda.current_stream(x.device).cuda_stream)
    plan.execute(x, out)
    return out


_PLAN_CACHE: dict = {}


def _plan_cache_get(n, batch, direction, inplace, bits, device):
    key = (n, batch, direction, inplace, bits, device)
    plan = _PLAN_CACHE.get(key)
    if plan is None:
        plan = Plan.create(n, direction, IN_PLACE if inplace else OUT_OF_PLACE,
                           bits=bits, batch=batch)
        _PLAN_CACHE[key] = plan
    return plan
