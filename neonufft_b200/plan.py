"""Python mirror of the reference GPU plan API (include/neonufft/gpu/plan.hpp:25-82).

``Plan`` and ``PlanT3`` take the same arguments as ``neonufft::gpu::Plan<T,DIM>`` and
``neonufft::gpu::PlanT3<T,DIM>`` and forward every call to the C ABI of libneonufft_b200.so.
Device arrays are torch CUDA tensors (or raw device pointers given as ints); the precision T is
taken from the coordinate tensors (float32 -> float plan, float64 -> double plan) unless
``dtype`` is given. The stream defaults to torch's current CUDA stream.

Errors raise the Python counterparts of the reference exception types
(include/neonufft/exceptions.hpp:16-103).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

from . import _lib as L

MODE_ORDER_FFT = 0
MODE_ORDER_CMCL = 1


class GenericError(RuntimeError):
    error_code = L.GENERIC_ERROR


class MemoryAllocError(GenericError):
    error_code = L.MEMORY_ALLOC_ERROR


class InternalError(GenericError):
    error_code = L.INTERNAL_ERROR


class InputError(GenericError):
    error_code = L.INPUT_ERROR


class GPUError(GenericError):
    error_code = L.GPU_ERROR


class NotImplementedError_(GenericError):
    error_code = L.NOT_IMPLEMENTED_ERROR


_ERRORS = {
    L.MEMORY_ALLOC_ERROR: MemoryAllocError,
    L.INTERNAL_ERROR: InternalError,
    L.INPUT_ERROR: InputError,
    L.GPU_ERROR: GPUError,
    L.NOT_IMPLEMENTED_ERROR: NotImplementedError_,
}


def check(code: int) -> None:
    if code == L.SUCCESS:
        return
    msg = L.load().nnb_last_error_message().decode(errors="replace")
    raise _ERRORS.get(code, GenericError)(msg or f"neonufft error {code}")


@dataclass
class Options:
    """Mirror of neonufft::Options (reference include/neonufft/plan.hpp:19-29) plus engine
    extensions (tile shape, spread method, kernel width override; 0 = automatic)."""
    tol: float = 0.001
    upsampfac: float = 2.0
    recenter_threshold: float = 0.1
    num_threads: int = 0
    sort_input: bool = True
    sort_output: bool = True
    kernel_approximation: bool = False
    order: int = MODE_ORDER_CMCL
    kernel_type: int = 0
    tile: tuple = (0, 0, 0)
    spread_method: int = 0
    n_spread: int = 0

    def to_c(self) -> L.NnbOptions:
        o = L.NnbOptions()
        L.load().nnb_options_default(C.byref(o))
        o.tol = float(self.tol)
        o.upsampfac = float(self.upsampfac)
        o.recenter_threshold = float(self.recenter_threshold)
        o.num_threads = int(self.num_threads)
        o.sort_input = int(bool(self.sort_input))
        o.sort_output = int(bool(self.sort_output))
        o.kernel_approximation = int(bool(self.kernel_approximation))
        o.order = int(self.order)
        o.kernel_type = int(self.kernel_type)
        t = list(self.tile) + [0] * (3 - len(self.tile))
        for i in range(3):
            o.tile[i] = int(t[i])
        o.spread_method = int(self.spread_method)
        o.n_spread = int(self.n_spread)
        return o


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    dp = getattr(x, "data_ptr", None)
    if dp is None:
        raise TypeError("expected a torch CUDA tensor or a device pointer (int)")
    if not x.is_cuda:
        raise TypeError("device arrays must be CUDA tensors")
    return dp()


def _stream(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _precision(dtype, arrays) -> int:
    if dtype is None:
        for a in arrays:
            dt = getattr(a, "dtype", None)
            if dt is not None:
                dtype = dt
                break
    name = str(dtype)
    if "float32" in name or name == "float":
        return L.NNB_FLOAT
    if "float64" in name or name == "double":
        return L.NNB_DOUBLE
    raise TypeError(f"cannot infer plan precision from {dtype!r}; pass dtype=torch.float32/float64")


class _Alloc:
    """Keeps a user allocator (object with allocate(size)->ptr and deallocate(ptr)) alive as
    C callbacks (the C ABI form of neonufft::Allocator)."""

    def __init__(self, alloc):
        self.obj = alloc

        def _a(ctx, size):
            try:
                p = alloc.allocate(int(size))
                return int(p) if p else None
            except Exception:  # a failing allocator reports NULL, the plan raises MemoryAllocError
                return None

        def _d(ctx, ptr):
            try:
                alloc.deallocate(int(ptr) if ptr else 0)
            except Exception:
                pass

        self.fa = L.AllocFn(_a)
        self.fd = L.FreeFn(_d)
        self.c = L.NnbAllocator(self.fa, self.fd, None)


class Plan:
    """Type-1 / type-2 plan: mirror of neonufft::gpu::Plan<T, DIM>."""

    def __init__(self, opt: Options, sign: int, num_nu: int, loc: Sequence, modes: Sequence[int],
                 stream=None, device_alloc=None, dtype=None):
        lib = L.load()
        self.dim = len(modes)
        if len(loc) != self.dim:
            raise InputError("loc and modes must have the same length")
        self.precision = _precision(dtype, loc)
        self.modes = [int(m) for m in modes]
        self.num_nu = int(num_nu)
        self._stream = _stream(stream)
        self._alloc = _Alloc(device_alloc) if device_alloc is not None else None
        h = C.c_void_p()
        c_opt = opt.to_c() if opt is not None else Options().to_c()
        check(lib.nnb_plan_create(C.byref(h), self.precision, self.dim, C.byref(c_opt), int(sign),
                                  int(num_nu), L.ptr_array([_ptr(a) for a in loc]),
                                  L.i64_array(self.modes), self._stream,
                                  C.byref(self._alloc.c) if self._alloc else None))
        self._h = h

    def transform_type_1(self, inp, out, out_strides: Sequence[int]) -> None:
        check(L.load().nnb_plan_transform_type_1(self._h, _ptr(inp), _ptr(out),
                                                 L.i64_array(out_strides)))

    def transform_type_1_many(self, inp, out, count: int, out_strides: Sequence[int],
                              in_bdist: int = 0, out_bdist: int = 0) -> None:
        """`count` type-1 transforms of the plan's points (engine extension): vector v of `inp`
        at offset v * in_bdist (default: the number of points), its modes at v * out_bdist of
        `out` (default: the number of modes). Single-precision plans on the z-window kernels
        spread two vectors per pass."""
        nm = 1
        for m in self.modes:
            nm *= int(m)
        in_bdist = int(in_bdist) or int(self.num_nu)
        out_bdist = int(out_bdist) or nm
        check(L.load().nnb_plan_transform_type_1_many(self._h, int(count), _ptr(inp), in_bdist,
                                                      _ptr(out), out_bdist,
                                                      L.i64_array(out_strides)))

    def transform_type_2(self, inp, in_strides: Sequence[int], out) -> None:
        check(L.load().nnb_plan_transform_type_2(self._h, _ptr(inp), L.i64_array(in_strides),
                                                 _ptr(out)))

    def set_points(self, num_nu: int, loc: Sequence) -> None:
        self.num_nu = int(num_nu)
        check(L.load().nnb_plan_set_points(self._h, int(num_nu),
                                           L.ptr_array([_ptr(a) for a in loc])))

    # ---- engine extensions ----
    def info(self) -> dict:
        i = L.NnbPlanInfo()
        check(L.load().nnb_plan_info(self._h, C.byref(i)))
        return _info_dict(i)

    def enable_timing(self, on: bool = True) -> None:
        check(L.load().nnb_plan_enable_timing(self._h, int(on)))

    def stage_times(self, reset: bool = True) -> dict:
        ms = (C.c_double * 6)()
        cnt = (C.c_int64 * 6)()
        check(L.load().nnb_plan_stage_times(self._h, ms, cnt, int(reset)))
        return {s: (ms[i], cnt[i]) for i, s in enumerate(L.STAGES)}

    def close(self) -> None:
        if getattr(self, "_h", None):
            L.load().nnb_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PlanT3:
    """Type-3 plan: mirror of neonufft::gpu::PlanT3<T, DIM>.

    Construct either from point sets ``PlanT3(opt, sign, num_in, input_points, num_out,
    output_points, stream, batch_size)`` or from bounds with ``PlanT3.from_bounds``.
    """

    def __init__(self, opt: Options, sign: int, num_in: int, input_points: Sequence,
                 num_out: int, output_points: Sequence, stream=None, batch_size: int = 1,
                 device_alloc=None, dtype=None, _bounds=None):
        lib = L.load()
        self._stream = _stream(stream)
        self._alloc = _Alloc(device_alloc) if device_alloc is not None else None
        c_opt = opt.to_c() if opt is not None else Options().to_c()
        h = C.c_void_p()
        if _bounds is None:
            self.dim = len(input_points)
            self.precision = _precision(dtype, list(input_points) + list(output_points))
            check(lib.nnb_plan_t3_create(
                C.byref(h), self.precision, self.dim, C.byref(c_opt), int(sign), int(num_in),
                L.ptr_array([_ptr(a) for a in input_points]), int(num_out),
                L.ptr_array([_ptr(a) for a in output_points]), self._stream, int(batch_size),
                C.byref(self._alloc.c) if self._alloc else None))
        else:
            in_min, in_max, out_min, out_max = _bounds
            self.dim = len(in_min)
            self.precision = _precision(dtype, [])
            check(lib.nnb_plan_t3_create_bounds(
                C.byref(h), self.precision, self.dim, C.byref(c_opt), int(sign),
                L.f64_array(in_min), L.f64_array(in_max), L.f64_array(out_min),
                L.f64_array(out_max), self._stream, int(batch_size),
                C.byref(self._alloc.c) if self._alloc else None))
        self._h = h

    @classmethod
    def from_bounds(cls, opt: Options, sign: int, input_min, input_max, output_min, output_max,
                    stream=None, batch_size: int = 1, device_alloc=None, dtype=None) -> "PlanT3":
        return cls(opt, sign, 0, [], 0, [], stream=stream, batch_size=batch_size,
                   device_alloc=device_alloc, dtype=dtype,
                   _bounds=(input_min, input_max, output_min, output_max))

    @staticmethod
    def grid_memory_size(opt: Options, input_min, input_max, output_min, output_max,
                         dtype) -> int:
        size = C.c_uint64()
        c_opt = opt.to_c()
        check(L.load().nnb_plan_t3_grid_memory_size(
            _precision(dtype, []), len(input_min), C.byref(c_opt), L.f64_array(input_min),
            L.f64_array(input_max), L.f64_array(output_min), L.f64_array(output_max),
            C.byref(size)))
        return int(size.value)

    def set_input_points(self, num_in: int, input_points: Sequence) -> None:
        check(L.load().nnb_plan_t3_set_input_points(self._h, int(num_in),
                                                    L.ptr_array([_ptr(a) for a in input_points])))

    def set_output_points(self, num_out: int, output_points: Sequence) -> None:
        check(L.load().nnb_plan_t3_set_output_points(
            self._h, int(num_out), L.ptr_array([_ptr(a) for a in output_points])))

    def add_input(self, inp, bdist: int = 0) -> None:
        check(L.load().nnb_plan_t3_add_input(self._h, _ptr(inp), int(bdist)))

    def transform(self, out, bdist: int = 0) -> None:
        check(L.load().nnb_plan_t3_transform(self._h, _ptr(out), int(bdist)))

    def reset(self) -> None:
        check(L.load().nnb_plan_t3_reset(self._h))

    def info(self) -> dict:
        i = L.NnbPlanInfo()
        check(L.load().nnb_plan_t3_info(self._h, C.byref(i)))
        return _info_dict(i)

    def enable_timing(self, on: bool = True) -> None:
        check(L.load().nnb_plan_t3_enable_timing(self._h, int(on)))

    def stage_times(self, reset: bool = True) -> dict:
        ms = (C.c_double * 6)()
        cnt = (C.c_int64 * 6)()
        check(L.load().nnb_plan_t3_stage_times(self._h, ms, cnt, int(reset)))
        return {s: (ms[i], cnt[i]) for i, s in enumerate(L.STAGES)}

    def close(self) -> None:
        if getattr(self, "_h", None):
            L.load().nnb_plan_t3_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _info_dict(i: L.NnbPlanInfo) -> dict:
    return {
        "dim": i.dim, "precision": "float" if i.precision == L.NNB_FLOAT else "double",
        "n_spread": i.n_spread, "spread_method": i.spread_method, "es_beta": i.es_beta,
        "grid": list(i.grid), "spread_grid": list(i.spread_grid), "tile": list(i.tile),
        "num_in": i.num_in, "num_out": i.num_out, "batch_size": i.batch_size,
        "device_bytes": i.device_bytes, "input_offset": list(i.input_offset),
        "output_offset": list(i.output_offset), "gamma": list(i.gamma), "h": list(i.h),
    }


class Batch:
    """Many independent type-1 / type-2 transforms of uneven sizes run together (engine
    extension, nnb_batch_* in include/neonufft_gpu.h): one plan per transform on internal streams,
    executed serially, concurrently, or as one captured CUDA graph; the FUSED modes also run the
    z-window spreading / interpolation steps of all 3D transforms as persistent launches over one
    queue of their work items."""

    SERIAL, STREAMS, GRAPH = L.NNB_BATCH_SERIAL, L.NNB_BATCH_STREAMS, L.NNB_BATCH_GRAPH
    FUSED, FUSED_GRAPH = L.NNB_BATCH_FUSED, L.NNB_BATCH_FUSED_GRAPH

    def __init__(self, opt: Options, dtype, num_streams: int = 4, stream=None,
                 device_alloc=None):
        lib = L.load()
        self.precision = _precision(dtype, [])
        self._stream = _stream(stream)
        self._alloc = _Alloc(device_alloc) if device_alloc is not None else None
        self._opt = opt if opt is not None else Options()
        self._keep = []  # tensors whose pointers the batch holds
        h = C.c_void_p()
        c_opt = self._opt.to_c()
        check(lib.nnb_batch_create(C.byref(h), self.precision, C.byref(c_opt), int(num_streams),
                                   self._stream, C.byref(self._alloc.c) if self._alloc else None))
        self._h = h

    def add(self, type_: int, sign: int, loc: Sequence, modes: Sequence[int], inp, out,
            strides: Sequence[int], opt: Options = None) -> int:
        """Adds a transform; the batch keeps references to loc, inp and out."""
        idx = C.c_int64(0)
        c_opt = opt.to_c() if opt is not None else None
        num_nu = int(loc[0].numel()) if hasattr(loc[0], "numel") else 0
        check(L.load().nnb_batch_add(self._h, len(modes), int(type_), int(sign), num_nu,
                                     L.ptr_array([_ptr(a) for a in loc]), L.i64_array(modes),
                                     _ptr(inp), _ptr(out), L.i64_array(strides),
                                     C.byref(c_opt) if c_opt is not None else None,
                                     C.byref(idx)))
        self._keep.append((loc, inp, out))
        return idx.value

    def execute(self, mode: int = GRAPH) -> None:
        check(L.load().nnb_batch_execute(self._h, int(mode)))

    def __len__(self) -> int:
        n = C.c_int64(0)
        check(L.load().nnb_batch_size(self._h, C.byref(n)))
        return n.value

    def info(self, index: int) -> dict:
        i = L.NnbPlanInfo()
        check(L.load().nnb_batch_info(self._h, int(index), C.byref(i)))
        return _info_dict(i)

    def close(self) -> None:
        if getattr(self, "_h", None):
            L.load().nnb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- FP64 direct sums on the GPU (accuracy measurement) -------------------------------------
def direct_type1_f64(sign: int, loc: Sequence, c, modes_idx, out, stream=None) -> None:
    """out[s] = sum_j c[j] exp(i sign k_s . x_j); modes_idx is an int64 CUDA tensor (S, dim)."""
    dim = len(loc)
    check(L.load().nnb_direct_type1_f64(dim, int(sign), int(loc[0].numel()),
                                        L.ptr_array([_ptr(a) for a in loc]), _ptr(c),
                                        int(modes_idx.shape[0]), _ptr(modes_idx), _ptr(out),
                                        _stream(stream)))


def direct_type2_f64(sign: int, modes: Sequence[int], f, loc: Sequence, point_idx, out,
                     stream=None) -> None:
    dim = len(modes)
    check(L.load().nnb_direct_type2_f64(dim, int(sign), L.i64_array(modes), _ptr(f),
                                        L.ptr_array([_ptr(a) for a in loc]),
                                        int(point_idx.numel()), _ptr(point_idx), _ptr(out),
                                        _stream(stream)))


def direct_type3_f64(sign: int, in_loc: Sequence, c, out_loc: Sequence, target_idx, out,
                     stream=None) -> None:
    dim = len(in_loc)
    check(L.load().nnb_direct_type3_f64(dim, int(sign), int(in_loc[0].numel()),
                                        L.ptr_array([_ptr(a) for a in in_loc]), _ptr(c),
                                        L.ptr_array([_ptr(a) for a in out_loc]),
                                        int(target_idx.numel()), _ptr(target_idx), _ptr(out),
                                        _stream(stream)))


def kernel_launches() -> int:
    """Engine kernel launches issued by this process so far."""
    return int(L.load().nnb_kernel_launches())


def check_device_status() -> None:
    """Synchronises the device; raises GPUError if a bounded wait inside an engine kernel gave
    up since the last check (nnb_check_device_status)."""
    check(L.load().nnb_check_device_status())
