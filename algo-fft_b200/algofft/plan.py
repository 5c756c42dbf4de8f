"""1-D complex plans: the reference's Plan[T] surface (plan.go) over the C ABI.

Buffers are either host arrays (numpy; the Go-slice methods, executed
through the ``*_host`` entry points with copies inside the call) or device
tensors (torch CUDA; the gpu.Buffer path, queued on the current stream).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import ErrNilSlice, PlanOptionsC, check, lib

COMPLEX64, COMPLEX128 = 0, 1
PlannerEstimate, PlannerMeasure, PlannerPatient, PlannerExhaustive = range(4)
PlannerLearned = 4  # no counterpart in the reference: the learned cost model (algofft.planner)
KernelAuto, KernelDIT, KernelStockham, KernelSixStep, KernelEightStep, KernelBluestein, KernelRecursive = range(7)


@dataclass
class PlanOptions:
    """plan_options.go:46-76 PlanOptions (+ gpu/types.go DeviceIndex)."""
    Planner: int = PlannerEstimate
    Strategy: int = KernelAuto
    Batch: int = 0
    Stride: int = 0
    InPlace: bool = False
    Device: int = 0

    def to_c(self) -> PlanOptionsC:
        return PlanOptionsC(self.Planner, self.Strategy, self.Batch, self.Stride, int(self.InPlace), self.Device)


def _is_device(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _ptr_len(x):
    """(pointer, element count, is_device) of a numpy array or torch tensor."""
    if x is None:
        return None, 0, False
    if _is_device(x):
        if not x.is_contiguous():
            raise ValueError("device tensors must be contiguous")
        return ctypes.c_void_p(x.data_ptr()), x.numel(), True
    if isinstance(x, np.ndarray):
        if not x.flags.c_contiguous:
            raise ValueError("host arrays must be C-contiguous")
        return ctypes.c_void_p(x.ctypes.data), x.size, False
    raise TypeError(f"unsupported buffer type {type(x)}")


def _stream(x):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)


def _dtype_prec(dtype) -> int:
    s = str(dtype)
    if s.endswith("complex64"):
        return COMPLEX64
    if s.endswith("complex128"):
        return COMPLEX128
    raise TypeError(f"unsupported element type {dtype}")


class Plan:
    """Plan[T] (plan.go:18).  T is complex64 (precision 0) or complex128."""

    def __init__(self, n: int, precision: int = COMPLEX64, opts: PlanOptions | None = None,
                 variant: str | None = None):
        self._h = ctypes.c_void_p()
        self.precision = precision
        self._opts = opts or PlanOptions()
        if variant is not None:
            check(lib().gfft_plan_new_variant(ctypes.byref(self._h), precision, n, variant.encode()))
        else:
            c_opts = self._opts.to_c()
            check(lib().gfft_plan_new(ctypes.byref(self._h), precision, n, ctypes.byref(c_opts)))

    @classmethod
    def _wrap(cls, h, precision: int, opts: PlanOptions) -> "Plan":
        p = cls.__new__(cls)
        p._h, p.precision, p._opts = h, precision, opts
        return p

    def Check(self) -> None:
        """Raises ErrTimeout if a bounded device wait of this plan expired."""
        check(lib().gfft_plan_check(self._h))

    def Clone(self) -> "Plan":
        """plan.go:1300 Clone: an independent plan with the same schedule."""
        h = ctypes.c_void_p()
        check(lib().gfft_plan_clone(ctypes.byref(h), self._h))
        return Plan._wrap(h, self.precision, self._opts)

    def NewExecutor(self) -> "Executor":
        """executor.go:11 NewExecutor."""
        return Executor(self)

    # -- lifecycle ---------------------------------------------------------
    def Close(self) -> None:
        if self._h:
            lib().gfft_plan_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.Close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.Close()

    def Len(self) -> int:
        return int(lib().gfft_plan_len(self._h))

    def Algorithm(self) -> str:
        buf = ctypes.create_string_buffer(256)
        check(lib().gfft_plan_algorithm(self._h, buf, 256))
        return buf.value.decode()

    # -- execution ---------------------------------------------------------
    def _call(self, dev_fn, host_fn, dst, src, *extra):
        if dst is None or src is None:
            raise ErrNilSlice("algo-fft: nil slice")
        dp, dl, dd = _ptr_len(dst)
        sp, sl, sd = _ptr_len(src)
        if dd != sd:
            raise ValueError("dst and src must both be host arrays or both device tensors")
        for a in (dst, src):
            if _dtype_prec(a.dtype) != self.precision:
                raise TypeError("buffer element type does not match the plan precision")
        L = lib()
        if dd:
            check(getattr(L, dev_fn)(self._h, dp, dl, sp, sl, *extra, _stream(dst)))
        else:
            check(getattr(L, host_fn)(self._h, dp, dl, sp, sl, *extra))
        return None

    def Forward(self, dst, src):
        """plan.go:332 Forward: one transform, dst may alias src."""
        return self._call("gfft_forward", "gfft_forward_host", dst, src)

    def Inverse(self, dst, src):
        """plan.go:382 Inverse (scaled by 1/n)."""
        return self._call("gfft_inverse", "gfft_inverse_host", dst, src)

    def InPlace(self, data):
        """plan.go:427."""
        return self.Forward(data, data)

    def InverseInPlace(self, data):
        """plan.go:437."""
        return self.Inverse(data, data)

    def Transform(self, dst, src, inverse: bool):
        """plan.go:483."""
        return self.Inverse(dst, src) if inverse else self.Forward(dst, src)

    def ForwardBatch(self, dst, src, count: int):
        """plan.go:504 ForwardBatch: count transforms on [i*n, (i+1)*n)."""
        return self._call("gfft_forward_batch", "gfft_forward_batch_host", dst, src, count)

    def InverseBatch(self, dst, src, count: int):
        """plan.go:545 InverseBatch."""
        return self._call("gfft_inverse_batch", "gfft_inverse_batch_host", dst, src, count)

    def ForwardStrided(self, dst, src, stride: int):
        """plan_strided.go:16 (device buffers)."""
        return self._strided("gfft_forward_strided", dst, src, stride)

    def InverseStrided(self, dst, src, stride: int):
        """plan_strided.go:25 (device buffers)."""
        return self._strided("gfft_inverse_strided", dst, src, stride)

    def StridedBatch(self, dst, src, count: int, stride: int, dist: int, inverse: bool = False):
        """count transforms, element j of transform b at b*dist + j*stride (device buffers)."""
        dp, dl, dd = _ptr_len(dst)
        sp, sl, sd = _ptr_len(src)
        check(lib().gfft_exec_strided_batch(self._h, 1 if inverse else -1, dp, dl, sp, sl, count, stride, dist,
                                            _stream(dst)))

    def _strided(self, fn, dst, src, stride):
        if dst is None or src is None:
            raise ErrNilSlice("algo-fft: nil slice")
        dp, dl, dd = _ptr_len(dst)
        sp, sl, sd = _ptr_len(src)
        if not (dd and sd):
            import torch
            d = torch.from_numpy(np.ascontiguousarray(dst)).cuda()
            s = torch.from_numpy(np.ascontiguousarray(src)).cuda()
            self._strided(fn, d, s, stride)
            torch.cuda.synchronize()
            dst[...] = d.cpu().numpy()
            return None
        check(getattr(lib(), fn)(self._h, dp, dl, sp, sl, stride, _stream(dst)))
        return None


class Executor:
    """Executor[T] (executor.go:11-40): one caller's handle on a plan.  The
    GPU plan is reentrant (no shared scratch), so an executor's part is its
    own CUDA stream: device calls run on it, ordered after the caller's
    current stream and joined back into it, so executors of one plan run
    concurrently.  Host buffers take the synchronous host path."""

    def __init__(self, plan: Plan):
        self.plan = plan
        self._stream = None

    def _run(self, fn, *args):
        if not _is_device(args[0]):
            return fn(*args)
        import torch
        if self._stream is None:
            self._stream = torch.cuda.Stream(device=args[0].device)
        cur = torch.cuda.current_stream(args[0].device)
        self._stream.wait_stream(cur)
        with torch.cuda.stream(self._stream):
            fn(*args)
        cur.wait_stream(self._stream)
        return None

    def Forward(self, dst, src):
        """executor.go:16."""
        return self._run(self.plan.Forward, dst, src)

    def Inverse(self, dst, src):
        """executor.go:21."""
        return self._run(self.plan.Inverse, dst, src)

    def ForwardInPlace(self, data):
        """executor.go:26."""
        return self._run(self.plan.InPlace, data)

    def InverseInPlace(self, data):
        """executor.go:31."""
        return self._run(self.plan.InverseInPlace, data)

    def Close(self) -> None:
        """executor.go:36 (the plan stays open)."""
        self._stream = None


def SetKernelStrategy(strategy: int) -> None:
    """plan.go:112 SetKernelStrategy (process-wide)."""
    lib().gfft_set_kernel_strategy(strategy)


def GetKernelStrategy() -> int:
    """plan.go:117 GetKernelStrategy."""
    return int(lib().gfft_get_kernel_strategy())


def RecordBenchmarkDecision(n: int, strategy: int) -> None:
    """plan.go:122 RecordBenchmarkDecision."""
    lib().gfft_record_benchmark_decision(n, strategy)


def NewPlanT(n: int, precision: int = COMPLEX64) -> Plan:
    """plan.go:596 NewPlanT[T]."""
    return Plan(n, precision)


def NewPlan(n: int) -> Plan:
    """plan.go:1013 NewPlan (complex64)."""
    return Plan(n, COMPLEX64)


def NewPlan32(n: int) -> Plan:
    """plan.go:1019 NewPlan32."""
    return Plan(n, COMPLEX64)


def NewPlan64(n: int) -> Plan:
    """plan.go:1025 NewPlan64 (complex128)."""
    return Plan(n, COMPLEX128)


def NewPlanWithOptions(n: int, opts: PlanOptions, precision: int = COMPLEX64) -> Plan:
    """plan.go:601 NewPlanWithOptions."""
    return Plan(n, precision, opts)
