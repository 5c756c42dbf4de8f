"""The reference's plan helpers: FastPlan (plan_fast.go), pooled plans
(plan.go:1040-1118) and the Planner (planner.go:5-74), over the same C ABI."""
from __future__ import annotations

import ctypes

from ._lib import ErrInvalidLength, check, lib
from .nd import NewPlan2D, NewPlan3D, NewPlanReal2D, PlanND
from .plan import COMPLEX64, COMPLEX128, Plan, PlanOptions
from .real import PlanReal


class FastPlan:
    """FastPlan[T] (plan_fast.go:46-135): power-of-two lengths only; the
    transforms check nothing beyond the plan's own arguments."""

    def __init__(self, n: int, precision: int = COMPLEX64):
        if n < 1 or n & (n - 1):
            raise ErrInvalidLength("algo-fft: invalid FFT length")
        self._p = Plan(n, precision)

    def Len(self) -> int:
        return self._p.Len()

    def Forward(self, dst, src):
        self._p.Forward(dst, src)

    def Inverse(self, dst, src):
        self._p.Inverse(dst, src)

    def InPlace(self, data):
        self._p.InPlace(data)

    def InverseInPlace(self, data):
        self._p.InverseInPlace(data)

    def Close(self):
        self._p.Close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.Close()


def NewFastPlan(n: int, precision: int = COMPLEX64) -> FastPlan:
    """plan_fast.go:46."""
    return FastPlan(n, precision)


def NewPlanPooledWithOptions(n: int, opts: PlanOptions | None = None, precision: int = COMPLEX64) -> Plan:
    """plan.go:1045: Close returns the plan to the pool of its shape."""
    o = opts or PlanOptions()
    h = ctypes.c_void_p()
    c = o.to_c()
    check(lib().gfft_plan_new_pooled(ctypes.byref(h), precision, n, ctypes.byref(c)))
    return Plan._wrap(h, precision, o)


def NewPlanPooled(n: int, precision: int = COMPLEX64) -> Plan:
    """plan.go:1040."""
    return NewPlanPooledWithOptions(n, None, precision)


def ClearPlanPool() -> None:
    """Frees every pooled plan (a process-wide cache)."""
    lib().gfft_plan_pool_clear()


class Planner:
    """Planner (planner.go:5-74): plan constructors sharing one PlanOptions."""

    def __init__(self, opts: PlanOptions | None = None):
        self.opts = opts or PlanOptions()

    def Plan1D32(self, n: int) -> Plan:
        return Plan(n, COMPLEX64, self.opts)

    def Plan1D64(self, n: int) -> Plan:
        return Plan(n, COMPLEX128, self.opts)

    def Plan2D32(self, rows: int, cols: int) -> PlanND:
        return NewPlan2D(rows, cols, COMPLEX64, self.opts)

    def Plan2D64(self, rows: int, cols: int) -> PlanND:
        return NewPlan2D(rows, cols, COMPLEX128, self.opts)

    def Plan3D32(self, depth: int, rows: int, cols: int) -> PlanND:
        return NewPlan3D(depth, rows, cols, COMPLEX64, self.opts)

    def Plan3D64(self, depth: int, rows: int, cols: int) -> PlanND:
        return NewPlan3D(depth, rows, cols, COMPLEX128, self.opts)

    def PlanND32(self, dims) -> PlanND:
        return PlanND(tuple(dims), COMPLEX64, False, self.opts)

    def PlanND64(self, dims) -> PlanND:
        return PlanND(tuple(dims), COMPLEX128, False, self.opts)

    def PlanReal(self, n: int) -> PlanReal:
        return PlanReal(n, COMPLEX64, self.opts)

    def PlanReal2D(self, rows: int, cols: int) -> PlanND:
        return NewPlanReal2D(rows, cols, self.opts)


def NewPlanner(opts: PlanOptions | None = None) -> Planner:
    """planner.go:12."""
    return Planner(opts)


def Plan1D(p: Planner, n: int, precision: int = COMPLEX64) -> Plan:
    """planner.go:22 Plan1D[T]."""
    return Plan(n, precision, p.opts)
