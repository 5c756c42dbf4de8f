"""algofft — the reference's Go API (CWBudde/algo-fft) over the sm_100a
engine's C ABI (include/gfft.h).

Importing this package loads ``libgfft.so`` from the package directory;
there is no CPU fallback: if the library is missing the import fails.
"""
from ._lib import (ErrCuda, ErrInvalidArgument, ErrInvalidLength, ErrInvalidSpectrum, ErrInvalidStride,
                   ErrLengthMismatch, ErrNilSlice, ErrNoDevice, ErrNotImplemented, ErrOutOfMemory, ErrTimeout,
                   ErrWisdom, GfftError, LIB_PATH, check, lib)
from .plan import (COMPLEX64, COMPLEX128, Executor, GetKernelStrategy, KernelAuto, KernelBluestein, KernelDIT, KernelEightStep, KernelRecursive,
                   KernelSixStep, KernelStockham, NewPlan, NewPlan32, NewPlan64, NewPlanT, NewPlanWithOptions, Plan,
                   PlanOptions, PlannerEstimate, RecordBenchmarkDecision, SetKernelStrategy, PlannerExhaustive, PlannerLearned, PlannerMeasure,
                   PlannerPatient)

from .distributed import PlanDistributed
from .convolve import (AutoCorrelate, AutoCorrelate128, Convolve, Convolve128, ConvolveReal, ConvolveRealBatch,
                       Correlate, Correlate128, CrossCorrelate, CrossCorrelate128)
from .nd import NewPlan2D, NewPlan3D, NewPlanND, NewPlanReal2D, NewPlanReal3D, PlanND
from .plan_helpers import (ClearPlanPool, FastPlan, NewFastPlan, NewPlanner, NewPlanPooled,
                           NewPlanPooledWithOptions, Plan1D, Planner)
from .real import NewPlanReal, NewPlanReal32, NewPlanReal64, NewPlanRealWithOptions, PlanReal
from .uneven import PlanUneven, uneven_lengths
from .wisdom import (Autotune, ClearWisdom, ExportWisdom, ExportWisdomToString, ImportWisdom,
                     ImportWisdomFromString, Variants, WisdomLen)

lib()  # fail loudly at import when the native library is absent


def device_count() -> int:
    import ctypes
    n = ctypes.c_int32(0)
    check(lib().gfft_device_count(ctypes.byref(n)))
    return n.value
