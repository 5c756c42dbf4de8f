"""Clone, Executor, pooled plans, FastPlan and the Planner helpers
(plan.go:1040-1118,1300, executor.go:11-40, plan_fast.go:46-135,
planner.go:5-74) over the GPU plans."""
import threading

import numpy as np
import pytest

import algofft
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("n", [1, 1024, 1 << 16, 1 << 21, 6000, 1009])
def test_clone_is_independent_and_identical(n):
    import torch
    x = seeded_complex(2 * n, seed=n % 7)
    p = algofft.NewPlan(n)
    c = p.Clone()
    assert c.Algorithm() == p.Algorithm() and c.Len() == n
    src = _dev(x)
    a, b = torch.empty_like(src), torch.empty_like(src)
    p.ForwardBatch(a, src, 2)
    p.Close()  # the clone outlives the original
    c.ForwardBatch(b, src, 2)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    c.Close()


def test_executors_run_concurrently_and_match_the_plan():
    import torch
    n, count = 4096, 8
    xs = [seeded_complex(n * count, seed=i) for i in range(4)]
    with algofft.NewPlan(n) as p:
        want = []
        for x in xs:
            y = torch.empty(n * count, dtype=torch.complex64, device="cuda")
            p.ForwardBatch(y, _dev(x), count)
            want.append(y)
        outs = [None] * 4

        def work(i):
            e = p.NewExecutor()
            src = _dev(xs[i])
            dst = torch.empty_like(src)
            for j in range(count):
                e.Forward(dst[j * n:(j + 1) * n], src[j * n:(j + 1) * n])
            e.ForwardInPlace(src[:n])
            torch.cuda.synchronize()
            outs[i] = (dst, src[:n].clone())
            e.Close()

        ts = [threading.Thread(target=work, args=(i,)) for i in range(4)]
        [t.start() for t in ts]
        [t.join() for t in ts]
    for i in range(4):
        assert torch.equal(outs[i][0], want[i])
        assert torch.equal(outs[i][1], want[i][:n])
    # host buffers take the synchronous path
    with algofft.NewPlan(64) as p:
        e = p.NewExecutor()
        x = seeded_complex(64, seed=1)
        y = np.empty_like(x)
        e.Forward(y, x)
        e.InverseInPlace(y)
        assert rel_l2(y, x) <= 2 * tol_c2c(64, False)


def test_pooled_plans_are_reused():
    algofft.ClearPlanPool()
    a = algofft.NewPlanPooled(2048)
    ha = a._h.value
    a.Close()  # back to the pool
    b = algofft.NewPlanPooled(2048)
    assert b._h.value == ha  # the same plan, tables not rebuilt
    c = algofft.NewPlanPooled(2048)  # pool empty: a new one
    assert c._h.value != ha
    x = seeded_complex(2048, seed=3)
    y = np.empty_like(x)
    b.Forward(y, x)
    assert rel_l2(y, np.fft.fft(x.astype(np.complex128))) <= tol_c2c(2048, False)
    b.Close()
    c.Close()
    d = algofft.NewPlanPooled(2048, algofft.COMPLEX128)  # another key
    assert d._h.value not in (ha, c._h.value)
    d.Close()
    algofft.ClearPlanPool()


def test_fast_plan():
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.NewFastPlan(1000)
    with algofft.NewFastPlan(256) as f:
        assert f.Len() == 256
        x = seeded_complex(256, seed=9)
        y = np.empty_like(x)
        f.Forward(y, x)
        assert rel_l2(y, np.fft.fft(x.astype(np.complex128))) <= tol_c2c(256, False)
        f.InverseInPlace(y)
        assert rel_l2(y, x) <= 2 * tol_c2c(256, False)


def test_planner_helpers_share_options():
    pl = algofft.NewPlanner(algofft.PlanOptions(Strategy=algofft.KernelBluestein))
    with pl.Plan1D32(512) as p:
        assert "bluestein" in p.Algorithm()
    with algofft.Plan1D(pl, 100, algofft.COMPLEX128) as p:
        x = seeded_complex(100, seed=2, dtype=np.complex128)
        y = np.empty_like(x)
        p.Forward(y, x)
        assert rel_l2(y, np.fft.fft(x)) <= tol_c2c(100, True)
    pl2 = algofft.NewPlanner()
    with pl2.Plan2D32(8, 16) as p2, pl2.Plan3D64(4, 4, 4) as p3, pl2.PlanReal(64) as pr, \
            pl2.PlanReal2D(8, 8) as prr, pl2.PlanND32((2, 3, 4)) as pnd:
        assert p2.Len() == 128 and p3.Len() == 64 and pr.Len() == 64 and prr.Len() == 64 and pnd.Len() == 24


def test_global_kernel_strategy_and_recorded_decisions():
    # plan.go:110-125: the process-wide strategy steers plans created with
    # KernelAuto; recorded per-length decisions apply under auto selection
    saved = algofft.ExportWisdomToString()
    algofft.ClearWisdom()
    try:
        assert algofft.GetKernelStrategy() == algofft.KernelAuto
        algofft.SetKernelStrategy(algofft.KernelBluestein)
        assert algofft.GetKernelStrategy() == algofft.KernelBluestein
        with algofft.NewPlan(1024) as p:
            assert "bluestein" in p.Algorithm()  # its inner FFT_M stays a normal plan
            x = seeded_complex(1024, seed=4)
            y = np.empty_like(x)
            p.Forward(y, x)
            assert rel_l2(y, np.fft.fft(x.astype(np.complex128))) <= tol_c2c(1024, False)
        algofft.SetKernelStrategy(algofft.KernelAuto)
        algofft.RecordBenchmarkDecision(8192, algofft.KernelSixStep)
        algofft.RecordBenchmarkDecision(4096, algofft.KernelBluestein)  # not a recordable class: ignored
        with algofft.NewPlan(8192) as p:
            assert "-tp-" in p.Algorithm()
        with algofft.NewPlan(4096) as p:
            assert "-p2-" in p.Algorithm()
        algofft.RecordBenchmarkDecision(8192, algofft.KernelStockham)
        with algofft.NewPlan(8192) as p:
            assert "-p2-" in p.Algorithm()
    finally:
        algofft.SetKernelStrategy(algofft.KernelAuto)
        algofft.ClearWisdom()
        algofft.ImportWisdomFromString(saved)
