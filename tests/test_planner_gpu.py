"""Learned planner on the GPU: the MLP kernels (inference, gradient,
training) against the CPU oracle, and plan creation with PlannerLearned."""
import ctypes

import numpy as np
import pytest

import algofft
import mlp as O  # oracle/mlp.py
from algofft import planner as P
from helpers import rel_l2, seeded_complex, tol_c2c

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _params(seed):
    rng = np.random.default_rng(seed)
    p = O.init(seed)
    p[O.H * O.D:O.H * O.D + O.H] = 0.1 * rng.standard_normal(O.H)  # nonzero biases
    return p


def test_forward_kernel_matches_oracle():
    import torch
    rng = np.random.default_rng(1)
    p = _params(1)
    X = rng.standard_normal((300, O.D)).astype(np.float32)
    out = torch.empty(300, dtype=torch.float32, device="cuda")
    dp, dx = _dev(p), _dev(X)  # held: a temporary's memory could be reused before the launch
    algofft.check(algofft.lib().gfft_mlp_forward(dp.data_ptr(), dx.data_ptr(), 300, out.data_ptr(), None))
    torch.cuda.synchronize()
    want = O.forward(p, X)
    assert np.max(np.abs(out.cpu().numpy() - want)) <= 1e-5 * (1 + np.max(np.abs(want)))


@pytest.mark.parametrize("n", [1, 7, 64])
def test_gradient_kernel_matches_oracle(n):
    import torch
    rng = np.random.default_rng(n)
    p = _params(2)
    X = rng.standard_normal((n, O.D)).astype(np.float32)
    y = rng.standard_normal(n).astype(np.float32)
    g = torch.empty(O.NP, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    dp, dx, dy = _dev(p), _dev(X), _dev(y)
    algofft.check(algofft.lib().gfft_mlp_grad(dp.data_ptr(), dx.data_ptr(), dy.data_ptr(), n, g.data_ptr(),
                                              loss.data_ptr(), None))
    torch.cuda.synchronize()
    want_loss, want = O.loss_and_grad(p, X, y)
    got = g.cpu().numpy()
    assert abs(loss.item() - want_loss) <= 1e-5 * (1 + want_loss)
    assert np.max(np.abs(got - want)) <= 1e-5 * (1 + np.max(np.abs(want)))
    assert rel_l2(got, want) <= 1e-5


def test_gradient_kernel_rejects_oversize_batch():
    import torch
    z = torch.zeros(O.NP * 65, dtype=torch.float32, device="cuda")
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.check(algofft.lib().gfft_mlp_grad(z.data_ptr(), z.data_ptr(), z.data_ptr(), 65, z.data_ptr(),
                                                  z.data_ptr(), None))


def _target(X):
    return (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] - 0.3 * X[:, 3] ** 2).astype(np.float32)


def test_training_is_deterministic_and_learns():
    rng = np.random.default_rng(4)
    X = rng.standard_normal((4000, O.D)).astype(np.float32)
    y = _target(X)
    a = P.train(X, y, steps=3000, seed=7)
    b = P.train(X, y, steps=3000, seed=7)
    assert np.array_equal(a.params, b.params)
    Xt = rng.standard_normal((1000, O.D)).astype(np.float32)
    yt = _target(Xt)
    pred = a.predict(Xt) * a.norm[-1] + a.norm[-2]
    mse = float(np.mean((pred - yt) ** 2))
    assert mse < 0.1 * float(np.var(yt)), mse
    # the GPU inference agrees with the oracle on the trained weights
    want = O.forward(a.params, a.standardize(Xt))
    assert np.max(np.abs(a.predict(Xt) - want)) <= 1e-4 * (1 + np.max(np.abs(want)))


def test_learned_plan_creation_picks_a_variant_and_transforms():
    import torch
    rng = np.random.default_rng(5)
    p = _params(5)
    norm = np.concatenate([np.zeros(O.D), np.ones(O.D), [0.0, 1.0]]).astype(np.float32)
    saved = algofft.ExportWisdomToString()
    algofft.ClearWisdom()
    try:
        P.Model(p, norm).install()
        for n in (4096, 1000, 65536):
            buf = ctypes.create_string_buffer(128)
            algofft.check(algofft.lib().gfft_planner_choose(0, n, 16, 1, 0, buf, 128))
            tok = buf.value.decode()
            assert tok in algofft.Variants(n)
            with algofft.NewPlanWithOptions(n, algofft.PlanOptions(Planner=algofft.PlannerLearned)) as pl:
                name = pl.Algorithm()
                assert name.startswith(tok.split("-m")[0]) or tok.startswith("gpu-sm100-bluestein") and "bluestein" in name
                x = seeded_complex(3 * n, seed=n)
                src = torch.from_numpy(x).cuda()
                dst = torch.empty_like(src)
                pl.ForwardBatch(dst, src, 3)
                torch.cuda.synchronize()
                assert rel_l2(dst.cpu().numpy()[:n], np.fft.fft(x[:n].astype(np.complex128))) <= 4 * tol_c2c(n, False)
    finally:
        algofft.check(algofft.lib().gfft_planner_set_model(None, None))
        algofft.ClearWisdom()
        algofft.ImportWisdomFromString(saved)


def test_learned_pick_covers_the_compiled_families():
    """With the shipped model, trained on shapes whose candidates include the
    compiled mixed-radix schedules: the pick for 7-smooth lengths is one of
    their variants, and a prime with both Bluestein FFT lengths gets one."""
    saved = algofft.ExportWisdomToString()
    algofft.ClearWisdom()
    P.Model.load(P.DEFAULT_MODEL).install()
    try:
        for n in (1000, 6000, 50421, 100000, 16411):
            # batch 0: unknown, as plan creation without PlanOptions.Batch asks
            buf = ctypes.create_string_buffer(128)
            algofft.check(algofft.lib().gfft_planner_choose(0, n, 0, 1, 0, buf, 128))
            tok = buf.value.decode()
            assert tok in algofft.Variants(n), (n, tok)
            with algofft.NewPlanWithOptions(n, algofft.PlanOptions(Planner=algofft.PlannerLearned)) as pl:
                assert pl.Algorithm().startswith(tok), (pl.Algorithm(), tok)
    finally:
        algofft.ClearWisdom()
        algofft.ImportWisdomFromString(saved)
