"""CPU checks of the compiled mixed-radix column tiles: the committed
kernels_mixcols_t*.cu files are what gen_mixcols.py writes, every table
entry fits its launch limits, and the Stockham index maps the tiles use
(gfft_mixcols.cuh: butterfly i of stage s reads rows i + r L/R_s, takes
W_L^{r k L/(P_s R_s)} with k = i mod P_s, writes rows (i - k) R_s + k + r P_s)
reproduce numpy's FFT for every schedule in the table."""
import importlib.util
import os

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(__file__), "..", "algo-fft_b200", "csrc")


def _gen():
    spec = importlib.util.spec_from_file_location("gen_mixcols", os.path.join(CSRC, "gen_mixcols.py"))
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    return g


def test_generated_files_are_current(tmp_path):
    g = _gen()
    g.main(str(tmp_path))
    names = ([f"kernels_mixcols_t{k}.cu" for k in range(g.PARTS)] + [f"kernels_mixbs_t{k}.cu" for k in range(g.BS_PARTS)]
             + [f"kernels_mixrows_t{k}.cu" for k in range(g.ROW_PARTS)])
    for name in names:
        with open(os.path.join(CSRC, name)) as a, open(tmp_path / name) as b:
            assert a.read() == b.read(), f"{name} is stale: run gen_mixcols.py"


def test_bluestein_lengths_are_table_lengths():
    g = _gen()
    bs = g.bs_lengths()
    assert bs == [80] + [L for L in range(112, 513) if g.smooth7(L) and L % 16 == 0] and len(bs) == 18
    assert max(bs) ** 2 == 1 << 18  # FFT lengths up to 2^18: n up to 131072


def _primes(n):
    sieve = np.ones(n + 1, bool)
    sieve[:2] = False
    for i in range(2, int(n ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    return [int(p) for p in np.nonzero(sieve)[0]]


def _bs_split(bs, n):
    """(M, M1) as bs_mixed_length (kernels_mixcols.cu) picks them: the
    smallest product M1 x M2 >= 2n - 1 of table lengths, M1 <= M2, the most
    balanced among equal products."""
    best, a_best = 0, 0
    for i, a in enumerate(bs):
        for b in bs[i:]:
            m = a * b
            if m >= 2 * n - 1 and (best == 0 or m < best or (m == best and a > a_best)):
                best, a_best = m, a
    return best, a_best


def test_bluestein_sweep_covers_every_factor_role():
    """The GPU sweep's primes run every Bluestein factor length in every
    role (M1: BSK_IN and BSK_OUT, M2: BSK_MID) that some prime beyond the
    one-CTA range reaches on the mixed chain."""
    import importlib
    g = _gen()
    bs = g.bs_lengths()
    sweep = importlib.import_module("test_mixcols_sweep_gpu").BS_PRIMES
    reach, got = set(), set()
    for n in _primes(131072):
        if n <= 8192:
            continue
        M, a = _bs_split(bs, n)
        if M and M < 1 << (2 * n - 2).bit_length():
            roles = {(a, 1), (M // a, 2)}
            reach |= roles
            if n in sweep:
                got |= roles
    assert got == reach
    assert {L for L, r in reach if r == 1} == set(bs) - {512}
    assert {L for L, r in reach if r == 2} == set(bs) - {80, 112, 128}


def test_every_length_has_a_launchable_plan():
    g = _gen()
    lengths = [L for L in range(48, 1025) if g.smooth7(L)]
    assert len(lengths) == 115
    for L in lengths:
        for es, pass_ in ((8, 1), (8, 2), (16, 1), (16, 2)):
            sched, nc, minb, tt = g.plan(L, es, pass_=pass_)
            three = L in g.THREE[es] or (pass_ == 2 and L in g.THREE2[es])
            assert int(np.prod(sched)) == L and len(sched) == (3 if three else 2)
            assert all(g.radix_ok(r) for r in sched)
            T = tt if tt else L // max(sched)
            assert T * nc <= 1024 and 1 <= minb <= 8
            pitch = nc + 1 if nc >= 16 else nc
            assert max(L * pitch, nc * (L | 1)) * es <= 200 * 1024


def test_rows_plans_fit_their_launch_limits():
    g = _gen()
    assert len(g.rows3_lengths(8)) == 218 and max(g.rows3_lengths(16)) <= 6144
    for L in [L for L in range(48, 1025) if g.smooth7(L)] + g.rows3_lengths(8):
        for es in (8, 16):
            if L > 1024 and L not in g.rows3_lengths(es):
                continue
            if L > 1024:
                assert int(np.prod(g.schedule3(L))) == L
            sched, nc, minb, tt = g.rows_plan(L, es)
            T = tt if tt else L // max(sched)
            assert nc & (nc - 1) == 0 and 1 <= nc <= 64 and T * nc <= 1024 and minb * T * nc <= 2048
            assert nc * g.rows_pitch(L, sched) * es <= (64 if nc > 1 else 200) * 1024


def _stockham(x, sched, T):
    """The tile's stage loop on one column, thread by thread (threads t < T,
    butterflies t, t + T, ...)."""
    L = x.size
    cur = x.astype(np.complex128)
    P = 1
    for R in sched:
        nb = L // R
        out = np.empty_like(cur)
        for t in range(T):
            for i in range(t, nb, T):
                k = i % P
                v = cur[i + nb * np.arange(R)]
                v = v * np.exp(-2j * np.pi * np.arange(R) * k * (L // (P * R)) / L)
                v = np.fft.fft(v)
                out[(i - k) * R + k + P * np.arange(R)] = v
        cur = out
        P *= R
    return cur


def test_three_stage_index_maps_match_fft():
    g = _gen()
    rng = np.random.default_rng(7)
    for L in g.rows3_lengths(8)[::11]:
        sched = g.schedule3(L)
        x = rng.standard_normal(L) + 1j * rng.standard_normal(L)
        got = _stockham(x, sched, L // max(sched))
        assert np.linalg.norm(got - np.fft.fft(x)) <= 1e-12 * np.linalg.norm(x) * np.sqrt(L), (L, sched)


@pytest.mark.parametrize("es", [8, 16])
def test_index_maps_match_fft(es):
    g = _gen()
    rng = np.random.default_rng(5)
    for L in [L for L in range(48, 1025) if g.smooth7(L)][::3]:
        sched, nc, minb, tt = g.plan(L, es)
        T = tt if tt else L // max(sched)
        x = rng.standard_normal(L) + 1j * rng.standard_normal(L)
        got = _stockham(x, sched, T)
        want = np.fft.fft(x)
        assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want), (L, sched, T)
