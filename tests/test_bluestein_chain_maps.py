"""CPU checks of the index maps the fused Bluestein chains use, run in numpy
on small lengths: the three-pass decomposition of gfft_threepass.cuh
(input m = (M1 M2) n1 + M2 m1 + m2, pass-1 twiddle W_L^{m k1}, pass-2
twiddle W_{M1 M2}^{m2 k'1}, output k = k1 + N1 k'1 + N1 M1 k'2) with the
hooks of kernels_bluestein_tp3.cu (chirp-weighted zero-padded pass-1 loads,
filter-product pass-3 stores in natural order, chirp and 1/L in the inverse
pass-3 stores of k < n), and the mixed chain of gfft_mixbs.cuh whose middle
tile runs the forward second pass and, on the inverse split M2 x M1, the
inverse first pass over the same columns.  Both against numpy's FFT
(plan_bluestein.go:7-58: chirp, FFT_L, filter, IFFT_L, chirp)."""
import numpy as np
import pytest


def _chirp(n):
    k = np.arange(n)
    return np.exp(-1j * np.pi * ((k * k) % (2 * n)) / n)


def _filter(n, L):
    w = _chirp(n)
    b = np.zeros(L, complex)
    b[:n] = np.conj(w)
    b[L - n + 1:] = np.conj(w[1:][::-1])
    return np.fft.fft(b)


def _three_pass(x, N1, M1, M2, sign, load=None, store=None):
    """One three-pass FFT of length L = N1 M1 M2 (sign -1 forward, +1
    inverse unscaled), pass-1 loads through load(m) and pass-3 stores through
    store(k, value) when given."""
    L, M = N1 * M1 * M2, M1 * M2
    idx = np.arange(L)
    a = load(idx) if load else x
    A = a.reshape(N1, M)  # [n1, m]
    Y = np.fft.fft(A, axis=0) if sign < 0 else np.fft.ifft(A, axis=0) * N1
    k1, m = np.meshgrid(np.arange(N1), np.arange(M), indexing="ij")
    Y = Y * np.exp(sign * 2j * np.pi * m * k1 / L)  # W_L^{m k1}
    Yr = Y.T.reshape(M1, M2, N1)  # [m1, m2, k1]: Y[m][k1], m = M2 m1 + m2
    Z = np.fft.fft(Yr, axis=0) if sign < 0 else np.fft.ifft(Yr, axis=0) * M1
    kp1, m2 = np.meshgrid(np.arange(M1), np.arange(M2), indexing="ij")
    Z = Z * np.exp(sign * 2j * np.pi * m2 * kp1 / M)[:, :, None]  # W_M^{m2 k'1}
    W = np.fft.fft(Z, axis=1) if sign < 0 else np.fft.ifft(Z, axis=1) * M2  # [k'1, k'2, k1]
    out = np.empty(L, complex)
    kk1, kkp1, kkp2 = np.meshgrid(np.arange(N1), np.arange(M1), np.arange(M2), indexing="ij")
    k = kk1 + N1 * kkp1 + N1 * M1 * kkp2
    out[k.ravel()] = W.transpose(2, 0, 1)[kk1, kkp1, kkp2].ravel()
    if store:
        return store(np.arange(L), out)
    return out


@pytest.mark.parametrize("split", [(4, 4, 4), (8, 4, 4), (8, 8, 4), (4, 2, 8)])
def test_three_pass_maps_match_fft(split):
    rng = np.random.default_rng(sum(split))
    x = rng.standard_normal(int(np.prod(split))) + 1j * rng.standard_normal(int(np.prod(split)))
    assert np.allclose(_three_pass(x, *split, -1), np.fft.fft(x), atol=1e-10)
    assert np.allclose(_three_pass(x, *split, +1), np.fft.ifft(x) * x.size, atol=1e-10)


@pytest.mark.parametrize("n,split", [(31, (4, 4, 4)), (61, (8, 4, 4)), (97, (4, 8, 8)), (127, (8, 8, 4))])
@pytest.mark.parametrize("inverse", [False, True])
def test_three_pass_bluestein_chain(n, split, inverse):
    """FWD1 (chirp-weighted, zero-padded loads), plain passes, FWD3 (stores
    Z_k = A_k F_k), plain inverse passes, INV3 (stores w_k z_k / L for
    k < n); the inverse transform takes conj(w), conj(F[(L - k) mod L]) and
    1/n."""
    L = int(np.prod(split))
    assert L >= 2 * n - 1
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    w, F = _chirp(n), _filter(n, L)
    if inverse:
        w, F = np.conj(w), np.conj(F[(L - np.arange(L)) % L])

    def load(m):
        a = np.zeros(L, complex)
        a[:n] = x * w
        return a[m]

    def filt(k, v):
        return v * F[k]

    z = _three_pass(None, *split, -1, load=load, store=filt)
    y = _three_pass(z, *split, +1) / L
    got = y[:n] * w * (1.0 / n if inverse else 1.0)
    want = np.fft.ifft(x) if inverse else np.fft.fft(x)
    assert np.allclose(got, want, atol=1e-9 * max(1.0, np.abs(want).max()))


@pytest.mark.parametrize("n,m1,m2", [(41, 8, 12), (70, 12, 12), (100, 14, 16)])
def test_mixed_chain_middle_tile(n, m1, m2):
    """gfft_mixbs.cuh: BSK_IN is the four-step's pass 1 over columns of M1
    (input m = M2 n1 + n2, times W_M^{n2 k1}, rows n2 of M1); BSK_MID runs
    column k1 of the forward pass 2 (length M2, output k = k1 + M1 k2),
    multiplies by F_k and runs the inverse FFT's pass 1 on the same column
    (the inverse split M2 rows of M1: its column k1, times W_M^{+k1 j2}),
    stored as rows k1 of M2; BSK_OUT is the inverse's pass 2 over columns of
    M1 (output k = j2 + M2 j1) with the chirp stores of k < n."""
    M = m1 * m2
    assert M >= 2 * n - 1
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    w, F = _chirp(n), _filter(n, M)
    a = np.zeros(M, complex)
    a[:n] = x * w
    # BSK_IN: columns n2 of the M1 x M2 matrix a[M2 n1 + n2]
    A = np.fft.fft(a.reshape(m1, m2), axis=0)  # [k1, n2]
    k1, n2 = np.meshgrid(np.arange(m1), np.arange(m2), indexing="ij")
    scratch = (A * np.exp(-2j * np.pi * n2 * k1 / M)).T  # rows n2 of M1: [n2, k1]
    # BSK_MID, column k1: forward over n2 -> k2, times F at k = k1 + M1 k2
    Zc = np.fft.fft(scratch, axis=0)  # [k2, k1]
    kk2, kk1 = np.meshgrid(np.arange(m2), np.arange(m1), indexing="ij")
    Zc = Zc * F[kk1 + m1 * kk2]
    # inverse pass 1 of the split M2 x M1 (input index k = M1 k2 + k1: column
    # k1, rows k2), times W_M^{+k1 j2}, rows k1 of M2
    I1 = np.fft.ifft(Zc, axis=0) * m2  # [j2, k1]
    j2, kc = np.meshgrid(np.arange(m2), np.arange(m1), indexing="ij")
    work = (I1 * np.exp(2j * np.pi * kc * j2 / M)).T  # [k1, j2]
    # BSK_OUT: columns j2 over k1 -> j1, output k = j2 + M2 j1
    O = np.fft.ifft(work, axis=0) * m1  # [j1, j2]
    jj1, jj2 = np.meshgrid(np.arange(m1), np.arange(m2), indexing="ij")
    y = np.empty(M, complex)
    y[(jj2 + m2 * jj1).ravel()] = O.ravel()
    got = w * y[:n] / M
    assert np.allclose(got, np.fft.fft(x), atol=1e-9 * np.abs(np.fft.fft(x)).max())
