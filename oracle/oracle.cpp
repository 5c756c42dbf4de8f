// CPU oracle for the batched-transform path.  TEST INFRASTRUCTURE ONLY.
//
// This file is the checker: it is linked by the tests, by the smoke check
// and by the CPU-baseline leg of the benchmark, never by the product
// library.  It restates, in C++, the reference's CPU algorithms for the path
// (CWBudde/algo-fft, pure-Go build) plus an FP64 naive DFT arbiter.  Each
// function cites the reference file:line it follows.
//
// Parity pinning: the reference is Go and no Go toolchain exists on either
// machine, so the reference cannot be run here.  This restatement is pinned
// instead against the reference's own known-answer tests (impulse, constant,
// sinusoid, Nyquist, R2C impulse/constant/cosine, Convolve/ConvolveReal
// basic cases) which live as committed fixtures under tests/golden, and
// against numpy's pocketfft as an independent FFT.
//
// Arithmetic follows Go's rules on amd64: complex64 products are evaluated
// in float32 as (ac-bd, ad+bc) without FMA contraction (built with
// -ffp-contract=off).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <atomic>
#include <thread>

namespace {

// Splits [0, count) into contiguous ranges, one per thread (the reference's
// "one Executor per goroutine over disjoint batch ranges", executor.go:11).
template <typename F>
void parallel_for(int64_t count, int nthreads, F&& body) {
  if (nthreads <= 1 || count <= 1) {
    for (int64_t i = 0; i < count; ++i) body(i);
    return;
  }
  int nt = int(std::min<int64_t>(nthreads, count));
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    int64_t lo = count * t / nt, hi = count * (t + 1) / nt;
    th.emplace_back([lo, hi, &body]() { for (int64_t i = lo; i < hi; ++i) body(i); });
  }
  for (auto& x : th) x.join();
}

template <typename R>
struct cx {
  R re, im;
};
template <typename R>
inline cx<R> operator+(cx<R> a, cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R>
inline cx<R> operator-(cx<R> a, cx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R>
inline cx<R> operator*(cx<R> a, cx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>
inline cx<R> conj(cx<R> a) { return {a.re, -a.im}; }

constexpr double kPi = 3.14159265358979323846264338327950288;

inline bool is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }
inline int ilog2(int64_t n) { int l = 0; while ((int64_t(1) << l) < n) ++l; return l; }
inline int64_t next_pow2(int64_t n) { int64_t m = 1; while (m < n) m <<= 1; return m; }

// internal/math/factor.go:30-43 IsHighlyComposite: only factors 2, 3, 5.
inline bool is_235_smooth(int64_t n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5}) while (n % p == 0) n /= p;
  return n == 1;
}

// internal/math/twiddle.go:8-21 ComputeTwiddleFactors: W_n^k = exp(-2πik/n),
// angle computed in float64, then cast to the element precision.
template <typename R>
std::vector<cx<R>> twiddles(int64_t n) {
  std::vector<cx<R>> tw(n);
  for (int64_t k = 0; k < n; ++k) {
    double angle = -2.0 * kPi * double(k) / double(n);
    tw[k] = {R(std::cos(angle)), R(std::sin(angle))};
  }
  return tw;
}

// internal/math/bitrev.go ComputeBitReversalIndices (radix-2 bit reversal).
std::vector<int64_t> bitrev(int64_t n) {
  int bits = ilog2(n);
  std::vector<int64_t> r(n);
  for (int64_t i = 0; i < n; ++i) {
    int64_t v = 0, x = i;
    for (int b = 0; b < bits; ++b) { v = (v << 1) | (x & 1); x >>= 1; }
    r[i] = v;
  }
  return r;
}

// internal/kernels/dit.go:204-330 ditForward/ditInverse: radix-2
// decimation-in-time with an explicit bit-reversal gather, twiddle
// twiddle[j*step] (conjugated for the inverse), inverse scaled by 1/n.
template <typename R>
void dit(cx<R>* dst, const cx<R>* src, const cx<R>* tw, int64_t n, bool inverse) {
  if (n == 1) { dst[0] = src[0]; return; }
  std::vector<cx<R>> work(n);
  std::vector<int64_t> br = bitrev(n);
  for (int64_t i = 0; i < n; ++i) work[i] = src[br[i]];
  for (int64_t size = 2; size <= n; size <<= 1) {
    int64_t half = size >> 1, step = n / size;
    for (int64_t base = 0; base < n; base += size) {
      for (int64_t j = 0; j < half; ++j) {
        cx<R> w = tw[j * step];
        if (inverse) w = conj(w);
        // internal/kernels/dit.go:465 butterfly2: (a + w*b, a - w*b)
        cx<R> a = work[base + j], b = work[base + j + half] * w;
        work[base + j] = a + b;
        work[base + j + half] = a - b;
      }
    }
  }
  if (inverse) {
    R s = R(1.0 / double(n));
    for (int64_t i = 0; i < n; ++i) work[i] = work[i] * cx<R>{s, 0};
  }
  std::memcpy(dst, work.data(), sizeof(cx<R>) * n);
}

// internal/kernels/stockham.go:21-100 radix-2 Stockham (forward): stages
// m = n, n/2, ..., 2; outLo = a+b, outHi = (a-b)*tw[j*step].  The inverse
// uses the conjugate twiddle and scales by 1/n (stockham.go:182-185).
template <typename R>
void stockham2(cx<R>* dst, const cx<R>* src, const cx<R>* tw, int64_t n, bool inverse) {
  if (n == 1) { dst[0] = src[0]; return; }
  std::vector<cx<R>> a(src, src + n), b(n);
  int stages = ilog2(n);
  int64_t halfN = n >> 1;
  for (int s = 0; s < stages; ++s) {
    int64_t m = int64_t(1) << (stages - s), half = m >> 1, step = n / m;
    for (int64_t k = 0; k < n / m; ++k) {
      for (int64_t j = 0; j < half; ++j) {
        cx<R> x = a[k * m + j], y = a[k * m + j + half];
        cx<R> w = tw[j * step];
        if (inverse) w = conj(w);
        b[k * half + j] = x + y;
        b[k * half + halfN + j] = (x - y) * w;
      }
    }
    std::swap(a, b);
  }
  if (inverse) {
    R sc = R(1.0 / double(n));
    for (auto& v : a) v = v * cx<R>{sc, 0};
  }
  std::memcpy(dst, a.data(), sizeof(cx<R>) * n);
}

// internal/transform/stockham_packed.go:86-196,306-432 packed Stockham:
// one radix-2 DIF stage when log2(n) is odd, then radix-4 DIF stages with
// packed twiddles W_m^{jk} (twiddle_packed.go:13-48) applied to the outputs.
template <typename R>
void stockham_packed(cx<R>* dst, const cx<R>* src, const cx<R>* tw, int64_t n, bool inverse) {
  if (n == 1) { dst[0] = src[0]; return; }
  int64_t rem = n;
  while (rem % 4 == 0) rem /= 4;
  std::vector<cx<R>> a(src, src + n), b(n);
  int64_t m = n;
  if (rem == 2) {
    int64_t half = m >> 1, step = n / m, halfN = n >> 1;
    for (int64_t k = 0; k < n / m; ++k)
      for (int64_t j = 0; j < half; ++j) {
        cx<R> x = a[k * m + j], y = a[k * m + j + half];
        cx<R> w = tw[j * step];
        if (inverse) w = conj(w);
        b[k * half + j] = x + y;
        b[k * half + halfN + j] = (x - y) * w;
      }
    std::swap(a, b);
    m = n / 2;
  }
  int64_t q = n / 4;
  while (m >= 4) {
    int64_t span = m / 4, step = n / m;
    for (int64_t k = 0; k < n / m; ++k) {
      for (int64_t j = 0; j < span; ++j) {
        cx<R> w1 = tw[(1 * j * step) % n], w2 = tw[(2 * j * step) % n], w3 = tw[(3 * j * step) % n];
        if (inverse) { w1 = conj(w1); w2 = conj(w2); w3 = conj(w3); }
        const cx<R>* in = &a[k * m];
        cx<R> a0 = in[j], a1 = in[j + span], a2 = in[j + 2 * span], a3 = in[j + 3 * span];
        cx<R> t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = a1 - a3;
        cx<R> y0 = t0 + t2, y2 = t0 - t2, y1, y3;
        if (inverse) {
          y1 = t1 + cx<R>{-t3.im, t3.re};
          y3 = t1 + cx<R>{t3.im, -t3.re};
        } else {
          y1 = t1 + cx<R>{t3.im, -t3.re};
          y3 = t1 + cx<R>{-t3.im, t3.re};
        }
        int64_t ob = k * span;
        b[ob + j] = y0;
        b[ob + q + j] = y1 * w1;
        b[ob + 2 * q + j] = y2 * w2;
        b[ob + 3 * q + j] = y3 * w3;
      }
    }
    std::swap(a, b);
    m /= 4;
  }
  if (inverse) {
    R sc = R(1.0 / double(n));
    for (auto& v : a) v = v * cx<R>{sc, 0};
  }
  std::memcpy(dst, a.data(), sizeof(cx<R>) * n);
}

// internal/kernels/sixstep.go:29-91 six-step for square n = m*m (the
// eight-step kernel of eightstep.go:27-154 is the same algorithm):
// transpose, m row FFTs, transpose, twiddle W_n^{ij}, m row FFTs, transpose.
// Row FFTs are radix-2 Stockham with row twiddles tw[i*(n/m)]; the inverse
// rows each scale by 1/m, giving 1/n overall.
template <typename R>
void sixstep(cx<R>* dst, const cx<R>* src, const cx<R>* tw, int64_t n, bool inverse) {
  int64_t m = int64_t(std::llround(std::sqrt(double(n))));
  std::vector<cx<R>> d(src, src + n);
  auto transpose = [&]() {
    for (int64_t i = 0; i < m; ++i)
      for (int64_t j = i + 1; j < m; ++j) std::swap(d[i * m + j], d[j * m + i]);
  };
  std::vector<cx<R>> rowtw(m);
  for (int64_t i = 0; i < m; ++i) rowtw[i] = tw[i * (n / m)];
  transpose();
  for (int64_t r = 0; r < m; ++r) stockham2(&d[r * m], &d[r * m], rowtw.data(), m, inverse);
  transpose();
  for (int64_t i = 0; i < m; ++i)
    for (int64_t j = 0; j < m; ++j) {
      cx<R> w = tw[(i * j) % n];
      d[i * m + j] = d[i * m + j] * (inverse ? conj(w) : w);
    }
  for (int64_t r = 0; r < m; ++r) stockham2(&d[r * m], &d[r * m], rowtw.data(), m, inverse);
  transpose();
  std::memcpy(dst, d.data(), sizeof(cx<R>) * n);
}

// internal/kernels/radix3.go:185, radix5.go:201 and radix4.go:193
// butterflies: plain DFT_r of the (already twiddled) inputs, with the
// conjugate kernel for the inverse.
template <typename R>
void small_dft(cx<R>* y, const cx<R>* a, int r, bool inverse) {
  double sgn = inverse ? 1.0 : -1.0;
  for (int k = 0; k < r; ++k) {
    cx<R> s{0, 0};
    for (int j = 0; j < r; ++j) {
      int64_t m = (int64_t(j) * k) % r;
      double ang = sgn * 2.0 * kPi * double(m) / double(r);
      s = s + a[j] * cx<R>{R(std::cos(ang)), R(std::sin(ang))};
    }
    y[k] = s;
  }
}

// internal/fft/mixedradix.go:128-188 mixedRadixSchedule: repeatedly take
// 5, then 4, then 3, then 2.  (The reference also short-circuits to a
// registered codelet size > 16; with a leaf radix > 5 its ping-pong
// butterfly at mixedradix.go:350-354 applies no butterfly, so that
// shortcut is not restated: the pure 5/4/3/2 schedule is.)
std::vector<int> mixed_schedule(int64_t n) {
  std::vector<int> r;
  while (n > 1) {
    if (n % 5 == 0) { r.push_back(5); n /= 5; }
    else if (n % 4 == 0) { r.push_back(4); n /= 4; }
    else if (n % 3 == 0) { r.push_back(3); n /= 3; }
    else if (n % 2 == 0) { r.push_back(2); n /= 2; }
    else return {};
  }
  return r;
}

// internal/fft/mixedradix.go:225-354 recursive ping-pong decimation in
// time: sub-transform j gathers src[j*stride + i*stride*radix], then the
// radix-r butterfly over k < span with twiddles twiddle[i*k*step].
template <typename R>
void mixed_rec(cx<R>* dst, const cx<R>* src, cx<R>* work, int64_t n, int64_t stride, int64_t step,
               const int* radices, int nrad, const cx<R>* tw, bool inverse) {
  if (n == 1) { dst[0] = src[0]; return; }
  int radix = radices[0];
  int64_t span = n / radix;
  for (int j = 0; j < radix; ++j) {
    if (nrad == 1) {
      for (int64_t i = 0; i < span; ++i) dst[j * span + i] = src[j * stride + i * stride];
    } else {
      mixed_rec(work + j * span, src + j * stride, dst + j * span, span, stride * radix, step * radix,
                radices + 1, nrad - 1, tw, inverse);
    }
  }
  const cx<R>* input = (nrad == 1) ? dst : work;
  cx<R> a[8], y[8];
  for (int64_t k = 0; k < span; ++k) {
    for (int j = 0; j < radix; ++j) {
      cx<R> w = tw[j * k * step];
      if (inverse) w = conj(w);
      a[j] = (j == 0) ? input[k] : w * input[j * span + k];
    }
    if (radix == 2) {
      y[0] = a[0] + a[1];
      y[1] = a[0] - a[1];
    } else {
      small_dft(y, a, radix, inverse);
    }
    for (int j = 0; j < radix; ++j) dst[j * span + k] = y[j];
  }
}

// internal/fft/mixedradix.go:45-126 mixedRadixTransform (scale 1/n inverse).
template <typename R>
bool mixed_radix(cx<R>* dst, const cx<R>* src, const cx<R>* tw, int64_t n, bool inverse) {
  if (n == 1) { dst[0] = src[0]; return true; }
  std::vector<int> rad = mixed_schedule(n);
  if (rad.empty()) return false;
  std::vector<cx<R>> out(n), scratch(n);
  mixed_rec(out.data(), src, scratch.data(), n, 1, 1, rad.data(), int(rad.size()), tw, inverse);
  if (inverse) {
    R s = R(1.0 / double(n));
    for (auto& v : out) v = v * cx<R>{s, 0};
  }
  std::memcpy(dst, out.data(), sizeof(cx<R>) * n);
  return true;
}

// internal/kernels/bluestein.go:20-32 ComputeChirpSequence:
// exp(-iπ k²/n) with the angle float64(k*k)/n (no mod-2n reduction).
template <typename R>
std::vector<cx<R>> chirp(int64_t n) {
  std::vector<cx<R>> c(n);
  double invN = 1.0 / double(n);
  for (int64_t k = 0; k < n; ++k) {
    double ang = -kPi * double(k * k) * invN;
    c[k] = {R(std::cos(ang)), R(std::sin(ang))};
  }
  return c;
}

// plan.go:864-890 + internal/kernels/bluestein.go:39-77 +
// plan_bluestein.go:7-58: M = NextPow2(2n-1), filter = DIT_M of
// conj(chirp) mirrored, y = IDIT_M(DIT_M(x*chirp) * filter) * chirp
// (times 1/n for the inverse, which uses the conjugate chirp).
template <typename R>
void bluestein(cx<R>* dst, const cx<R>* src, int64_t n, bool inverse) {
  int64_t M = next_pow2(2 * n - 1);
  std::vector<cx<R>> c = chirp<R>(n);
  if (inverse) for (auto& v : c) v = conj(v);
  std::vector<cx<R>> twM = twiddles<R>(M);
  std::vector<cx<R>> b(M, cx<R>{0, 0});
  b[0] = conj(c[0]);
  for (int64_t k = 1; k < n; ++k) { b[k] = conj(c[k]); b[M - k] = conj(c[k]); }
  dit(b.data(), b.data(), twM.data(), M, false);
  std::vector<cx<R>> x(M, cx<R>{0, 0});
  for (int64_t i = 0; i < n; ++i) x[i] = src[i] * c[i];
  dit(x.data(), x.data(), twM.data(), M, false);
  for (int64_t i = 0; i < M; ++i) x[i] = x[i] * b[i];
  dit(x.data(), x.data(), twM.data(), M, true);
  if (inverse) {
    cx<R> s{R(1.0 / double(n)), 0};
    for (int64_t i = 0; i < n; ++i) dst[i] = x[i] * c[i] * s;
  } else {
    for (int64_t i = 0; i < n; ++i) dst[i] = x[i] * c[i];
  }
}

// Strategy choice of the reference for one transform of length n:
// planner.go:43-78 (Bluestein unless pow2 or 2/3/5-smooth),
// selection.go:66-108 (six/eight-step for square n >= 2^18, DIT <= the
// codelet range, Stockham above), plan.go:343-368 (dispatch order).
enum Algo { kDIT = 0, kStockham = 1, kSixStep = 2, kMixed = 3, kBluestein = 4 };
int choose(int64_t n) {
  if (!is_pow2(n)) return is_235_smooth(n) ? kMixed : kBluestein;
  int64_t m = int64_t(std::llround(std::sqrt(double(n))));
  if (m * m == n && n >= (int64_t(1) << 18)) return kSixStep;
  if (n <= 16384) return kDIT;  // size-specific DIT codelets 4..16384
  return kStockham;
}

template <typename R>
int transform(cx<R>* dst, const cx<R>* src, int64_t n, bool inverse, const cx<R>* tw) {
  switch (choose(n)) {
    case kDIT: dit(dst, src, tw, n, inverse); return 0;
    case kStockham: stockham_packed(dst, src, tw, n, inverse); return 0;
    case kSixStep: sixstep(dst, src, tw, n, inverse); return 0;
    case kMixed: return mixed_radix(dst, src, tw, n, inverse) ? 0 : 6;
    default: bluestein(dst, src, n, inverse); return 0;
  }
}

// plan.go:504-571 ForwardBatch/InverseBatch: count independent transforms
// on [i*n, (i+1)*n).  The reference loop is serial; nthreads > 1 splits the
// batch over threads the way P goroutines with one Executor each would.
template <typename R>
int batch(R* dst, const R* src, int64_t n, int64_t count, bool inverse, int nthreads) {
  auto* d = reinterpret_cast<cx<R>*>(dst);
  auto* s = reinterpret_cast<const cx<R>*>(src);
  std::vector<cx<R>> tw = twiddles<R>(n);
  std::atomic<int> rc{0};
  parallel_for(count, nthreads, [&](int64_t i) {
    int r = transform(d + i * n, s + i * n, n, inverse, tw.data());
    if (r) rc.fetch_or(r);
  });
  return rc.load();
}

// plan_real_generic.go:64-98 weights U[k] = 0.5*(1 + i W_N^k), evaluated
// as 0.5*(1+sin θ) + i 0.5 cos θ with θ = 2πk/N, cast to the precision.
template <typename R>
std::vector<cx<R>> real_weights(int64_t n) {
  std::vector<cx<R>> w(n / 2 + 1);
  for (int64_t k = 0; k <= n / 2; ++k) {
    double th = 2.0 * kPi * double(k) / double(n);
    w[k] = {R(0.5 * (1.0 + std::sin(th))), R(0.5 * std::cos(th))};
  }
  return w;
}

// plan_real_generic.go:142-229 forwardSingle: pack pairs as complex, half
// size C2C, DC/Nyquist from y0, X[k] = A - U[k](A - conj(Y[h-k])).
template <typename R>
void real_forward(cx<R>* dst, const R* src, int64_t n) {
  int64_t h = n / 2;
  std::vector<cx<R>> buf(h);
  std::memcpy(buf.data(), src, sizeof(R) * n);
  std::vector<cx<R>> tw = twiddles<R>(h);
  transform(buf.data(), buf.data(), h, false, tw.data());
  std::vector<cx<R>> w = real_weights<R>(n);
  cx<R> y0 = buf[0];
  dst[0] = {y0.re + y0.im, 0};
  dst[h] = {y0.re - y0.im, 0};
  for (int64_t k = 1; k < h; ++k) {
    cx<R> a = buf[k], b = conj(buf[h - k]);
    cx<R> c = w[k] * (a - b);
    dst[k] = a - c;
  }
}

// plan_real_generic.go:289-355 inverseSingle + internal/fft/real_repack.go:
// 5-100 RepackInverse, then the half-size inverse (1/h) and unpack.
// Returns 5 (invalid spectrum) when DC/Nyquist imaginary parts exceed eps.
template <typename R>
int real_inverse(R* dst, const cx<R>* src, int64_t n) {
  int64_t h = n / 2;
  double eps = sizeof(R) == 4 ? 1e-4 : 1e-12;
  if (std::fabs(double(src[0].im)) > eps || std::fabs(double(src[h].im)) > eps) return 5;
  std::vector<cx<R>> w = real_weights<R>(n);
  std::vector<cx<R>> buf(h);
  R x0 = src[0].re, xh = src[h].re;
  buf[0] = {R(0.5) * (x0 + xh), R(0.5) * (x0 - xh)};
  for (int64_t k = 1; k < h; ++k) {
    int64_t m = h - k;
    if (k > m) continue;
    cx<R> xk = src[k], xmkc = conj(src[m]);
    cx<R> u = w[k];
    cx<R> one{1, 0}, two{2, 0};
    cx<R> omu = one - u;
    cx<R> det = one - two * u;
    cx<R> inv = conj(det);
    cx<R> a = (xk * omu - xmkc * u) * inv;
    cx<R> b = (omu * xmkc - u * xk) * inv;
    buf[k] = a;
    if (k != m) buf[m] = conj(b);
  }
  std::vector<cx<R>> tw = twiddles<R>(h);
  transform(buf.data(), buf.data(), h, true, tw.data());
  std::memcpy(dst, buf.data(), sizeof(R) * n);
  return 0;
}

}  // namespace

extern "C" {

// FP64 naive DFT, the arbiter.  Follows internal/reference/dft.go:16-150
// (NaiveDFT128/NaiveIDFT128: sum x[j] exp(∓2πi jk/n), inverse * 1/n) but
// reduces the angle exactly as (j*k mod n) before the float64 evaluation,
// so its angles are within 1 ulp of the exact ones for every n.
void orc_naive_dft_f64(const double* in, double* out, int64_t n, int inverse) {
  const auto* x = reinterpret_cast<const cx<double>*>(in);
  auto* y = reinterpret_cast<cx<double>*>(out);
  std::vector<cx<double>> w(n);
  double sgn = inverse ? 1.0 : -1.0;
  for (int64_t m = 0; m < n; ++m) {
    double ang = sgn * 2.0 * kPi * double(m) / double(n);
    w[m] = {std::cos(ang), std::sin(ang)};
  }
  int nt = n >= 1024 ? int(std::max(1u, std::thread::hardware_concurrency())) : 1;
  parallel_for(n, nt, [&](int64_t k) {
    // long double accumulation keeps the O(n) summation error far below
    // the tolerances the tests use for complex128.
    long double sr = 0, si = 0;
    int64_t m = 0;
    for (int64_t j = 0; j < n; ++j) {
      const cx<double>& a = x[j];
      const cx<double>& t = w[m];
      sr += (long double)a.re * t.re - (long double)a.im * t.im;
      si += (long double)a.re * t.im + (long double)a.im * t.re;
      m += k;
      if (m >= n) m -= n;
    }
    double s = inverse ? 1.0 / double(n) : 1.0;
    y[k] = {double(sr) * s, double(si) * s};
  });
}

// internal/reference/dft.go:16-51 NaiveDFT / :61-96 NaiveIDFT verbatim
// formula (angle = ∓2π·k·j/n in float64 without reduction), complex128
// accumulation, used to pin the arbiter against the reference's own oracle.
void orc_naive_dft_ref(const double* in, double* out, int64_t n, int inverse) {
  const auto* x = reinterpret_cast<const cx<double>*>(in);
  auto* y = reinterpret_cast<cx<double>*>(out);
  double sgn = inverse ? 2.0 : -2.0;
  for (int64_t k = 0; k < n; ++k) {
    cx<double> s{0, 0};
    for (int64_t j = 0; j < n; ++j) {
      double ang = sgn * kPi * double(k) * double(j) / double(n);
      s = s + x[j] * cx<double>{std::cos(ang), std::sin(ang)};
    }
    if (inverse) s = s * cx<double>{1.0 / double(n), 0};
    y[k] = s;
  }
}

// internal/reference/dft2d.go:17-160 NaiveDFT2D / NaiveIDFT2D (and the
// complex128 forms) and internal/reference/dft3d.go:18-146 NaiveDFT3D /
// NaiveIDFT3D, generalised over the axis count: row-major input
// x[i0*d1*..*d(r-1) + ...], output bin (k0, .., k(r-1)) in the same order;
// per input sample the phase is the sum over axes of ∓2π·k_a·m_a/d_a, each
// term formed in float64 without reduction exactly as the reference does,
// then cos/sin of the sum, complex128 accumulation, the inverse scaled by
// 1/(d0·..·d(r-1)).  The complex64 reference versions round the complex128
// sum to complex64 at the end; the caller does that cast.
void orc_naive_dft_nd_ref(const double* in, double* out, int ndims, const int64_t* dims, int inverse) {
  const auto* x = reinterpret_cast<const cx<double>*>(in);
  auto* y = reinterpret_cast<cx<double>*>(out);
  int64_t total = 1;
  for (int a = 0; a < ndims; ++a) total *= dims[a];
  const double sgn = inverse ? 2.0 : -2.0;
  std::vector<int64_t> k(ndims), m(ndims);
  for (int64_t kk = 0; kk < total; ++kk) {
    for (int64_t r = kk, a = ndims - 1; a >= 0; --a) {
      k[a] = r % dims[a];
      r /= dims[a];
    }
    cx<double> s{0, 0};
    for (int64_t mm = 0; mm < total; ++mm) {
      for (int64_t r = mm, a = ndims - 1; a >= 0; --a) {
        m[a] = r % dims[a];
        r /= dims[a];
      }
      double phase = 0;
      for (int a = 0; a < ndims; ++a) phase += sgn * kPi * double(k[a] * m[a]) / double(dims[a]);
      s = s + x[mm] * cx<double>{std::cos(phase), std::sin(phase)};
    }
    if (inverse) s = s * cx<double>{1.0 / double(total), 0};
    y[kk] = s;
  }
}

// FP64 N-D arbiter: the same sum with every axis term reduced exactly
// (k_a·m_a mod d_a in integers) and the phase accumulated as a fraction of
// a turn in long double, long double accumulation of the products.
void orc_naive_dft_nd_f64(const double* in, double* out, int ndims, const int64_t* dims, int inverse) {
  const auto* x = reinterpret_cast<const cx<double>*>(in);
  auto* y = reinterpret_cast<cx<double>*>(out);
  int64_t total = 1;
  for (int a = 0; a < ndims; ++a) total *= dims[a];
  const long double sgn = inverse ? 1.0L : -1.0L;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  std::vector<int64_t> k(ndims), m(ndims);
  for (int64_t kk = 0; kk < total; ++kk) {
    for (int64_t r = kk, a = ndims - 1; a >= 0; --a) {
      k[a] = r % dims[a];
      r /= dims[a];
    }
    long double sr = 0, si = 0;
    for (int64_t mm = 0; mm < total; ++mm) {
      for (int64_t r = mm, a = ndims - 1; a >= 0; --a) {
        m[a] = r % dims[a];
        r /= dims[a];
      }
      long double turn = 0;
      for (int a = 0; a < ndims; ++a) turn += (long double)((k[a] * m[a]) % dims[a]) / (long double)dims[a];
      turn -= std::floor(turn);
      const long double c = std::cos(sgn * two_pi * turn), sn = std::sin(sgn * two_pi * turn);
      sr += (long double)x[mm].re * c - (long double)x[mm].im * sn;
      si += (long double)x[mm].re * sn + (long double)x[mm].im * c;
    }
    const long double s = inverse ? 1.0L / (long double)total : 1.0L;
    y[kk] = {double(sr * s), double(si * s)};
  }
}

// The reference's algorithm choice for n (plan.go:343-368): 0 DIT,
// 1 Stockham, 2 six-step, 3 mixed radix, 4 Bluestein.
int orc_algorithm(int64_t n) { return choose(n); }

// Plan.ForwardBatch / InverseBatch restated (plan.go:504-571).
int orc_batch_c64(float* dst, const float* src, int64_t n, int64_t count, int inverse, int nthreads) {
  return batch<float>(dst, src, n, count, inverse != 0, nthreads);
}
int orc_batch_c128(double* dst, const double* src, int64_t n, int64_t count, int inverse, int nthreads) {
  return batch<double>(dst, src, n, count, inverse != 0, nthreads);
}

// Forcing one algorithm (SetKernelStrategy, selection.go:22-29).
int orc_transform_algo_c64(float* dst, const float* src, int64_t n, int inverse, int algo) {
  auto* d = reinterpret_cast<cx<float>*>(dst);
  auto* s = reinterpret_cast<const cx<float>*>(src);
  std::vector<cx<float>> tw = twiddles<float>(n);
  switch (algo) {
    case kDIT: if (!is_pow2(n)) return 6; dit(d, s, tw.data(), n, inverse); return 0;
    case kStockham: if (!is_pow2(n)) return 6; stockham_packed(d, s, tw.data(), n, inverse); return 0;
    case kSixStep: {
      int64_t m = int64_t(std::llround(std::sqrt(double(n))));
      if (m * m != n || !is_pow2(n)) return 6;
      sixstep(d, s, tw.data(), n, inverse); return 0;
    }
    case kMixed: return mixed_radix(d, s, tw.data(), n, inverse) ? 0 : 6;
    case kBluestein: bluestein(d, s, n, inverse); return 0;
  }
  return 6;
}

// PlanReal Forward/Inverse for a batch of contiguous transforms
// (plan_real_generic.go:111-139,256-287 with Batch>1, default strides).
int orc_real_forward_f32(float* dst, const float* src, int64_t n, int64_t batch, int nthreads) {
  if (n < 2 || n % 2) return 1;
  parallel_for(batch, nthreads, [&](int64_t b) {
    real_forward<float>(reinterpret_cast<cx<float>*>(dst) + b * (n / 2 + 1), src + b * n, n);
  });
  return 0;
}
int orc_real_inverse_f32(float* dst, const float* src, int64_t n, int64_t batch, int nthreads) {
  if (n < 2 || n % 2) return 1;
  std::atomic<int> rc{0};
  parallel_for(batch, nthreads, [&](int64_t b) {
    int r = real_inverse<float>(dst + b * n, reinterpret_cast<const cx<float>*>(src) + b * (n / 2 + 1), n);
    if (r) rc.fetch_or(r);
  });
  return rc.load();
}
int orc_real_forward_f64(double* dst, const double* src, int64_t n, int64_t batch) {
  if (n < 2 || n % 2) return 1;
  for (int64_t b = 0; b < batch; ++b)
    real_forward<double>(reinterpret_cast<cx<double>*>(dst) + b * (n / 2 + 1), src + b * n, n);
  return 0;
}
int orc_real_inverse_f64(double* dst, const double* src, int64_t n, int64_t batch) {
  if (n < 2 || n % 2) return 1;
  int rc = 0;
  for (int64_t b = 0; b < batch; ++b)
    rc |= real_inverse<double>(dst + b * n, reinterpret_cast<const cx<double>*>(src) + b * (n / 2 + 1), n);
  return rc;
}

// convolve_real.go:9-66 ConvolveReal: real plan at NextPow2(len(a)+len(b)-1)
// (at least 2), two forwards, pointwise product, inverse, truncate.
int orc_convolve_real_f32(float* dst, const float* a, int64_t na, const float* b, int64_t nb) {
  if (na == 0 || nb == 0) return 1;
  int64_t L = na + nb - 1, F = std::max<int64_t>(2, next_pow2(L));
  std::vector<float> ap(F, 0.f), bp(F, 0.f), t(F);
  std::memcpy(ap.data(), a, sizeof(float) * na);
  std::memcpy(bp.data(), b, sizeof(float) * nb);
  std::vector<cx<float>> A(F / 2 + 1), B(F / 2 + 1);
  real_forward<float>(A.data(), ap.data(), F);
  real_forward<float>(B.data(), bp.data(), F);
  for (int64_t i = 0; i <= F / 2; ++i) A[i] = A[i] * B[i];
  int rc = real_inverse<float>(t.data(), A.data(), F);
  std::memcpy(dst, t.data(), sizeof(float) * L);
  return rc;
}

// convolve.go:9-59 Convolve (complex64): plan at exactly len(a)+len(b)-1,
// two forwards, pointwise product (complex_mul.go:23), inverse.
int orc_convolve_c64(float* dst, const float* a, int64_t na, const float* b, int64_t nb) {
  if (na == 0 || nb == 0) return 1;
  int64_t L = na + nb - 1;
  std::vector<cx<float>> ap(L, cx<float>{0, 0}), bp(L, cx<float>{0, 0}), A(L), B(L);
  std::memcpy(ap.data(), a, sizeof(cx<float>) * na);
  std::memcpy(bp.data(), b, sizeof(cx<float>) * nb);
  std::vector<cx<float>> tw = twiddles<float>(L);
  int rc = transform(A.data(), ap.data(), L, false, tw.data());
  rc |= transform(B.data(), bp.data(), L, false, tw.data());
  for (int64_t i = 0; i < L; ++i) A[i] = A[i] * B[i];
  rc |= transform(reinterpret_cast<cx<float>*>(dst), A.data(), L, true, tw.data());
  return rc;
}

// twiddle.go:8-21 table (complex64 and complex128 casts).
void orc_twiddles_c64(float* out, int64_t n) {
  std::vector<cx<float>> t = twiddles<float>(n);
  std::memcpy(out, t.data(), sizeof(cx<float>) * n);
}
void orc_twiddles_c128(double* out, int64_t n) {
  std::vector<cx<double>> t = twiddles<double>(n);
  std::memcpy(out, t.data(), sizeof(cx<double>) * n);
}

int orc_max_threads(void) { return int(std::max(1u, std::thread::hardware_concurrency())); }

}  // extern "C"
