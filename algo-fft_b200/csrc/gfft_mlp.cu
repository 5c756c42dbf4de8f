// Learned planner: an FP32 MLP cost model with its own CUDA inference,
// gradient and training kernels, and the plan-creation hook that uses it.
//
// The model scores a (shape, candidate variant) pair: 16 features (the
// shape: log2 n, the exponents of 2/3/5/7 in n, log2 of n's largest prime
// factor, log2 batch, precision, log2 stride, real/complex; the candidate:
// one-hot kind p2/tp/mixed/bluestein plus two numeric shape parameters of
// the variant; the three-pass form is kind tp with both parameters 0),
// standardized with stored means and deviations, through
// 16 -> 64 -> 64 -> 1 with ReLU, to a standardized log(ns per element).
// Plan creation with GFFT_PLANNER_LEARNED evaluates every candidate of the
// length in one inference launch and takes the smallest prediction; the
// wisdom store still wins where it has an entry, and exhaustive measurement
// (GFFT_PLANNER_MEASURE and up, the autotuner) stays the arbiter the model is
// trained on and scored against.  The reference decides by size class alone
// (internal/planner/planner.go:43-78, selection.go:66-108) and measures per
// size (internal/fft/measure.go:89-228); it has no learned model.
//
// Parameters, flat FP32 in this order (row-major weights):
//   W1[64][16] b1[64] W2[64][64] b2[64] w3[64] b3
// Kernels keep them in shared memory with padded rows (17 and 65 floats) so
// the lane-per-unit accesses are conflict free.
//
// Training is deterministic: mini-batch indices come from a counter hash of
// (seed, step, slot), and every gradient entry is a sum over the batch in a
// fixed order by one thread (no atomics), followed by an Adam step.
#include <dlfcn.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <string>
#include <vector>
#include "gfft_internal.h"

namespace gfft {
namespace mlp {

constexpr int D = 16, H = 64;
constexpr int W1 = 0, B1 = H * D, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H, B3 = W3 + H, NP = B3 + 1;
constexpr int SW1 = 0, SB1 = SW1 + H * (D + 1), SW2 = SB1 + H, SB2 = SW2 + H * (H + 1), SW3 = SB2 + H,
              SB3 = SW3 + H, SNP = SB3 + 1;
constexpr int MAXB = 64;  // samples per training step / gradient call
constexpr int TPB = 256;  // training CTA
// training shared memory: parameters, then per-sample x, h1, h2, d2, d1, dy, y
constexpr int SM_X = SNP, SM_H1 = SM_X + MAXB * D, SM_H2 = SM_H1 + MAXB * H, SM_D2 = SM_H2 + MAXB * H,
              SM_D1 = SM_D2 + MAXB * H, SM_DY = SM_D1 + MAXB * H, SM_Y = SM_DY + MAXB, SM_TOTAL = SM_Y + MAXB;

__device__ __forceinline__ int padded(int e) {
  if (e < B1) return SW1 + (e / D) * (D + 1) + e % D;
  if (e < W2) return SB1 + (e - B1);
  if (e < B2) return SW2 + ((e - W2) / H) * (H + 1) + (e - W2) % H;
  if (e < W3) return SB2 + (e - B2);
  if (e < B3) return SW3 + (e - W3);
  return SB3;
}

__device__ __forceinline__ void load_params(float* P, const float* params) {
  for (int e = threadIdx.x; e < NP; e += blockDim.x) P[padded(e)] = params[e];
}

// One sample by one warp: lane owns hidden units lane and lane + 32.
// Returns the prediction (every lane); h1/h2 are post-ReLU activations.
__device__ __forceinline__ float forward_warp(const float* P, const float* x, int lane, float h1[2], float h2[2]) {
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int u = lane + 32 * q;
    float a = P[SB1 + u];
#pragma unroll
    for (int d = 0; d < D; ++d) a = fmaf(P[SW1 + u * (D + 1) + d], x[d], a);
    h1[q] = fmaxf(a, 0.f);
  }
  float a0 = P[SB2 + lane], a1 = P[SB2 + lane + 32];
#pragma unroll 8
  for (int k = 0; k < H; ++k) {
    const float hk = __shfl_sync(0xffffffffu, k < 32 ? h1[0] : h1[1], k & 31);
    a0 = fmaf(P[SW2 + lane * (H + 1) + k], hk, a0);
    a1 = fmaf(P[SW2 + (lane + 32) * (H + 1) + k], hk, a1);
  }
  h2[0] = fmaxf(a0, 0.f);
  h2[1] = fmaxf(a1, 0.f);
  float part = fmaf(P[SW3 + lane], h2[0], P[SW3 + lane + 32] * h2[1]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
  return part + P[SB3];
}

__global__ void k_mlp_forward(const float* __restrict__ params, const float* __restrict__ X, int64_t n,
                              float* __restrict__ out) {
  __shared__ float P[SNP];
  load_params(P, params);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t s = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); s < n; s += warps) {
    float x[D], h1[2], h2[2];
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = X[s * D + d];
    const float y = forward_warp(P, x, lane, h1, h2);
    if (lane == 0) out[s] = y;
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Mini-batch of B samples: forward, backward, then gradient entry e by one
// thread as a fixed-order sum over the batch.  With train, an Adam step
// (beta1 0.9, beta2 0.999, eps 1e-8) per mini-batch for `steps` steps;
// without, one pass over samples 0..B-1 writing grad[] and the loss.
__global__ void __launch_bounds__(TPB) k_mlp_train(float* params, float* am, float* av, const float* __restrict__ X,
                                                   const float* __restrict__ Y, int64_t n, int steps, int B, float lr,
                                                   uint64_t seed, int64_t step0, int train, float* loss_out,
                                                   float* grad_out) {
  extern __shared__ float sm[];
  float* P = sm;
  float* xs = sm + SM_X;
  float* h1s = sm + SM_H1;
  float* h2s = sm + SM_H2;
  float* d2s = sm + SM_D2;
  float* d1s = sm + SM_D1;
  float* dys = sm + SM_DY;
  float* ys = sm + SM_Y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  load_params(P, params);
  double loss_sum = 0;
  for (int step = 0; step < steps; ++step) {
    __syncthreads();
    // gather the batch
    for (int i = tid; i < B * D; i += TPB) {
      const int s = i / D, d = i % D;
      const int64_t idx = train ? int64_t(mix64(seed ^ mix64(uint64_t(step0 + step) * 1024 + s)) % uint64_t(n)) : s;
      xs[i] = X[idx * D + d];
      if (d == 0) ys[s] = Y[idx];
    }
    __syncthreads();
    // forward + backward, one warp per sample
    for (int s = warp; s < B; s += TPB / 32) {
      float h1[2], h2[2];
      const float yh = forward_warp(P, xs + s * D, lane, h1, h2);
      const float dy = 2.f * (yh - ys[s]) / float(B);
      float d2[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int u = lane + 32 * q;
        h1s[s * H + u] = h1[q];
        h2s[s * H + u] = h2[q];
        d2[q] = h2[q] > 0.f ? dy * P[SW3 + u] : 0.f;
        d2s[s * H + u] = d2[q];
      }
      if (lane == 0) dys[s] = dy;
      __syncwarp();
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int k = lane + 32 * q;
        float acc = 0.f;
        for (int u = 0; u < H; ++u) acc = fmaf(d2s[s * H + u], P[SW2 + u * (H + 1) + k], acc);
        d1s[s * H + k] = h1[q] > 0.f ? acc : 0.f;
      }
    }
    __syncthreads();
    if (tid == 0) {
      // (yh - y)^2 = (dy * B / 2)^2
      float l = 0.f;
      for (int s = 0; s < B; ++s) l += (0.5f * float(B) * dys[s]) * (0.5f * float(B) * dys[s]);
      loss_sum += double(l) / double(B);
    }
    // gradients (fixed order) and the update
    const int64_t t = step0 + step + 1;
    const float c1 = float(1.0 - std::pow(0.9, double(t))), c2 = float(1.0 - std::pow(0.999, double(t)));
    for (int e = tid; e < NP; e += TPB) {
      float g = 0.f;
      if (e < B1) {
        const int u = e / D, d = e % D;
        for (int s = 0; s < B; ++s) g = fmaf(d1s[s * H + u], xs[s * D + d], g);
      } else if (e < W2) {
        for (int s = 0; s < B; ++s) g += d1s[s * H + (e - B1)];
      } else if (e < B2) {
        const int u = (e - W2) / H, k = (e - W2) % H;
        for (int s = 0; s < B; ++s) g = fmaf(d2s[s * H + u], h1s[s * H + k], g);
      } else if (e < W3) {
        for (int s = 0; s < B; ++s) g += d2s[s * H + (e - B2)];
      } else if (e < B3) {
        for (int s = 0; s < B; ++s) g = fmaf(dys[s], h2s[s * H + (e - W3)], g);
      } else {
        for (int s = 0; s < B; ++s) g += dys[s];
      }
      if (!train) {
        grad_out[e] = g;
        continue;
      }
      const float m = 0.9f * am[e] + 0.1f * g;
      const float v = 0.999f * av[e] + 0.001f * g * g;
      am[e] = m;
      av[e] = v;
      P[padded(e)] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
    }
  }
  __syncthreads();
  if (train)
    for (int e = tid; e < NP; e += TPB) params[e] = P[padded(e)];
  if (tid == 0 && loss_out) *loss_out = float(loss_sum / double(steps > 0 ? steps : 1));
}

// ---- the installed model ---------------------------------------------------

struct Model {
  std::mutex mu;
  bool loaded = false, tried_default = false;
  std::vector<float> params;   // NP
  std::vector<float> norm;     // x_mu[D], x_sd[D], y_mu, y_sd
  int device = -1;
  float* d_params = nullptr;
  float* d_x = nullptr;        // candidates x D
  float* d_y = nullptr;
  int cap = 0;
};

Model& model() {
  static Model m;
  return m;
}

static int ilog2f(int64_t v) {
  int l = 0;
  while ((int64_t(1) << (l + 1)) <= v) ++l;
  return l;
}

}  // namespace mlp

// Raw (unstandardized) features of one (shape, candidate) pair.
static bool plan_features(int prec, int64_t n, int64_t batch, int64_t stride, int real, const std::string& tok,
                          float* f) {
  using namespace mlp;
  std::fill(f, f + D, 0.f);
  if (n < 1) return false;
  int64_t r = n;
  int ex[4] = {0, 0, 0, 0};
  const int pr[4] = {2, 3, 5, 7};
  for (int i = 0; i < 4; ++i)
    while (r % pr[i] == 0) {
      r /= pr[i];
      ++ex[i];
    }
  int64_t lpf = 1, m = n;
  for (int64_t p = 2; p * p <= m; ++p)
    while (m % p == 0) {
      lpf = p;
      m /= p;
    }
  if (m > 1) lpf = std::max(lpf, m);
  const size_t es = elem_bytes(prec);
  if (batch <= 0) batch = std::max<int64_t>(1, (int64_t(1) << 27) / (n * int64_t(es)));  // unknown: 128 MB
  f[0] = float(std::log2(double(n)));
  for (int i = 0; i < 4; ++i) f[1 + i] = float(ex[i]);
  f[5] = float(std::log2(double(lpf)));
  f[6] = float(std::log2(double(batch)));
  f[7] = float(prec);
  f[8] = float(std::log2(double(std::max<int64_t>(1, stride))));
  f[9] = float(real ? 1 : 0);
  int a = 0, b = 0, te = 0, e = 0, ns = 0, l = 0;
  long long l1 = 0, l2 = 0, ln = 0;
  if (std::sscanf(tok.c_str(), "gpu-sm100-p2-n%d-e%d", &a, &e) == 2) {
    f[10] = 1.f;
    f[14] = float(ilog2f(e));
  } else if (std::sscanf(tok.c_str(), "gpu-sm100-tp-%dx%d-t%d-e%d", &a, &b, &te, &e) == 4) {
    f[11] = 1.f;
    f[14] = float(ilog2f(e));
    f[15] = float(ilog2f(te));
  } else if (std::sscanf(tok.c_str(), "gpu-sm100-tp3-%dx%dx%d", &a, &b, &te) == 3) {
    f[11] = 1.f;  // a multi-pass schedule with no tile parameters: the three-pass form
  } else if (std::sscanf(tok.c_str(), "gpu-sm100-tp3t-%dx%dx%d-t%d-e%d-s%d", &a, &b, &l, &te, &e, &ns) == 6) {
    // the TMA-staged three-pass form: tile and elements per thread, the
    // latter offset by 4 so that it never coincides with a plain tile
    f[11] = 1.f;
    f[14] = float(ilog2f(e) + 4);
    f[15] = float(ilog2f(te));
  } else if (std::sscanf(tok.c_str(), "gpu-sm100-mixed2-%lldx%lld", &l1, &l2) == 2) {
    f[12] = 1.f;
    f[14] = 1.f;
    f[15] = float(std::log2(double(l1)));
  } else if (std::sscanf(tok.c_str(), "gpu-sm100-mixc-%lldx%lld", &l1, &l2) == 2) {
    f[12] = 1.f;  // the compiled mixed-radix four-step (marker 3)
    f[14] = 3.f;
    f[15] = float(std::log2(double(l1)));
  } else if (std::sscanf(tok.c_str(), "gpu-sm100-mixed-n%lld", &ln) == 1) {
    f[12] = 1.f;
  } else if (std::sscanf(tok.c_str(), "gpu-sm100-mixr-n%lld", &ln) == 1) {
    f[12] = 1.f;  // the compiled single pass (marker 2)
    f[14] = 2.f;
  } else if (std::sscanf(tok.c_str(), "gpu-sm100-bluestein-n%lld", &ln) == 1) {
    // FFT length: NextPow2(2n - 1), or the mixed length for "-mx" (marker 1)
    int64_t M = 1;
    while (M < 2 * n - 1) M <<= 1;
    const std::string mx = "gpu-sm100-bluestein-n" + std::to_string(n) + "-mx";
    int64_t m1 = 0;
    const int64_t x = tok.compare(0, mx.size(), mx) == 0 ? bs_mixed_choice(n, &m1) : 0;
    if (x > 0) {
      M = x;
      f[14] = 1.f;
    }
    f[13] = 1.f;
    f[15] = float(std::log2(double(M)));
  } else {
    return false;
  }
  return true;
}

static gfft_status model_install(const float* params, const float* norm) {
  using namespace mlp;
  Model& M = model();
  if (!params) {
    M.loaded = false;
    return GFFT_OK;
  }
  if (!norm) return GFFT_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < D; ++i)
    if (!(norm[D + i] > 0.f)) {
      set_error("feature deviation must be positive");
      return GFFT_ERR_INVALID_ARGUMENT;
    }
  if (!(norm[2 * D + 1] > 0.f)) return GFFT_ERR_INVALID_ARGUMENT;
  M.params.assign(params, params + NP);
  M.norm.assign(norm, norm + 2 * D + 2);
  M.loaded = true;
  M.device = -1;  // device copy refreshed on next use
  return GFFT_OK;
}

// Model file: 8-byte magic "GFMLP1\0\0", int32 D, int32 H, NP floats of
// parameters, 2D+2 floats of standardization, little-endian.
static gfft_status model_load_file(const std::string& path) {
  using namespace mlp;
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    set_error("cannot open " + path);
    return GFFT_ERR_INVALID_ARGUMENT;
  }
  char magic[8];
  int32_t dims[2];
  std::vector<float> prm(NP), nrm(2 * D + 2);
  in.read(magic, 8);
  in.read(reinterpret_cast<char*>(dims), sizeof dims);
  in.read(reinterpret_cast<char*>(prm.data()), NP * sizeof(float));
  in.read(reinterpret_cast<char*>(nrm.data()), nrm.size() * sizeof(float));
  if (!in || std::memcmp(magic, "GFMLP1\0\0", 8) != 0 || dims[0] != D || dims[1] != H) {
    set_error("not a planner model file: " + path);
    return GFFT_ERR_INVALID_ARGUMENT;
  }
  return model_install(prm.data(), nrm.data());
}

static void model_try_default() {
  mlp::Model& M = mlp::model();
  if (M.loaded || M.tried_default) return;
  M.tried_default = true;
  Dl_info info;
  if (!dladdr(reinterpret_cast<void*>(&model_try_default), &info) || !info.dli_fname) return;
  std::string dir(info.dli_fname);
  dir = dir.substr(0, dir.find_last_of('/') + 1);
  model_load_file(dir + "wisdom/planner_b200.bin");
  clear_error();
}

// One inference launch over the candidates (device = current device).
static bool model_predict(const std::vector<float>& xs, int rows, std::vector<float>* out) {
  using namespace mlp;
  Model& M = model();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (M.device != dev || rows > M.cap) {
    if (M.d_params) cudaFree(M.d_params);
    if (M.d_x) cudaFree(M.d_x);
    if (M.d_y) cudaFree(M.d_y);
    M.d_params = M.d_x = M.d_y = nullptr;
    M.cap = std::max(rows, 64);
    if (cudaMalloc(&M.d_params, NP * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&M.d_x, size_t(M.cap) * D * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&M.d_y, size_t(M.cap) * sizeof(float)) != cudaSuccess)
      return false;
    M.device = -1;
  }
  if (M.device != dev) {
    if (cudaMemcpy(M.d_params, M.params.data(), NP * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
      return false;
    M.device = dev;
  }
  if (cudaMemcpy(M.d_x, xs.data(), size_t(rows) * D * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
    return false;
  k_mlp_forward<<<(rows + 7) / 8, 256>>>(M.d_params, M.d_x, rows, M.d_y);
  out->resize(rows);
  return cudaGetLastError() == cudaSuccess &&
         cudaMemcpy(out->data(), M.d_y, size_t(rows) * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess;
}

bool learned_choose(int prec, int64_t n, const PlanHint& hint, std::string* token) {
  using namespace mlp;
  Model& M = model();
  std::lock_guard<std::mutex> g(M.mu);
  model_try_default();
  if (!M.loaded) return false;
  // candidates of a kind the model has no features for are left out
  std::vector<std::string> toks;
  std::vector<float> xs;
  for (const std::string& t : variant_tokens(prec, n)) {
    float f[D];
    if (!plan_features(prec, n, hint.batch, hint.stride, hint.real, t, f)) continue;
    for (int d = 0; d < D; ++d) xs.push_back((f[d] - M.norm[d]) / M.norm[D + d]);
    toks.push_back(t);
  }
  if (toks.size() < 2) return false;
  std::vector<float> pred;
  if (!model_predict(xs, int(toks.size()), &pred)) return false;
  size_t best = 0;
  for (size_t i = 1; i < pred.size(); ++i)
    if (pred[i] < pred[best]) best = i;
  *token = toks[best];
  return true;
}

}  // namespace gfft

using namespace gfft;

extern "C" {

void gfft_mlp_sizes(int32_t* in_dim, int32_t* hidden, int64_t* nparams) {
  if (in_dim) *in_dim = mlp::D;
  if (hidden) *hidden = mlp::H;
  if (nparams) *nparams = mlp::NP;
}

gfft_status gfft_mlp_forward(const float* params, const float* x, int64_t n, float* out, void* stream) {
  clear_error();
  if (!params || !x || !out) return GFFT_ERR_NIL_SLICE;
  if (n < 1) return GFFT_ERR_INVALID_LENGTH;
  const int64_t blocks = std::min<int64_t>((n + 7) / 8, 148 * 16);
  mlp::k_mlp_forward<<<unsigned(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(params, x, n, out);
  GFFT_CUDA(cudaGetLastError());
  return GFFT_OK;
}

static gfft_status mlp_launch(float* params, float* am, float* av, const float* x, const float* y, int64_t n, int steps,
                              int batch, float lr, uint64_t seed, int64_t step0, int train, float* loss, float* grad,
                              cudaStream_t st) {
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(&mlp::k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(mlp::SM_TOTAL * sizeof(float)));
  });
  GFFT_CUDA(attr);
  mlp::k_mlp_train<<<1, mlp::TPB, mlp::SM_TOTAL * sizeof(float), st>>>(params, am, av, x, y, n, steps, batch, lr,
                                                                       seed, step0, train, loss, grad);
  GFFT_CUDA(cudaGetLastError());
  return GFFT_OK;
}

gfft_status gfft_mlp_grad(const float* params, const float* x, const float* y, int64_t n, float* grad, float* loss,
                          void* stream) {
  clear_error();
  if (!params || !x || !y || !grad) return GFFT_ERR_NIL_SLICE;
  if (n < 1 || n > mlp::MAXB) {
    set_error("gfft_mlp_grad takes 1..64 samples");
    return GFFT_ERR_INVALID_LENGTH;
  }
  return mlp_launch(const_cast<float*>(params), nullptr, nullptr, x, y, n, 1, int(n), 0.f, 0, 0, 0, loss, grad,
                    static_cast<cudaStream_t>(stream));
}

gfft_status gfft_mlp_train(float* params, float* adam_m, float* adam_v, const float* x, const float* y, int64_t n,
                           int32_t steps, int32_t batch, float lr, uint64_t seed, int64_t step0, float* loss,
                           void* stream) {
  clear_error();
  if (!params || !adam_m || !adam_v || !x || !y) return GFFT_ERR_NIL_SLICE;
  if (n < 1 || steps < 1 || batch < 1 || batch > mlp::MAXB || step0 < 0) return GFFT_ERR_INVALID_LENGTH;
  if (!(lr > 0.f)) return GFFT_ERR_INVALID_ARGUMENT;
  return mlp_launch(params, adam_m, adam_v, x, y, n, steps, batch, lr, seed, step0, 1, loss, nullptr,
                    static_cast<cudaStream_t>(stream));
}

gfft_status gfft_planner_features(int32_t precision, int64_t n, int64_t batch, int64_t stride, int32_t real,
                                  const char* token, float* out) {
  clear_error();
  if (!token || !out) return GFFT_ERR_NIL_SLICE;
  if (precision != GFFT_COMPLEX64 && precision != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  if (n < 1) return GFFT_ERR_INVALID_LENGTH;
  if (!plan_features(precision, n, batch, stride, real, token, out)) {
    set_error(std::string("unknown variant token '") + token + "'");
    return GFFT_ERR_INVALID_ARGUMENT;
  }
  return GFFT_OK;
}

gfft_status gfft_planner_set_model(const float* params, const float* norm) {
  clear_error();
  mlp::Model& M = mlp::model();
  std::lock_guard<std::mutex> g(M.mu);
  M.tried_default = true;
  return model_install(params, norm);
}

gfft_status gfft_planner_load_model(const char* path) {
  clear_error();
  if (!path) return GFFT_ERR_NIL_SLICE;
  mlp::Model& M = mlp::model();
  std::lock_guard<std::mutex> g(M.mu);
  M.tried_default = true;
  return model_load_file(path);
}

int32_t gfft_planner_has_model(void) {
  mlp::Model& M = mlp::model();
  std::lock_guard<std::mutex> g(M.mu);
  model_try_default();
  return M.loaded ? 1 : 0;
}

gfft_status gfft_planner_choose(int32_t precision, int64_t n, int64_t batch, int64_t stride, int32_t real, char* token,
                                size_t cap) {
  clear_error();
  if (!token || cap == 0) return GFFT_ERR_NIL_SLICE;
  if (precision != GFFT_COMPLEX64 && precision != GFFT_COMPLEX128) return GFFT_ERR_INVALID_ARGUMENT;
  if (n < 1) return GFFT_ERR_INVALID_LENGTH;
  PlanHint h;
  h.planner = GFFT_PLANNER_LEARNED;
  h.batch = batch;
  h.stride = stride;
  h.real = real;
  std::string tok;
  if (!learned_choose(precision, n, h, &tok)) {
    set_error("no model loaded, or fewer than two variants for this length");
    return GFFT_ERR_NOT_IMPLEMENTED;
  }
  std::strncpy(token, tok.c_str(), cap - 1);
  token[cap - 1] = 0;
  return GFFT_OK;
}

}  // extern "C"
