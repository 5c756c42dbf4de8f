// Bluestein chain for FFT lengths M = 2^21..2^24 on the three-pass FFT_M
// (gfft_threepass.cuh, split M = N1 x M1 x M2 as the plain three-pass plans)
// with the element-wise steps fused into the passes:
//   BS3_FWD1  the forward FFT's first pass, its loads the chirp-weighted,
//             zero-padded input a_m = x_m w_m (m < n), scratch out;
//   the forward second pass is the plain three-pass kernel (scratch, in place);
//   BS3_FWD3  the forward third pass, its stores the spectrum times the
//             filter, Z_k = A_k F_k, in natural order into the work buffer;
//   the inverse first and second passes are the plain kernels (work to
//             scratch, scratch in place);
//   BS3_INV3  the inverse third pass, its stores y_k = w_k z_k / M (and the
//             transform's scale) for k < n only, into the user's output.
// Six launches and about 12 M + 2 n element transfers per transform,
// against about 16 M + 2 n for the separate chain of pad, FFT, product,
// IFFT and chirp (plan_bluestein.go:7-58, internal/kernels/bluestein.go:20-77).
//
// Index maps are the three-pass kernels': input m = (M1 M2) n1 + m', output
// k = k1 + N1 k'1 + N1 M1 k'2 (pass 3 writes column k1 of row group k'1,
// rows k'2).
#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>
#include "gfft_internal.h"
#include "gfft_threepass.cuh"
#include "kernels_twopass.cuh"

namespace gfft {
namespace {

enum { BS3_FWD1 = 0, BS3_FWD3 = 1, BS3_INV3 = 2 };

struct Bs3Params {
  const void* x;      // user input
  void* y;            // user output
  void* scratch;      // chunk x M: the passes' intermediate
  void* work;         // chunk x M: spectrum times filter
  const void* w;      // chirp of the direction asked for (n)
  const void* f;      // filter spectrum of that direction (M)
  const void* tw1;    // W_N1
  const void* tw3;    // W_M2
  BigTwiddle bt;      // W_M (pass-1 twiddle)
  int64_t n, idist, odist;
  double inv_m;       // 1/M
  double scale;       // 1 for the forward transform, 1/n for the inverse
};

// chirp-weighted, zero-padded input: m = row * pitch + col0 + c
template <typename C>
struct Bs3In {
  const C* x;
  const C* w;
  int64_t n, pitch, col0;
  __device__ __forceinline__ C load(int row, int c) const {
    const int64_t m = int64_t(row) * pitch + col0 + c;
    return m < n ? cmul(ld_stream(x + m), __ldg(w + m)) : C{0, 0};
  }
};

// spectrum k = base + c + rstride * row times F_k into the work row
template <typename C>
struct Bs3Filt {
  C* z;
  const C* f;
  int64_t base, rstride;
  __device__ __forceinline__ void store(int row, int c, C v) const {
    const int64_t k = base + c + rstride * int64_t(row);
    __stcg(z + k, cmul(v, __ldg(f + k)));
  }
};

// outputs k < n times the chirp and the transform's scale (1/M is in v)
template <typename C>
struct Bs3Out {
  C* y;
  const C* w;
  int64_t n, base, rstride;
  typename RealOf<C>::type scale;
  __device__ __forceinline__ void store(int row, int c, C v) const {
    const int64_t k = base + c + rstride * int64_t(row);
    if (k < n) st_stream(y + k, cscale(cmul(v, __ldg(w + k)), scale));
  }
};

template <typename C, int N1, int E1, int C1, int M1, int E2, int C2, int M2, int E3, int C3, int KIND>
__global__ void __launch_bounds__(ThreePass<C, N1, E1, C1, M1, E2, C2, M2, E3, C3, -1>::TPB)
k_bs_tp3(Bs3Params p, int64_t b0) {
  using TP = ThreePass<C, N1, E1, C1, M1, E2, C2, M2, E3, C3, -1>;
  using Re = typename RealOf<C>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x;
  C* scratch = static_cast<C*>(p.scratch);
  C v[TP::EPT];
  if constexpr (KIND == BS3_FWD1) {
    using S = typename TP::S1;
    const int64_t bl = blockIdx.x / TP::TILES1;
    const int col0 = int(blockIdx.x % TP::TILES1) * C1;
    const int c = tid % C1, t = tid / C1;
    const Bs3In<C> io{static_cast<const C*>(p.x) + (b0 + bl) * p.idist, static_cast<const C*>(p.w), p.n, TP::M,
                      col0};
    C* y = scratch + bl * TP::N;
    col_stage<C, N1, E1, C1, -1, 1, LOAD_FN, OUT_SMEM_TWIDDLE, TP::M, 0, false, Bs3In<C>>(
        v, nullptr, nullptr, sh, t, c, tid < S::TPB, static_cast<const C*>(p.tw1), Re(1), p.bt, int64_t(col0 + c), 0,
        io);
    for (int e = tid; e < N1 * C1; e += TP::TPB) {  // Y[m][k1], rows of N1
      const int cc = e / N1, row = e % N1;
      __stcg(y + int64_t(col0 + cc) * N1 + row, sh[S::phys(row, cc)]);
    }
  } else {
    using S = typename TP::S3;
    const int64_t bl = blockIdx.x / TP::TILES3, r = blockIdx.x % TP::TILES3;
    const int k1p = int(r / (N1 / C3)), col0 = int(r % (N1 / C3)) * C3;
    const int c = tid % C3, t = tid / C3;
    const C* in = scratch + bl * TP::N + int64_t(M2) * k1p * N1 + col0;  // row m2 at in + m2 * N1
    const int64_t base = int64_t(N1) * k1p + col0;
    constexpr int64_t RSTR = int64_t(N1) * M1;
    if constexpr (KIND == BS3_FWD3) {
      const Bs3Filt<C> io{static_cast<C*>(p.work) + bl * TP::N, static_cast<const C*>(p.f), base, RSTR};
      col_stage<C, M2, E3, C3, -1, 1, LOAD_L2, OUT_FN, N1, RSTR, false, Bs3Filt<C>>(
          v, in, nullptr, sh, t, c, tid < S::TPB, static_cast<const C*>(p.tw3), Re(1), p.bt, 0, 0, io);
    } else {
      const Bs3Out<C> io{static_cast<C*>(p.y) + (b0 + bl) * p.odist, static_cast<const C*>(p.w), p.n, base, RSTR,
                         Re(p.scale)};
      col_stage<C, M2, E3, C3, +1, 1, LOAD_L2, OUT_FN, N1, RSTR, false, Bs3Out<C>>(
          v, in, nullptr, sh, t, c, tid < S::TPB, static_cast<const C*>(p.tw3), Re(p.inv_m), p.bt, 0, 0, io);
    }
  }
}

using Bs3Fn = cudaError_t (*)(const Bs3Params& p, int kind, int64_t b0, int64_t nb, cudaStream_t st);

struct Bs3Kernel {
  int prec, n1, m1, m2;
  int smem;
  const void* fn[3];
  Bs3Fn launch;
};

std::vector<Bs3Kernel>& table() {
  static std::vector<Bs3Kernel> t;
  return t;
}

// The tile shapes of the plain three-pass kernels of the same split.
template <typename C, int N1, int M1, int M2>
struct Bs3Of {
  static constexpr int TE = sizeof(C) == 8 ? 8192 : 4096, EMAX = sizeof(C) == 8 ? 16 : 8;
  using A = TileRule<TE, EMAX, N1>;
  using B = TileRule<TE, EMAX, M1>;
  using D = TileRule<TE, EMAX, M2>;
  using TP = ThreePass<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, -1>;
  template <int KIND>
  static const void* fn() {
    return reinterpret_cast<const void*>(&k_bs_tp3<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, KIND>);
  }
  static cudaError_t launch(const Bs3Params& p, int kind, int64_t b0, int64_t nb, cudaStream_t st) {
    const int64_t tiles = nb * (kind == BS3_FWD1 ? TP::TILES1 : TP::TILES3);
    if (tiles <= 0) return cudaSuccess;
    if (tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    const unsigned g = unsigned(tiles);
    if (kind == BS3_FWD1)
      k_bs_tp3<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, BS3_FWD1><<<g, TP::TPB, TP::SMEM, st>>>(p, b0);
    else if (kind == BS3_FWD3)
      k_bs_tp3<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, BS3_FWD3><<<g, TP::TPB, TP::SMEM, st>>>(p, b0);
    else
      k_bs_tp3<C, N1, A::EPT, A::NC, M1, B::EPT, B::NC, M2, D::EPT, D::NC, BS3_INV3><<<g, TP::TPB, TP::SMEM, st>>>(p, b0);
    return cudaGetLastError();
  }
};

template <typename C, int N1, int M1, int M2>
void reg() {
  using K = Bs3Of<C, N1, M1, M2>;
  Bs3Kernel k;
  k.prec = sizeof(C) == 8 ? kC64 : kC128;
  k.n1 = N1;
  k.m1 = M1;
  k.m2 = M2;
  k.smem = K::TP::SMEM;
  k.fn[0] = K::template fn<BS3_FWD1>();
  k.fn[1] = K::template fn<BS3_FWD3>();
  k.fn[2] = K::template fn<BS3_INV3>();
  k.launch = &K::launch;
  table().push_back(k);
}

// the splits of the plain three-pass kernels (kernels_threepass.cu)
struct RegBs3 {
  RegBs3() {
    reg<float2, 128, 128, 128>();
    reg<float2, 256, 128, 128>();
    reg<float2, 256, 256, 128>();
    reg<float2, 256, 256, 256>();
    reg<double2, 128, 128, 128>();
    reg<double2, 256, 128, 128>();
    reg<double2, 256, 256, 128>();
    reg<double2, 256, 256, 256>();
  }
} reg_bs_tp3;

// The chain kernels of this split, with their shared-memory limit raised
// once per device.
const Bs3Kernel* bs3_ready(int prec, const ThreePassKernel* plain, cudaError_t* err) {
  static std::mutex mu;
  static std::vector<std::pair<const void*, int>> done;
  *err = cudaSuccess;
  for (const auto& k : table()) {
    if (k.prec != prec || k.n1 != plain->n1 || k.m1 != plain->m1 || k.m2 != plain->m2) continue;
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> g(mu);
    if (std::find(done.begin(), done.end(), std::make_pair(k.fn[0], dev)) == done.end()) {
      if (k.smem > 48 * 1024)
        for (const void* f : k.fn) {
          *err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
          if (*err != cudaSuccess) return nullptr;
        }
      done.push_back({k.fn[0], dev});
    }
    return &k;
  }
  *err = cudaErrorNotSupported;
  return nullptr;
}

}  // namespace

bool bluestein_tp3_supported(int prec, int64_t M) {
  const ThreePassKernel* f = find_threepass(prec, M, -1);
  if (!f || !find_threepass(prec, M, +1)) return false;
  for (const auto& k : table())
    if (k.prec == prec && k.n1 == f->n1 && k.m1 == f->m1 && k.m2 == f->m2) return true;
  return false;
}

gfft_status exec_bluestein_tp3(const PlanCore* sub, const void* src, void* dst, int64_t count, int64_t idist,
                               int64_t odist, int64_t n, const void* chirp, const void* filt, double scale,
                               cudaStream_t st) {
  const ThreePassKernel* kf = sub->t3[0];
  const ThreePassKernel* ki = sub->t3[1];
  if (!kf || !ki || kf->tma || ki->tma) return GFFT_ERR_NOT_IMPLEMENTED;
  cudaError_t e;
  const Bs3Kernel* k = bs3_ready(sub->prec, kf, &e);
  if (!k) return cuda_status(e, "k_bs_tp3");
  const int64_t M = sub->n;
  const int64_t es = int64_t(elem_bytes(sub->prec));
  // chunks of at most 512 MB per buffer, of equal size
  const int64_t cap = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(512) << 20) / (M * es)));
  const int64_t nchunks = (count + cap - 1) / cap;
  const int64_t chunk = (count + nchunks - 1) / nchunks;
  void* buf = nullptr;
  GFFT_CUDA(ws_alloc(&buf, 2 * size_t(chunk) * size_t(M) * size_t(es), st));
  void* scratch = buf;
  void* work = static_cast<char*>(buf) + size_t(chunk) * size_t(M) * size_t(es);
  const BigTwiddle bt{sub->bt_lo, sub->bt_hi, sub->bt_shift};
  Bs3Params p{};
  p.x = src;
  p.y = dst;
  p.scratch = scratch;
  p.work = work;
  p.w = chirp;
  p.f = filt;
  p.tw1 = sub->tw1;
  p.tw3 = sub->tw3;
  p.bt = bt;
  p.n = n;
  p.idist = idist;
  p.odist = odist;
  p.inv_m = 1.0 / double(M);
  p.scale = scale;
  // the plain passes: forward pass 2 on the scratch, inverse passes 1 (work
  // to scratch) and 2
  ThreePassParams q{};
  q.src = work;
  q.scratch = scratch;
  q.idist = M;
  q.tw1 = sub->tw1;
  q.tw2 = sub->tw2;
  q.tw3 = sub->tw3;
  q.bt = bt;
  q.btm = BigTwiddle{sub->btm_lo, sub->btm_hi, sub->btm_shift};
  q.status = sub->status;
  q.spin_limit = 1u << 22;
  for (int64_t b0 = 0; b0 < count && e == cudaSuccess; b0 += chunk) {
    const int64_t nb = std::min(chunk, count - b0);
    e = k->launch(p, BS3_FWD1, b0, nb, st);
    if (e == cudaSuccess) e = kf->launch(q, 2, 0, nb, st);
    if (e == cudaSuccess) e = k->launch(p, BS3_FWD3, b0, nb, st);
    if (e == cudaSuccess) e = ki->launch(q, 1, 0, nb, st);
    if (e == cudaSuccess) e = ki->launch(q, 2, 0, nb, st);
    if (e == cudaSuccess) e = k->launch(p, BS3_INV3, b0, nb, st);
  }
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) return cuda_status(e, "k_bs_tp3");
  return GFFT_OK;
}

}  // namespace gfft
