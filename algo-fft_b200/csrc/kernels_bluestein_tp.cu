// Bluestein chain for FFT lengths M = 2^15..2^20 (two-pass FFT_M) with the
// element-wise steps fused into the passes: the chirp multiply and zero pad
// into the loads of the forward FFT's first pass, the filter product into
// the stores of its second pass, the chirp multiply (with 1/M, and 1/n for
// the inverse) into the stores of the inverse FFT's second pass, which
// writes only the n outputs.  Four launches and about 6 M + 2 n element
// transfers per transform, where the separate chain (plan_bluestein.go:7-58,
// internal/kernels/bluestein.go:20-77: pad, FFT, product, IFFT, chirp) moves
// about 13 M.
//
// Index maps are the two-pass kernels' (gfft_twopass.cuh): input m = N2 n1
// + n2 (pass 1 reads columns n2), output k = k1 + N1 k2 (pass 2 writes
// column k1, row k2).
#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>
#include "gfft_internal.h"
#include "kernels_twopass.cuh"

namespace gfft {
namespace {

// chirp-weighted, zero-padded input: m = row * N2 + col0 + c
template <typename C>
struct BsChirpIn {
  const C* x;  // this transform's input
  const C* w;
  int64_t n, n2, col0;
  __device__ __forceinline__ C load(int row, int c) const {
    const int64_t m = int64_t(row) * n2 + col0 + c;
    return m < n ? cmul(ld_stream(x + m), __ldg(w + m)) : C{0, 0};
  }
};

// spectrum times the filter, k = col0 + c + N1 * row, kept in L2 for the
// inverse FFT that reads it next
template <typename C>
struct BsFilterOut {
  C* y;  // this transform's work row
  const C* f;
  int64_t n1, col0;
  __device__ __forceinline__ void store(int row, int c, C v) const {
    const int64_t k = col0 + c + n1 * int64_t(row);
    __stcg(y + k, cmul(v, __ldg(f + k)));
  }
};

// outputs k < n times the chirp and the user scale (1/M is already in v)
template <typename C>
struct BsChirpOut {
  C* y;  // this transform's output
  const C* w;
  int64_t n, n1, col0;
  typename RealOf<C>::type scale;
  __device__ __forceinline__ void store(int row, int c, C v) const {
    const int64_t k = col0 + c + n1 * int64_t(row);
    if (k < n) st_stream(y + k, cscale(cmul(v, __ldg(w + k)), scale));
  }
};

struct BsTpParams {
  const void* x;     // user input
  void* out;         // user output
  void* scratch;     // pass-1 intermediate, chunk x M
  void* work;        // spectrum times filter, chunk x M
  const void* w;     // chirp of the direction
  const void* f;     // filter spectrum of the direction
  const void* tw1;   // W_N1
  const void* tw2;   // W_N2
  BigTwiddle bt;     // W_M
  int64_t n, idist, odist;
  double inv_m, scale;
};

enum { BS_FWD1 = 0, BS_FWD2 = 1, BS_INV2 = 2 };

template <typename C, int N1, int EPT1, int NC1, int N2, int EPT2, int NC2, int KIND>
__global__ void __launch_bounds__(TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, -1>::TPB,
                                  TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, -1>::MIN_BLOCKS)
k_bs_tp(BsTpParams p, int64_t b0) {
  using TP = TwoPass<C, N1, EPT1, NC1, N2, EPT2, NC2, -1>;
  using S1 = typename TP::S1;
  using S2 = typename TP::S2;
  using Re = typename RealOf<C>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x;
  C* scratch = static_cast<C*>(p.scratch);
  C v[TP::EPT];
  if constexpr (KIND == BS_FWD1) {
    const int64_t bl = blockIdx.x / TP::TILES1;
    const int col0 = int(blockIdx.x % TP::TILES1) * NC1;
    const bool active = tid < S1::TPB;
    const int c = tid % NC1, t = tid / NC1;
    const BsChirpIn<C> io{static_cast<const C*>(p.x) + (b0 + bl) * p.idist, static_cast<const C*>(p.w), p.n, N2,
                          col0};
    C* y = scratch + bl * TP::N;
    col_stage<C, N1, EPT1, NC1, -1, 1, LOAD_FN, OUT_SMEM_TWIDDLE, N2, 0, false, BsChirpIn<C>>(
        v, nullptr, nullptr, sh, t, c, active, static_cast<const C*>(p.tw1), Re(1), p.bt, int64_t(col0 + c), 0,
        io);
    for (int e = tid; e < N1 * NC1; e += TP::TPB) {
      const int cc = e / N1, row = e % N1;
      __stcg(y + int64_t(col0 + cc) * N1 + row, sh[S1::phys(row, cc)]);
    }
  } else {
    const int64_t bl = blockIdx.x / TP::TILES2;
    const int col0 = int(blockIdx.x % TP::TILES2) * NC2;
    const bool active = tid < S2::TPB;
    const int c = tid % NC2, t = tid / NC2;
    const C* y = scratch + bl * TP::N + col0;
    if constexpr (KIND == BS_FWD2) {
      const BsFilterOut<C> io{static_cast<C*>(p.work) + bl * TP::N, static_cast<const C*>(p.f), N1, col0};
      col_stage<C, N2, EPT2, NC2, -1, 1, LOAD_L2, OUT_FN, N1, N1, false, BsFilterOut<C>>(
          v, y, nullptr, sh, t, c, active, static_cast<const C*>(p.tw2), Re(1), p.bt, 0, 0, io);
    } else {
      const BsChirpOut<C> io{static_cast<C*>(p.out) + (b0 + bl) * p.odist, static_cast<const C*>(p.w), p.n, N1, col0,
                             Re(p.scale)};
      col_stage<C, N2, EPT2, NC2, +1, 1, LOAD_L2, OUT_FN, N1, N1, false, BsChirpOut<C>>(
          v, y, nullptr, sh, t, c, active, static_cast<const C*>(p.tw2), Re(p.inv_m), p.bt, 0, 0, io);
    }
  }
}

struct BsTpKernel {
  int prec;
  int64_t m;
  int n1;
  int tpb, smem;
  const void* fn[4];  // the three fused passes and this file's plain inverse first pass
  cudaError_t (*run)(const BsTpParams& p, int64_t count, void* scratch, void* work, cudaStream_t st);
};

std::vector<BsTpKernel>& table() {
  static std::vector<BsTpKernel> t;
  return t;
}

template <typename C, int N1, int N2>
struct BsTpOf {
  static constexpr int TE = sizeof(C) == 8 ? 8192 : 4096, EMAX = sizeof(C) == 8 ? 32 : 8;
  using A = TileRule<TE, EMAX, N1>;
  using B = TileRule<TE, EMAX, N2>;
  using TP = TwoPass<C, N1, A::EPT, A::NC, N2, B::EPT, B::NC, -1>;
  template <int KIND>
  static const void* fn() {
    return reinterpret_cast<const void*>(&k_bs_tp<C, N1, A::EPT, A::NC, N2, B::EPT, B::NC, KIND>);
  }
  // The whole chain over `count` transforms in chunks that fill the
  // scratch and work buffers (bluestein_tp_chunk_bytes each).
  static cudaError_t run(const BsTpParams& p0, int64_t count, void* scratch, void* work, cudaStream_t st) {
    BsTpParams p = p0;
    p.scratch = scratch;
    p.work = work;
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(256) << 20) / (TP::N * int64_t(sizeof(C)))));
    TwoPassParams q{};
    q.scratch = scratch;
    q.idist = TP::N;
    q.tw1 = p.tw1;
    q.tw2 = p.tw2;
    q.bt = p.bt;
    for (int64_t b0 = 0; b0 < count; b0 += chunk) {
      const int64_t nb = std::min(chunk, count - b0);
      k_bs_tp<C, N1, A::EPT, A::NC, N2, B::EPT, B::NC, BS_FWD1>
          <<<unsigned(nb * TP::TILES1), TP::TPB, TP::SMEM, st>>>(p, b0);
      k_bs_tp<C, N1, A::EPT, A::NC, N2, B::EPT, B::NC, BS_FWD2>
          <<<unsigned(nb * TP::TILES2), TP::TPB, TP::SMEM, st>>>(p, b0);
      // inverse FFT, first pass: plain, from the work rows into scratch
      q.src = work;
      k_tp_split<C, N1, A::EPT, A::NC, N2, B::EPT, B::NC, +1, 1>
          <<<unsigned(nb * TP::TILES1), TP::TPB, TP::SMEM, st>>>(q, 0);
      k_bs_tp<C, N1, A::EPT, A::NC, N2, B::EPT, B::NC, BS_INV2>
          <<<unsigned(nb * TP::TILES2), TP::TPB, TP::SMEM, st>>>(p, b0);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
};

template <typename C, int N1, int N2>
void reg() {
  using O = BsTpOf<C, N1, N2>;
  BsTpKernel k;
  k.prec = sizeof(C) == 8 ? kC64 : kC128;
  k.m = int64_t(N1) * N2;
  k.n1 = N1;
  k.tpb = O::TP::TPB;
  k.smem = O::TP::SMEM;
  k.fn[0] = O::template fn<BS_FWD1>();
  k.fn[1] = O::template fn<BS_FWD2>();
  k.fn[2] = O::template fn<BS_INV2>();
  k.fn[3] = reinterpret_cast<const void*>(
      &k_tp_split<C, N1, O::A::EPT, O::A::NC, N2, O::B::EPT, O::B::NC, +1, 1>);
  k.run = &O::run;
  table().push_back(k);
}

struct RegBsTp {
  RegBsTp() {
    reg<float2, 128, 256>();
    reg<float2, 256, 256>();
    reg<float2, 256, 512>();
    reg<float2, 512, 512>();
    reg<float2, 512, 1024>();
    reg<float2, 1024, 1024>();
    reg<double2, 128, 256>();
    reg<double2, 256, 256>();
    reg<double2, 256, 512>();
    reg<double2, 512, 512>();
    reg<double2, 512, 1024>();
    reg<double2, 1024, 1024>();
  }
} reg_bs_tp;

}  // namespace

bool bluestein_tp_supported(int prec, int64_t M, int n1) {
  for (const auto& k : table())
    if (k.prec == prec && k.m == M && k.n1 == n1) return true;
  return false;
}

size_t bluestein_tp_chunk_bytes(int prec, int64_t M, int64_t count) {
  const int64_t es = prec == kC64 ? 8 : 16;
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t(256) << 20) / (M * es)));
  return size_t(chunk) * size_t(M) * size_t(es);
}

cudaError_t exec_bluestein_tp(int prec, int64_t M, const void* src, void* dst, int64_t count, int64_t idist,
                              int64_t odist, int64_t n, const void* chirp, const void* filt, const void* tw1,
                              const void* tw2, BigTwiddle bt, double scale, void* scratch, void* work,
                              cudaStream_t st) {
  static std::mutex mu;
  static std::vector<std::pair<const void*, int>> done;  // (kernel, device) with the smem limit raised
  for (const auto& k : table()) {
    if (k.prec != prec || k.m != M) continue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
      std::lock_guard<std::mutex> g(mu);
      if (std::find(done.begin(), done.end(), std::make_pair(k.fn[0], dev)) == done.end()) {
        if (k.smem > 48 * 1024)
          for (const void* f : k.fn) {
            e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
            if (e != cudaSuccess) return e;
          }
        done.push_back({k.fn[0], dev});
      }
    }
    BsTpParams p{};
    p.x = src;
    p.out = dst;
    p.w = chirp;
    p.f = filt;
    p.tw1 = tw1;
    p.tw2 = tw2;
    p.bt = bt;
    p.n = n;
    p.idist = idist;
    p.odist = odist;
    p.inv_m = 1.0 / double(M);
    p.scale = scale;
    return k.run(p, count, scratch, work, st);
  }
  return cudaErrorNotSupported;
}

}  // namespace gfft
