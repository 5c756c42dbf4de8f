// Three-pass schedule for the largest power-of-two lengths (N = 2^21..2^24):
// N = N1 * M, M = M1 * M2, every factor <= 256, so every pass is a column
// FFT of at most 256 points over tiles of 16..64 adjacent columns (rows of
// 128..512 bytes), where the two-pass split must use 2048..4096-row columns
// whose tiles hold only 2..8 columns.
//
// Index maps: n = M n1 + m, m = M2 m1 + m2; k = k1 + N1 k', k' = k'1 + M1 k'2.
//   pass 1: for each column m of x (an N1 x M matrix): FFT over n1,
//           x W_N^{m k1}, transposed store Y[m][k1] (rows of N1) -- the
//           two-pass kernel's first pass;
//   pass 2: for each (m2, k1): FFT over m1 of Y[M2 m1 + m2][k1],
//           x W_M^{m2 k'1}, stored in place as Z[M2 k'1 + m2][k1];
//   pass 3: for each (k'1, k1): FFT over m2 of Z[M2 k'1 + m2][k1], stored
//           at X[k1 + N1 k'1 + N1 M1 k'2] (natural order).
// Passes 2 and 3 take NC adjacent k1 per tile, so every access is a run of
// NC contiguous elements.  Each pass is one plain launch over a chunk of
// transforms; the intermediate lives in scratch (in place for pass 2).
#pragma once
#include "gfft_twopass.cuh"

namespace gfft {

struct ThreePassParams {
  const void* src;
  void* dst;
  void* scratch;        // chunk of transforms x N elements
  int64_t idist, odist;
  const void* tw1;      // W_N1
  const void* tw2;      // W_M1
  const void* tw3;      // W_M2
  BigTwiddle bt;        // W_N (pass-1 twiddle)
  BigTwiddle btm;       // W_M (pass-2 twiddle)
  double scale;         // applied by pass 3 (1/N for the inverse)
  unsigned* status;     // set to 1 when a bounded wait of a TMA-staged pass expires
  unsigned spin_limit;  // try_wait rounds of that wait
};

template <typename C, int N1, int E1, int C1, int M1, int E2, int C2, int M2, int E3, int C3, int DIR>
struct ThreePass {
  using S1 = ColShape<N1, E1, C1, sizeof(C)>;
  using S2 = ColShape<M1, E2, C2, sizeof(C)>;
  using S3 = ColShape<M2, E3, C3, sizeof(C)>;
  static constexpr int64_t M = int64_t(M1) * M2;
  static constexpr int64_t N = int64_t(N1) * M;
  static constexpr int64_t TILES1 = M / C1;                   // pass 1: C1 columns m
  static constexpr int64_t TILES2 = int64_t(M2) * (N1 / C2);  // pass 2: (m2, C2 columns k1)
  static constexpr int64_t TILES3 = int64_t(M1) * (N1 / C3);  // pass 3: (k'1, C3 columns k1)
  static constexpr int TPB = S1::TPB > S2::TPB ? (S1::TPB > S3::TPB ? S1::TPB : S3::TPB)
                                               : (S2::TPB > S3::TPB ? S2::TPB : S3::TPB);
  static constexpr int SMEM = S1::SMEM > S2::SMEM ? (S1::SMEM > S3::SMEM ? S1::SMEM : S3::SMEM)
                                                  : (S2::SMEM > S3::SMEM ? S2::SMEM : S3::SMEM);
  static constexpr int EPT = E1 > E2 ? (E1 > E3 ? E1 : E3) : (E2 > E3 ? E2 : E3);
};

template <typename C, int N1, int E1, int C1, int M1, int E2, int C2, int M2, int E3, int C3, int DIR, int PASS>
__global__ void __launch_bounds__(ThreePass<C, N1, E1, C1, M1, E2, C2, M2, E3, C3, DIR>::TPB)
k_tp3(ThreePassParams p, int64_t b0) {
  using TP = ThreePass<C, N1, E1, C1, M1, E2, C2, M2, E3, C3, DIR>;
  using Re = typename RealOf<C>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sh = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x;
  C* scratch = static_cast<C*>(p.scratch);
  C v[TP::EPT];
  if constexpr (PASS == 1) {
    using S = typename TP::S1;
    const int64_t bl = blockIdx.x / TP::TILES1;
    const int col0 = int(blockIdx.x % TP::TILES1) * C1;
    const int c = tid % C1, t = tid / C1;
    const C* in = static_cast<const C*>(p.src) + (b0 + bl) * p.idist + col0;
    C* y = scratch + bl * TP::N;
    col_stage<C, N1, E1, C1, DIR, 1, LOAD_STREAM, OUT_SMEM_TWIDDLE, TP::M, 0>(
        v, in, nullptr, sh, t, c, tid < S::TPB, static_cast<const C*>(p.tw1), Re(1), p.bt, int64_t(col0 + c));
    for (int e = tid; e < N1 * C1; e += TP::TPB) {  // Y[m][k1], rows of N1
      const int cc = e / N1, row = e % N1;
      __stcg(y + int64_t(col0 + cc) * N1 + row, sh[S::phys(row, cc)]);
    }
  } else if constexpr (PASS == 2) {
    using S = typename TP::S2;
    const int64_t bl = blockIdx.x / TP::TILES2, r = blockIdx.x % TP::TILES2;
    const int m2 = int(r / (N1 / C2)), col0 = int(r % (N1 / C2)) * C2;
    const int c = tid % C2, t = tid / C2;
    C* base = scratch + bl * TP::N + int64_t(m2) * N1 + col0;  // row m1 at base + m1 * M2 * N1
    col_stage<C, M1, E2, C2, DIR, 1, LOAD_L2, OUT_SMEM_TWIDDLE, int64_t(M2) * N1, 0>(
        v, base, nullptr, sh, t, c, tid < S::TPB, static_cast<const C*>(p.tw2), Re(1), p.btm, int64_t(m2));
    for (int e = tid; e < M1 * C2; e += TP::TPB) {  // back in place, row k'1
      const int row = e / C2, cc = e % C2;
      __stcg(base + int64_t(row) * M2 * N1 + cc, sh[S::phys(row, cc)]);
    }
  } else {
    using S = typename TP::S3;
    const int64_t bl = blockIdx.x / TP::TILES3, r = blockIdx.x % TP::TILES3;
    const int k1p = int(r / (N1 / C3)), col0 = int(r % (N1 / C3)) * C3;
    const int c = tid % C3, t = tid / C3;
    const C* in = scratch + bl * TP::N + int64_t(M2) * k1p * N1 + col0;  // row m2 at in + m2 * N1
    C* out = static_cast<C*>(p.dst) + (b0 + bl) * p.odist + int64_t(N1) * k1p + col0;
    col_stage<C, M2, E3, C3, DIR, 1, LOAD_L2, OUT_COLUMNS, N1, int64_t(N1) * M1>(
        v, in, out, sh, t, c, tid < S::TPB, static_cast<const C*>(p.tw3), Re(p.scale), p.bt, 0);
  }
}

}  // namespace gfft
