// TMA-staged form of the three-pass schedule (same index maps and the same
// intermediate layout as k_tp3, so a pass of either form can follow a pass
// of the other).
//
// Each pass is a persistent kernel: CTA b takes tiles b, b + grid, ...  A
// tile (L rows of NC adjacent columns) arrives in shared memory by one TMA
// tile copy into one of NST stage buffers; one thread keeps up to NST - 1
// copies in flight ahead of the tile being transformed, so the copy engine streams
// the next tiles while the threads run the Stockham stages in place on the
// current one (rows of NC elements, the layout the copy writes; whole-row
// warp accesses keep it bank-conflict free).  Stores:
//   pass 1: the twiddled columns are written transposed into the stage
//           buffer, in boxes of 128-byte rows in the copy engine's 128-byte
//           swizzle (bank-conflict free for the threads' writes), and leave
//           by L / RE TMA tile stores as whole columns, Y[m][k1];
//   pass 2: the twiddled tile goes back in place by one TMA tile store;
//   pass 3: the scaled tile goes to the output by one TMA tile store.
// A stage buffer is refilled only after the store that read it has finished
// reading (bulk-group wait).  Waits on the copies are bounded: on expiry the
// kernel sets the plan's status word, waits (bounded) for its own copies in
// flight and returns.
#pragma once
#include "gfft_threepass.cuh"
#include "gfft_tma.cuh"

namespace gfft {

// Tile rule of the TMA form: NC = TE / L columns (at most 64), EPT = EMAX
// with at least 8 threads per column.
template <int TE, int EMAX, int L>
struct TmaTile {
  static constexpr int NC0 = TE / L;
  static constexpr int NC = NC0 > 64 ? 64 : NC0;
  static constexpr int EPT = (L / EMAX >= 8) ? EMAX : (L / 8 >= 2 ? L / 8 : 2);
};

template <typename C, int N1, int M1, int M2, int TE, int EMAX, int NST, int PASS>
struct Tp3t {
  static constexpr int ES = sizeof(C);
  static constexpr int L = PASS == 1 ? N1 : PASS == 2 ? M1 : M2;
  using R = TmaTile<TE, EMAX, L>;
  static constexpr int NC = R::NC, EPT = R::EPT;
  static_assert(NC * ES >= 128, "TMA-staged tiles need rows of at least 128 bytes");
  static_assert(L <= 256, "one TMA box spans at most 256 rows");
  using S = ColShape<L, EPT, NC, ES, true>;
  static constexpr int TPB = S::TPB;
  static constexpr int64_t M = int64_t(M1) * M2;
  static constexpr int64_t N = int64_t(N1) * M;
  static constexpr int TILE_BYTES = L * NC * ES;
  static constexpr int RE = 128 / ES;  // elements per 128-byte row of a swizzled box
  static_assert(L % RE == 0, "whole swizzled boxes");
  // buffers on 1024-byte boundaries (the swizzle pattern repeats every 1 KB)
  static constexpr int BUF_BYTES = (L * NC * ES + 1023) / 1024 * 1024;
  static constexpr int SMEM = NST * BUF_BYTES + 1024;  // + alignment slack
  static constexpr int MINB = (200 * 1024) / SMEM < 1 ? 1 : ((200 * 1024) / SMEM > 4 ? 4 : (200 * 1024) / SMEM);
  static constexpr int64_t TILES = PASS == 1 ? M / NC : PASS == 2 ? int64_t(M2) * (N1 / NC) : int64_t(M1) * (N1 / NC);
  static constexpr int W = ES / 4;  // FP32 words per element (tensor-map x unit)
};

struct Tp3tArgs {
  int64_t tiles;         // tiles of this launch (transforms x TILES)
  const void* tw;        // W_L table of the pass
  BigTwiddle bt;         // pass 1: W_N; pass 2: W_M
  double scale;          // pass 3
  unsigned* status;
  unsigned spin_limit;
};

template <typename C, int N1, int M1, int M2, int TE, int EMAX, int NST, int DIR, int PASS>
__global__ void __launch_bounds__(Tp3t<C, N1, M1, M2, TE, EMAX, NST, PASS>::TPB,
                                  Tp3t<C, N1, M1, M2, TE, EMAX, NST, PASS>::MINB)
k_tp3t(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout, Tp3tArgs a) {
  using K = Tp3t<C, N1, M1, M2, TE, EMAX, NST, PASS>;
  using Re = typename RealOf<C>::type;
  constexpr int L = K::L, NC = K::NC, EPT = K::EPT, W = K::W;
  constexpr int BUFE = K::BUF_BYTES / K::ES;
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[NST];
  __shared__ int s_fail;
  __shared__ C s_tw[L];  // W_L, read by every tile's stages
  C* bufs = reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x;
  const int c = tid % NC, t = tid / NC;
  const int64_t nloc = a.tiles > blockIdx.x ? (a.tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

  // tile -> (transform, row coordinate, first column)
  auto decode = [&](int64_t tile, int64_t& bl, int& rowc, int& col0) {
    if constexpr (PASS == 1) {
      bl = tile / K::TILES;
      col0 = int(tile % K::TILES) * NC;
      rowc = 0;
    } else {
      bl = tile / K::TILES;
      const int r = int(tile % K::TILES);
      rowc = r / (N1 / NC);  // pass 2: m2; pass 3: k'1
      col0 = (r % (N1 / NC)) * NC;
    }
  };
  auto issue = [&](int64_t j) {
    int64_t bl;
    int rowc, col0;
    decode(blockIdx.x + j * gridDim.x, bl, rowc, col0);
    const int s = int(j % NST);
    mbar_expect_tx(&bar[s], K::TILE_BYTES);
    if constexpr (PASS == 1) tma_load_3d(bufs + s * BUFE, &tin, &bar[s], col0 * W, 0, int(bl));
    else if constexpr (PASS == 2) tma_load_4d(bufs + s * BUFE, &tin, &bar[s], col0 * W, rowc, 0, int(bl));
    else tma_load_3d(bufs + s * BUFE, &tin, &bar[s], col0 * W, M2 * rowc, int(bl));
  };

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
    fence_async_smem();
    s_fail = 0;
  }
  for (int i = tid; i < L; i += K::TPB) s_tw[i] = static_cast<const C*>(a.tw)[i];
  __syncthreads();
  int64_t issued = 0;  // meaningful in thread 0
  if (tid == 0)
    for (; issued < NST - 1 && issued < nloc; ++issued) issue(issued);

  C v[EPT];
  int64_t j = 0;
  // Refill of the buffer tile j - 1 used, with tile j + NST - 1.  With three
  // or more stages it comes after tile j's butterflies, when the store that
  // read that buffer (committed one tile earlier) has long finished; with
  // two it must come first, or no copy would overlap the butterflies.
  constexpr bool LATE = NST >= 3;
  auto refill = [&]() {
    if (tid == 0 && issued < nloc) {
      bulk_wait_read();
      fence_async_smem();
      issue(issued);
      ++issued;
    }
  };
  for (; j < nloc; ++j) {
    const int s = int(j % NST);
    C* sh = bufs + s * BUFE;
    if constexpr (!LATE) refill();
    // one thread waits for the copy; the barrier passes its completion on
    // to the others (the copy's writes are ordered before the phase flip
    // that thread 0 observes, and the barrier orders the rest after it)
    if (tid == 0 && !mbar_wait(&bar[s], uint32_t((j / NST) & 1), a.spin_limit)) s_fail = 1;
    __syncthreads();
    if (s_fail) break;
    int64_t bl;
    int rowc, col0;
    decode(blockIdx.x + j * gridDim.x, bl, rowc, col0);
    // every branch ends its butterflies with a fence for the copy engine and
    // a barrier, so the tile is complete in shared memory before its store
    if constexpr (PASS == 1) {
      col_stage<C, L, EPT, NC, DIR, 1, LOAD_SMEM, OUT_SMEM_TWIDDLE_SW, 1, 1, true>(
          v, nullptr, nullptr, sh, t, c, true, s_tw, Re(1), a.bt, int64_t(col0 + c));
      if constexpr (LATE) refill();
      if (tid == 0) {  // Y[m][k1]: box i holds rows k1 = i*RE.. of columns m = col0..
        for (int i = 0; i < L / K::RE; ++i) tma_store_3d(&tout, sh + i * NC * K::RE, i * K::RE * W, col0, int(bl));
        bulk_commit();
      }
    } else if constexpr (PASS == 2) {
      col_stage<C, L, EPT, NC, DIR, 1, LOAD_SMEM, OUT_SMEM_TWIDDLE, 1, 1, true>(
          v, nullptr, nullptr, sh, t, c, true, s_tw, Re(1), a.bt, int64_t(rowc));
      if constexpr (LATE) refill();
      if (tid == 0) {
        tma_store_4d(&tin, sh, col0 * W, rowc, 0, int(bl));  // in place
        bulk_commit();
      }
    } else {
      col_stage<C, L, EPT, NC, DIR, 1, LOAD_SMEM, OUT_SMEM, 1, 1, true>(
          v, nullptr, nullptr, sh, t, c, true, s_tw, Re(a.scale), a.bt, 0);
      fence_async_smem();
      __syncthreads();
      if constexpr (LATE) refill();
      if (tid == 0) {
        tma_store_4d(&tout, sh, col0 * W, rowc, 0, int(bl));
        bulk_commit();
      }
    }
    // the early refill of the next iteration reuses this buffer
    if constexpr (!LATE) __syncthreads();
  }
  if (tid == 0) {
    if (j < nloc) {
      // a wait expired: flag it, then let the copies still in flight land
      // (bounded) before the CTA's shared memory goes away
      atomicExch(a.status, 1u);
      for (int64_t k = j; k < issued; ++k)
        mbar_wait(&bar[int(k % NST)], uint32_t((k / NST) & 1), a.spin_limit);
    }
    bulk_wait_all();
  }
}

}  // namespace gfft
