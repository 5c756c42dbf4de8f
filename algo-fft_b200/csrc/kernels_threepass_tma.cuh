// Launch and registration of the TMA-staged three-pass kernels (k_tp3t).
#pragma once
#include <algorithm>
#include <type_traits>
#include "gfft_registry.h"
#include "gfft_threepass_tma.cuh"

namespace gfft {

template <typename C, int N1, int M1, int M2, int TE, int EMAX, int NST, int DIR>
struct Tp3tOf {
  template <int PASS>
  using K = Tp3t<C, N1, M1, M2, TE, EMAX, NST, PASS>;
  static constexpr int64_t M = int64_t(M1) * M2, N = int64_t(N1) * M;

  template <int PASS>
  static const void* fn() {
    return reinterpret_cast<const void*>(&k_tp3t<C, N1, M1, M2, TE, EMAX, NST, DIR, PASS>);
  }

  template <int PASS>
  static cudaError_t run(const CUtensorMap& tin, const CUtensorMap& tout, Tp3tArgs a, int64_t nb, cudaStream_t st) {
    a.tiles = nb * K<PASS>::TILES;
    if (a.tiles <= 0) return cudaSuccess;
    static const int occ = [] {
      cudaFuncSetAttribute(fn<PASS>(), cudaFuncAttributeMaxDynamicSharedMemorySize, K<PASS>::SMEM);
      int n = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, &k_tp3t<C, N1, M1, M2, TE, EMAX, NST, DIR, PASS>, K<PASS>::TPB,
                                                        K<PASS>::SMEM) != cudaSuccess)
        n = 1;
      return n > 0 ? n : 1;
    }();
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = std::min<int64_t>(a.tiles, int64_t(sms) * occ);
    k_tp3t<C, N1, M1, M2, TE, EMAX, NST, DIR, PASS><<<unsigned(grid), K<PASS>::TPB, K<PASS>::SMEM, st>>>(tin, tout, a);
    return cudaGetLastError();
  }

  // One pass over transforms [b0, b0 + nb).  Falls back to the plain kernel
  // of the same factors when the copy engine cannot address the buffers
  // (a pointer or a batch distance off a 16-byte boundary).
  static cudaError_t launch(const ThreePassParams& p, int pass, int64_t b0, int64_t nb, cudaStream_t st) {
    constexpr int ES = sizeof(C);
    CUtensorMap tin, tout;
    Tp3tArgs a{};
    a.status = p.status;
    a.spin_limit = p.spin_limit;
    cudaError_t e = cudaSuccess;
    if (pass == 1) {
      const int64_t dims[3] = {M, N1, nb}, str[3] = {1, M, p.idist};
      const int box[3] = {K<1>::NC, N1, 1};
      e = encode_tile_map(&tin, static_cast<const char*>(p.src) + b0 * p.idist * ES, ES, 3, dims, str, box);
      const int64_t ydims[3] = {N1, M, nb}, ystr[3] = {1, N1, N};
      const int ybox[3] = {K<1>::RE, K<1>::NC, 1};
      if (e == cudaSuccess) e = encode_tile_map(&tout, p.scratch, ES, 3, ydims, ystr, ybox, true);
      a.tw = p.tw1;
      a.bt = p.bt;
    } else if (pass == 2) {
      const int64_t dims[4] = {N1, M2, M1, nb}, str[4] = {1, N1, int64_t(M2) * N1, N};
      const int box[4] = {K<2>::NC, 1, M1, 1};
      e = encode_tile_map(&tin, p.scratch, ES, 4, dims, str, box);
      tout = tin;
      a.tw = p.tw2;
      a.bt = p.btm;
    } else {
      const int64_t dims[3] = {N1, M, nb}, str[3] = {1, N1, N};
      const int box[3] = {K<3>::NC, M2, 1};
      e = encode_tile_map(&tin, p.scratch, ES, 3, dims, str, box);
      const int64_t odims[4] = {N1, M1, M2, nb}, ostr[4] = {1, N1, int64_t(N1) * M1, p.odist};
      const int obox[4] = {K<3>::NC, 1, M2, 1};
      if (e == cudaSuccess)
        e = encode_tile_map(&tout, static_cast<char*>(p.dst) + b0 * p.odist * ES, ES, 4, odims, ostr, obox);
      a.tw = p.tw3;
      a.scale = p.scale;
    }
    if (e != cudaSuccess) {
      const ThreePassKernel* plain = find_threepass(ES == 8 ? kC64 : kC128, N, DIR);
      if (!plain) return cudaErrorInvalidValue;
      return plain->launch(p, pass, b0, nb, st);
    }
    if (pass == 1) return run<1>(tin, tout, a, nb, st);
    if (pass == 2) return run<2>(tin, tout, a, nb, st);
    return run<3>(tin, tout, a, nb, st);
  }
};

template <typename C, int N1, int M1, int M2, int TE, int EMAX, int NST>
void reg_tp3t() {
  auto one = [](auto tag) {
    using T = decltype(tag);
    ThreePassKernel k;
    k.prec = sizeof(C) == 8 ? kC64 : kC128;
    k.n1 = N1;
    k.m1 = M1;
    k.m2 = M2;
    k.dir = T::value;
    k.tma = 1;
    k.te = TE;
    k.nst = NST;
    k.emax = EMAX;
    using O = Tp3tOf<C, N1, M1, M2, TE, EMAX, NST, T::value>;
    k.tpb = std::max({O::template K<1>::TPB, O::template K<2>::TPB, O::template K<3>::TPB});
    k.smem = std::max({O::template K<1>::SMEM, O::template K<2>::SMEM, O::template K<3>::SMEM});
    k.func[0] = O::template fn<1>();
    k.func[1] = O::template fn<2>();
    k.func[2] = O::template fn<3>();
    k.launch = &O::launch;
    register_threepass(k);
  };
  one(std::integral_constant<int, -1>{});
  one(std::integral_constant<int, 1>{});
}

}  // namespace gfft
