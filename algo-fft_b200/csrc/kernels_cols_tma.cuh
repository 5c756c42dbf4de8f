// Launch and registration of the TMA-staged three-pass kernels (k_tp3t):
// tensor maps per call (they hold the buffers' addresses), a
// persistent grid of SMs x resident CTAs, and the plain kernels of the same
// factors when the copy engine cannot address the buffers (a pointer or a
// batch distance off a 16-byte boundary).
#pragma once
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>
#include "gfft_cols_tma.cuh"
#include "gfft_registry.h"

namespace gfft {

// Persistent launch of one TMA-staged pass kernel `fn` (parameters: two
// tensor maps, ColTArgs).  Raises the kernel's shared-memory limit and reads
// its occupancy once per (kernel, device).
inline cudaError_t colt_launch(const void* fn, int tpb, int smem, const CUtensorMap& tin, const CUtensorMap& tout,
                               ColTArgs a, cudaStream_t st) {
  if (a.tiles <= 0) return cudaSuccess;
  static std::mutex mu;
  static std::vector<std::pair<std::pair<const void*, int>, int>> occ_of;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int occ = 0;
  {
    std::lock_guard<std::mutex> g(mu);
    for (const auto& kv : occ_of)
      if (kv.first.first == fn && kv.first.second == dev) occ = kv.second;
    if (occ == 0) {
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, tpb, smem);
      if (e != cudaSuccess) return e;
      occ = std::max(occ, 1);
      occ_of.push_back({{fn, dev}, occ});
    }
  }
  int sms = 148;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int64_t grid = std::min<int64_t>(a.tiles, int64_t(sms) * occ);
  CUtensorMap tin_v = tin, tout_v = tout;
  void* args[] = {&tin_v, &tout_v, &a};
  return cudaLaunchKernel(fn, dim3(unsigned(grid)), dim3(unsigned(tpb)), args, size_t(smem), st);
}

// ---------------------------------------------------------------- three-pass

template <typename C, int N1, int M1, int M2, int TE, int EMAX, int NST, int DIR>
struct Tp3tOf {
  template <int PASS>
  using K = ColT<C, Tp3Pass<N1, M1, M2, PASS>::L, TE, EMAX, NST, Tp3Pass<N1, M1, M2, PASS>::KIND>;
  static constexpr int64_t M = int64_t(M1) * M2, N = int64_t(N1) * M;

  template <int PASS>
  static const void* fn() {
    return reinterpret_cast<const void*>(&k_tp3t<C, N1, M1, M2, TE, EMAX, NST, DIR, PASS>);
  }

  // One pass over transforms [b0, b0 + nb).
  static cudaError_t launch(const ThreePassParams& p, int pass, int64_t b0, int64_t nb, cudaStream_t st) {
    constexpr int ES = sizeof(C);
    CUtensorMap tin, tout;
    ColTArgs a{};
    a.status = p.status;
    a.spin_limit = p.spin_limit;
    cudaError_t e = cudaSuccess;
    if (pass == 1) {
      const int64_t dims[3] = {M, N1, nb}, str[3] = {1, M, p.idist};
      const int box[3] = {K<1>::NC, K<1>::BR, 1};
      e = encode_tile_map(&tin, static_cast<const char*>(p.src) + b0 * p.idist * ES, ES, 3, dims, str, box);
      const int64_t ydims[3] = {N1, M, nb}, ystr[3] = {1, N1, N};
      const int ybox[3] = {K<1>::RE, K<1>::NC, 1};
      if (e == cudaSuccess) e = encode_tile_map(&tout, p.scratch, ES, 3, ydims, ystr, ybox, true);
      a.tpt = M / K<1>::NC;
      a.tw = p.tw1;
      a.bt = p.bt;
    } else if (pass == 2) {
      const int64_t dims[4] = {N1, M2, M1, nb}, str[4] = {1, N1, int64_t(M2) * N1, N};
      const int box[4] = {K<2>::NC, 1, M1, 1};
      e = encode_tile_map(&tin, p.scratch, ES, 4, dims, str, box);
      tout = tin;
      a.groups = N1 / K<2>::NC;
      a.tpt = int64_t(M2) * a.groups;
      a.tw = p.tw2;
      a.bt = p.btm;
    } else {
      const int64_t dims[3] = {N1, M, nb}, str[3] = {1, N1, N};
      const int box[3] = {K<3>::NC, K<3>::BR, 1};
      e = encode_tile_map(&tin, p.scratch, ES, 3, dims, str, box);
      const int64_t odims[4] = {N1, M1, M2, nb}, ostr[4] = {1, N1, int64_t(N1) * M1, p.odist};
      const int obox[4] = {K<3>::NC, 1, K<3>::BR, 1};
      if (e == cudaSuccess)
        e = encode_tile_map(&tout, static_cast<char*>(p.dst) + b0 * p.odist * ES, ES, 4, odims, ostr, obox);
      a.groups = N1 / K<3>::NC;
      a.tpt = int64_t(M1) * a.groups;
      a.tw = p.tw3;
      a.scale = p.scale;
    }
    if (e != cudaSuccess) {
      const ThreePassKernel* plain = find_threepass(ES == 8 ? kC64 : kC128, N, DIR);
      if (!plain) return cudaErrorInvalidValue;
      return plain->launch(p, pass, b0, nb, st);
    }
    a.tiles = nb * a.tpt;
    if (pass == 1) return colt_launch(fn<1>(), K<1>::TPB, K<1>::SMEM, tin, tout, a, st);
    if (pass == 2) return colt_launch(fn<2>(), K<2>::TPB, K<2>::SMEM, tin, tout, a, st);
    return colt_launch(fn<3>(), K<3>::TPB, K<3>::SMEM, tin, tout, a, st);
  }
};

template <typename C, int N1, int M1, int M2, int TE, int EMAX, int NST>
void reg_tp3t() {
  auto one = [](auto tag) {
    using T = decltype(tag);
    using O = Tp3tOf<C, N1, M1, M2, TE, EMAX, NST, T::value>;
    ThreePassKernel k;
    k.prec = sizeof(C) == 8 ? kC64 : kC128;
    k.n1 = N1;
    k.m1 = M1;
    k.m2 = M2;
    k.dir = T::value;
    k.tma = 1;
    k.te = TE;
    k.emax = EMAX;
    k.nst = NST;
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
