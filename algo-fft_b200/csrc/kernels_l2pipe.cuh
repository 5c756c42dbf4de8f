// Launch and registration of the L2-pipelined two-pass kernels (k_l2p):
// tensor maps per call (they hold the buffers' addresses), a persistent grid
// of SMs x resident CTAs.  cudaErrorNotSupported when the copy engine cannot
// address the buffers (a pointer or a batch distance off a 16-byte
// boundary); the caller then runs the split two-pass kernels.
#pragma once
#include <mutex>
#include <utility>
#include <vector>
#include "gfft_l2pipe.cuh"
#include "gfft_registry.h"

namespace gfft {

template <typename C, int N1, int N2, int NC1, int NC2, int EPT1, int EPT2, int NST, int DIR>
cudaError_t l2p_launch(const L2pParams& p0, cudaStream_t st) {
  using K = L2p<C, N1, N2, NC1, NC2, EPT1, EPT2, NST>;
  constexpr int ES = K::ES;
  const void* fn = reinterpret_cast<const void*>(&k_l2p<C, N1, N2, NC1, NC2, EPT1, EPT2, NST, DIR>);
  L2pParams p = p0;
  CUtensorMap tx, tys, tyl, tz;
  const int64_t slots = int64_t(p.S) * p.G;
  const int64_t xd[3] = {N2, N1, p.count}, xs[3] = {1, N2, p.idist};
  const int xb[3] = {NC1, K::BR1, 1};
  const int64_t yd[3] = {N1, N2, slots}, ys[3] = {1, N1, K::N};
  const int ysb[3] = {K::RE, NC1, 1}, ylb[3] = {NC2, K::BR2, 1};
  const int64_t zd[3] = {N1, N2, p.count}, zs[3] = {1, N1, p.odist};
  const int zb[3] = {NC2, K::BR2, 1};
  if (encode_tile_map(&tx, p.src, ES, 3, xd, xs, xb) != cudaSuccess ||
      encode_tile_map(&tys, p.scratch, ES, 3, yd, ys, ysb, true) != cudaSuccess ||
      encode_tile_map(&tyl, p.scratch, ES, 3, yd, ys, ylb) != cudaSuccess ||
      encode_tile_map(&tz, p.dst, ES, 3, zd, zs, zb) != cudaSuccess)
    return cudaErrorNotSupported;
  static std::mutex mu;
  static std::vector<std::pair<int, int>> occ_of;  // (device, resident CTAs per SM)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int occ = 0;
  {
    std::lock_guard<std::mutex> g(mu);
    for (const auto& kv : occ_of)
      if (kv.first == dev) occ = kv.second;
    if (occ == 0) {
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, K::SMEM);
      if (e != cudaSuccess) return e;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, K::TPB, K::SMEM);
      if (e != cudaSuccess) return e;
      occ = occ < 1 ? 1 : occ;
      occ_of.emplace_back(dev, occ);
    }
  }
  int sms = 148;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int64_t total = int64_t(p.groups) * p.G * (K::TA + K::TB);
  const int64_t grid = total < int64_t(sms) * occ ? total : int64_t(sms) * occ;
  void* args[] = {&tx, &tys, &tyl, &tz, &p};
  return cudaLaunchKernel(fn, dim3(unsigned(grid)), dim3(unsigned(K::TPB)), args, size_t(K::SMEM), st);
}

template <typename C, int N1, int N2, int NC1, int NC2, int EPT1, int EPT2, int NST>
void reg_l2p() {
  using K = L2p<C, N1, N2, NC1, NC2, EPT1, EPT2, NST>;
  for (int dir : {-1, 1}) {
    L2PipeKernel k;
    k.prec = sizeof(C) == 8 ? kC64 : kC128;
    k.n1 = N1;
    k.n2 = N2;
    k.nc1 = NC1;
    k.nc2 = NC2;
    k.ept1 = EPT1;
    k.ept2 = EPT2;
    k.nst = NST;
    k.dir = dir;
    k.tpb = K::TPB;
    k.smem = K::SMEM;
    k.func = dir < 0 ? reinterpret_cast<const void*>(&k_l2p<C, N1, N2, NC1, NC2, EPT1, EPT2, NST, -1>)
                     : reinterpret_cast<const void*>(&k_l2p<C, N1, N2, NC1, NC2, EPT1, EPT2, NST, 1>);
    k.launch = dir < 0 ? &l2p_launch<C, N1, N2, NC1, NC2, EPT1, EPT2, NST, -1>
                       : &l2p_launch<C, N1, N2, NC1, NC2, EPT1, EPT2, NST, 1>;
    register_l2pipe(k);
  }
}

// Tile rule of the registered shapes: TE elements per tile (NC = TE / L
// columns), EPT elements per thread.
template <typename C, int N1, int N2, int TE, int EPT, int NST>
void reg_l2p_te() {
  reg_l2p<C, N1, N2, TE / N1, TE / N2, EPT, EPT, NST>();
}

}  // namespace gfft
