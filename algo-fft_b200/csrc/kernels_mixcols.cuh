// Launchers and table entries of the compiled mixed-radix column tiles
// (gfft_mixcols.cuh) and of the Bluestein chain on them (gfft_mixbs.cuh).
// The generated kernels_mixcols_t*.cu / kernels_mixbs_t*.cu files each
// instantiate a share of the tables (gen_mixcols.py picks the schedules);
// kernels_mixcols.cu gathers them.
#pragma once
#include "gfft_internal.h"
#include "gfft_mixbs.cuh"
#include "gfft_mixcols.cuh"

namespace gfft {

using MixFn = cudaError_t (*)(const MixColsParams&, int64_t, cudaStream_t);

struct MixEntry {
  int L;
  int nc[2];          // tile width of pass 1 per precision (pass 2 takes the same)
  int nc2[2];         // tile width of pass 2 per precision
  MixFn fn[2][2][2];  // [prec][dir < 0 ? 0 : 1][pass - 1]
};

// One pass: schedule SC, NC columns per tile, MINB resident CTAs per SM,
// TT threads per column (0: L / max radix).
template <typename SC, int NC, int MINB, int TT = 0>
struct MixCfg {
  using Sched = SC;
  static constexpr int nc = NC, minb = MINB, tt = TT;
};

template <typename C, typename CFG, int DIR, int PASS>
cudaError_t launch_mix(const MixColsParams& p, int64_t count, cudaStream_t st) {
  using SC = typename CFG::Sched;
  constexpr int NC = CFG::nc;
  using TL = MixTile<SC, NC, CFG::tt>;
  constexpr int smem = (PASS == MIX_PASS1 ? TL::ELEMS1 : TL::ELEMS2) * int(sizeof(C));
  auto kern = &k_mix_cols<C, SC, NC, DIR, PASS, CFG::minb, CFG::tt>;
  static const cudaError_t attr =
      smem > 48 * 1024 ? cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) : cudaSuccess;
  if (attr != cudaSuccess) return attr;
  const int64_t blocks = p.tiles * count;
  if (blocks <= 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  kern<<<unsigned(blocks), TL::TPB, smem, st>>>(p);
  return cudaGetLastError();
}

// Table entry of length L from the four pass configurations
// (complex64 pass 1 / pass 2, complex128 pass 1 / pass 2).
template <typename F1, typename F2, typename D1, typename D2>
MixEntry mix_entry() {
  static_assert(F1::Sched::L == F2::Sched::L && F1::Sched::L == D1::Sched::L && F1::Sched::L == D2::Sched::L,
                "one length per entry");
  MixEntry e{};
  e.L = F1::Sched::L;
  e.nc[kC64] = F1::nc;
  e.nc2[kC64] = F2::nc;
  e.nc[kC128] = D1::nc;
  e.nc2[kC128] = D2::nc;
  e.fn[kC64][0][0] = &launch_mix<float2, F1, -1, MIX_PASS1>;
  e.fn[kC64][0][1] = &launch_mix<float2, F2, -1, MIX_PASS2>;
  e.fn[kC64][1][0] = &launch_mix<float2, F1, +1, MIX_PASS1>;
  e.fn[kC64][1][1] = &launch_mix<float2, F2, +1, MIX_PASS2>;
  e.fn[kC128][0][0] = &launch_mix<double2, D1, -1, MIX_PASS1>;
  e.fn[kC128][0][1] = &launch_mix<double2, D2, -1, MIX_PASS2>;
  e.fn[kC128][1][0] = &launch_mix<double2, D1, +1, MIX_PASS1>;
  e.fn[kC128][1][1] = &launch_mix<double2, D2, +1, MIX_PASS2>;
  return e;
}


using MixBsFn = cudaError_t (*)(const MixBsParams&, int64_t, cudaStream_t);

struct MixBsEntry {
  int L;
  int nc[2];           // tile width per precision
  MixBsFn fn[2][3];    // [prec][BSK_IN / BSK_MID / BSK_OUT]
};

template <typename C, typename CFG, int KIND>
cudaError_t launch_mix_bs(const MixBsParams& p, int64_t blocks, cudaStream_t st) {
  using SC = typename CFG::Sched;
  constexpr int NC = CFG::nc;
  using TL = MixTile<SC, NC, CFG::tt>;
  constexpr int smem = (KIND == BSK_OUT ? TL::ELEMS2 : TL::ELEMS1) * int(sizeof(C));
  auto kern = &k_mix_bs<C, SC, NC, KIND, CFG::minb, CFG::tt>;
  static const cudaError_t attr =
      smem > 48 * 1024 ? cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) : cudaSuccess;
  if (attr != cudaSuccess) return attr;
  if (blocks <= 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  kern<<<unsigned(blocks), TL::TPB, smem, st>>>(p);
  return cudaGetLastError();
}

// Bluestein-chain entry of length L from its complex64 and complex128
// configurations (the column tiles' own).
template <typename F, typename D>
MixBsEntry mix_bs_entry() {
  static_assert(F::Sched::L == D::Sched::L, "one length per entry");
  MixBsEntry e{};
  e.L = F::Sched::L;
  e.nc[kC64] = F::nc;
  e.nc[kC128] = D::nc;
  e.fn[kC64][BSK_IN] = &launch_mix_bs<float2, F, BSK_IN>;
  e.fn[kC64][BSK_MID] = &launch_mix_bs<float2, F, BSK_MID>;
  e.fn[kC64][BSK_OUT] = &launch_mix_bs<float2, F, BSK_OUT>;
  e.fn[kC128][BSK_IN] = &launch_mix_bs<double2, D, BSK_IN>;
  e.fn[kC128][BSK_MID] = &launch_mix_bs<double2, D, BSK_MID>;
  e.fn[kC128][BSK_OUT] = &launch_mix_bs<double2, D, BSK_OUT>;
  return e;
}

using MixRowsFn = cudaError_t (*)(const MixRowsParams&, cudaStream_t);

struct MixRowsEntry {
  int L;
  int nc[2];           // transforms per CTA per precision
  MixRowsFn fn[2][2];  // [prec][dir < 0 ? 0 : 1]; null where a precision has no schedule
};

template <typename C, typename CFG, int DIR>
cudaError_t launch_mix_rows(const MixRowsParams& p, cudaStream_t st) {
  using SC = typename CFG::Sched;
  constexpr int NC = CFG::nc;
  using TL = MixTileRows<SC, NC, CFG::tt>;
  constexpr int smem = TL::ELEMS * int(sizeof(C));
  auto kern = &k_mix_rows<C, SC, NC, DIR, CFG::minb, CFG::tt>;
  static const cudaError_t attr =
      smem > 48 * 1024 ? cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) : cudaSuccess;
  if (attr != cudaSuccess) return attr;
  const int64_t blocks = (p.count + NC - 1) / NC;
  if (blocks <= 0) return cudaSuccess;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  kern<<<unsigned(blocks), TL::TPB, smem, st>>>(p);
  return cudaGetLastError();
}

// Complex64 only (lengths beyond a complex128 transform's shared memory).
template <typename F>
MixRowsEntry mix_rows_entry64() {
  MixRowsEntry e{};
  e.L = F::Sched::L;
  e.nc[kC64] = F::nc;
  e.fn[kC64][0] = &launch_mix_rows<float2, F, -1>;
  e.fn[kC64][1] = &launch_mix_rows<float2, F, +1>;
  return e;
}

template <typename F, typename D>
MixRowsEntry mix_rows_entry() {
  static_assert(F::Sched::L == D::Sched::L, "one length per entry");
  MixRowsEntry e{};
  e.L = F::Sched::L;
  e.nc[kC64] = F::nc;
  e.nc[kC128] = D::nc;
  e.fn[kC64][0] = &launch_mix_rows<float2, F, -1>;
  e.fn[kC64][1] = &launch_mix_rows<float2, F, +1>;
  e.fn[kC128][0] = &launch_mix_rows<double2, D, -1>;
  e.fn[kC128][1] = &launch_mix_rows<double2, D, +1>;
  return e;
}

}  // namespace gfft
