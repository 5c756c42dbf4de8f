// Kernel registry: every compiled kernel variant with its launch shape, so
// plans and the autotuner can pick among them at run time.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

namespace gfft {

enum Prec { kC64 = 0, kC128 = 1 };


// Single-pass power-of-two kernel (k_pow2) of one (precision, N, EPT, dir).
struct Pow2Kernel {
  int prec, n, ept, dir;
  int tpb;        // threads per CTA
  int per_cta;    // transforms per CTA
  int smem;       // dynamic shared memory bytes per CTA
  const void* func;
  cudaError_t (*launch)(const void* src, void* dst, int64_t count, int64_t idist, int64_t odist,
                        const void* tw, double scale, cudaStream_t st);
};

// Persistent two-pass kernel (k_twopass) of one (precision, N1 x N2, dir).
struct TwoPassParams;
struct TwoPassKernel {
  int prec, n1, n2, dir;
  int tpb, smem;
  int nc1, nc2;   // columns per tile in pass 1 / pass 2
  int te = 0, emax = 0;  // variant: tile elements, max elements per thread
  const void* func;
  cudaError_t (*launch)(const TwoPassParams& p, int grid, cudaStream_t st);
  const void* split_func[2];  // k_tp_split pass 1, pass 2
  cudaError_t (*split)(const TwoPassParams& p, int pass, int64_t b0, int64_t nb, cudaStream_t st);
};

// Three-pass kernels (k_tp3) of one (precision, N1 x M1 x M2, dir).
struct ThreePassParams;
struct ThreePassKernel {
  int prec, n1, m1, m2, dir;
  int tpb, smem;
  int tma = 0, te = 0, emax = 0, nst = 0;  // TMA-staged variant: tile elements, elements per thread, stages
  const void* func[3];  // passes 1..3
  cudaError_t (*launch)(const ThreePassParams& p, int pass, int64_t b0, int64_t nb, cudaStream_t st);
};

// L2-pipelined two-pass kernel (k_l2p) of one (precision, N1 x N2, tile
// shape, stages, dir).
struct L2pParams;
struct L2PipeKernel {
  int prec, n1, n2, nc1, nc2, ept1, ept2, nst, dir;
  int tpb, smem;
  const void* func;
  cudaError_t (*launch)(const L2pParams& p, cudaStream_t st);
};

void register_l2pipe(const L2PipeKernel& k);
// The variant of this shape and direction; nc1 = 0 takes the first registered.
const L2PipeKernel* find_l2pipe(int prec, int64_t n, int dir, int n1 = 0, int nc1 = 0, int nc2 = 0, int nst = 0);
std::vector<const L2PipeKernel*> l2pipe_variants(int prec, int64_t n, int dir);

void register_pow2(const Pow2Kernel& k);
void register_threepass(const ThreePassKernel& k);
// The plain kernels (tma = 0) unless a TMA-staged variant is named.
const ThreePassKernel* find_threepass(int prec, int64_t n, int dir, int tma = 0, int te = 0, int emax = 0,
                                      int nst = 0);
std::vector<const ThreePassKernel*> threepass_variants(int prec, int64_t n, int dir);
void register_twopass(const TwoPassKernel& k);
const TwoPassKernel* find_twopass(int prec, int64_t n, int dir, int te = 0, int emax = 0);
std::vector<const TwoPassKernel*> twopass_variants(int prec, int64_t n, int dir);
const Pow2Kernel* find_pow2(int prec, int n, int ept, int dir);
std::vector<const Pow2Kernel*> pow2_variants(int prec, int n, int dir);

// Ensures every registered kernel has its shared-memory limit raised (once
// per device).
cudaError_t prepare_kernels();

}  // namespace gfft
