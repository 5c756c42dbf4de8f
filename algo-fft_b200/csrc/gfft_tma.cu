// Host-side tensor-map encoding for the TMA tile copies.  The driver entry
// point is looked up once through the runtime, so the library keeps linking
// only the CUDA runtime.
#include <cudaTypedefs.h>
#include <mutex>
#include "gfft_tma.cuh"

namespace gfft {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

}  // namespace

cudaError_t encode_tile_map(CUtensorMap* map, const void* base, int elem_bytes, int rank, const int64_t* dims,
                            const int64_t* strides_elems, const int* box, bool swizzle128) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  if (rank < 1 || rank > 5 || (elem_bytes != 8 && elem_bytes != 16)) return cudaErrorInvalidValue;
  if (reinterpret_cast<uintptr_t>(base) & 15) return cudaErrorInvalidValue;
  const int words = elem_bytes / 4;
  cuuint64_t gdim[5], gstride[4];
  cuuint32_t bdim[5], estr[5];
  gdim[0] = cuuint64_t(dims[0]) * words;
  bdim[0] = cuuint32_t(box[0]) * words;
  estr[0] = 1;
  if (dims[0] < 1 || box[0] < 1 || bdim[0] > 256 || (bdim[0] * 4) % 16 != 0) return cudaErrorInvalidValue;
  if (swizzle128 && bdim[0] * 4 != 128) return cudaErrorInvalidValue;
  for (int i = 1; i < rank; ++i) {
    if (dims[i] < 1 || dims[i] > (int64_t(1) << 32) || box[i] < 1 || box[i] > 256 || strides_elems[i] < 1)
      return cudaErrorInvalidValue;
    const int64_t sb = strides_elems[i] * elem_bytes;
    if (sb % 16 != 0 || sb >= (int64_t(1) << 40)) return cudaErrorInvalidValue;
    gdim[i] = cuuint64_t(dims[i]);
    gstride[i - 1] = cuuint64_t(sb);
    bdim[i] = cuuint32_t(box[i]);
    estr[i] = 1;
  }
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, cuuint32_t(rank), const_cast<void*>(base), gdim,
                        gstride, bdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace gfft
