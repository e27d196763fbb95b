// smvs_tma.cu — TMA descriptors of the reference image (host side).
//
// The checkerboard kernels stage their block's reference tile in shared memory
// with one cp.async.bulk.tensor load (smvs_sweep.cuh). The descriptor is built
// here with the driver's cuTensorMapEncodeTiled, reached through
// cudaGetDriverEntryPoint so that the library links against the runtime only.
#include <cstdint>
#include <mutex>

#include <cudaTypedefs.h>

#include "smvs_kernels.h"

namespace smvs {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 Encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    (void)cudaGetLastError();
  });
  return fn;
}

}  // namespace

bool EncodeRefMap(CUtensorMap* map, const float* ref, int W, int H, int bx, int tpp, int R) {
  if (!map || !ref || !ValidSweepShape(bx, tpp)) return false;
  const int box_w = RefTileW(bx, R), box_h = RefTileH(bx, tpp, R);
  // Row pitch and base must be multiples of 16 bytes; the box must fit the
  // descriptor's limits (<= 256 per dimension, inner extent a multiple of 16
  // bytes) and the image.
  if (W % 4 != 0 || (reinterpret_cast<uintptr_t>(ref) & 15) != 0) return false;
  if (box_w > 256 || box_h > 256 || box_w % 4 != 0 || W < box_w || H < box_h) return false;
  PFN_cuTensorMapEncodeTiled_v12000 fn = Encoder();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
  const cuuint64_t strides[1] = {(cuuint64_t)W * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(ref), dims, strides, box, elem,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);  // out-of-bounds elements read as zero
  return r == CUDA_SUCCESS;
}

}  // namespace smvs
