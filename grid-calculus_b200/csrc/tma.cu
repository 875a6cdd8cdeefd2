// Host side of the TMA helpers: tensor-map encoding through the driver
// entry point (no link-time dependency on libcuda).
#include <mutex>

#include "tma.cuh"

namespace gcb {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}
}  // namespace

bool make_tensor_map_2d(CUtensorMap* map, const void* base, int nx, int ny, int elem_bytes, int box_x,
                        int box_y) {
  auto fn = encode_fn();
  if (!fn) return false;
  if (reinterpret_cast<uintptr_t>(base) % 16 != 0) return false;
  if ((static_cast<size_t>(nx) * elem_bytes) % 16 != 0) return false;
  if ((static_cast<size_t>(box_x) * elem_bytes) % 16 != 0) return false;
  if (box_x > 256 || box_y > 256 || box_x > nx || box_y > ny) return false;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(nx), static_cast<cuuint64_t>(ny)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(nx) * elem_bytes};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(box_x), static_cast<cuuint32_t>(box_y)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                  const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace gcb
