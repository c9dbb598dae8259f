// Host side of the fused tile-stage kernel: TMA descriptors of the engine's
// block pools and the launch (the kernel instantiations are in
// tile_step_<scheme>.cu).
#include <cudaTypedefs.h>

#include <mutex>

#include "kernels.cuh"
#include "tile_api.cuh"

namespace alp {

extern template cudaError_t tile_kernel_info<FV_CHAR>(int, int, TileKernelInfo *);
extern template cudaError_t tile_kernel_info<FV_PRIM>(int, int, TileKernelInfo *);
extern template cudaError_t tile_kernel_info<FS_ROE>(int, int, TileKernelInfo *);

cudaError_t tile_info(int scheme, int variant, int precision, TileKernelInfo *out) {
  if (variant < 0 || variant >= kTileVariants) return cudaErrorInvalidValue;
  switch (scheme) {
    case FV_CHAR: return tile_kernel_info<FV_CHAR>(variant, precision, out);
    case FV_PRIM: return tile_kernel_info<FV_PRIM>(variant, precision, out);
    case FS_ROE: return tile_kernel_info<FS_ROE>(variant, precision, out);
  }
  return cudaErrorInvalidValue;
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// A pool [block][field][24][24][24] of doubles as a 5D tensor (z fastest) with
// boxes of bk (z) x bj (y) x 1 (x) x 5 fields x 1 block.
bool encode_pool(CUtensorMap *m, double *pool, int capacity, unsigned bk, unsigned bj,
                 std::string &why) {
  auto fn = encode_fn();
  if (!fn) {
    why = "cuTensorMapEncodeTiled is not available";
    return false;
  }
  cuuint64_t const dims[5] = {TC, TC, TC, 5, (cuuint64_t)capacity};
  cuuint64_t const strides[4] = {TC * 8, TC * TC * 8, TC * TC * TC * 8, 5ull * TC * TC * TC * 8};
  cuuint32_t const box[5] = {bk, bj, 1, 5, 1};
  cuuint32_t const es[5] = {1, 1, 1, 1, 1};
  CUresult const r =
      fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, pool, dims, strides, box, es,
         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    why = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
    return false;
  }
  return true;
}
}  // namespace

bool tile_encode(TileArgs &a, double *const pools[3], int capacity, std::string &why) {
  for (int p = 0; p < 3; ++p) {
    a.pool[p] = pools[p];
    if (!encode_pool(&a.plane[p], pools[p], capacity, IC, IC, why) ||
        !encode_pool(&a.yhalo[p], pools[p], capacity, IC, 3, why) ||
        !encode_pool(&a.zhalo[p], pools[p], capacity, 4, IC, why))
      return false;
  }
  return true;
}

cudaError_t tile_launch(TileArgs const &a, TileKernelInfo const &k, int grid, cudaStream_t st) {
  void *args[] = {const_cast<TileArgs *>(&a)};
  return cudaLaunchKernel(k.fn, dim3(grid), dim3(k.threads), args, k.smem, st);
}

}  // namespace alp
