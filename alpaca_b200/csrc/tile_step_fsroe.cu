// Instantiations of the fused tile-stage kernel for one scheme (tile_step.cuh);
// one file per scheme so that they compile in parallel.
#include "tile_step.cuh"

namespace alp {
template cudaError_t tile_kernel_info<FS_ROE>(int variant, int precision, TileKernelInfo *out);
}  // namespace alp
