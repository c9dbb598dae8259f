// Host interface of the fused tile-stage kernel (tile_step.cuh, tile_step.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>

#include "layout.cuh"

namespace alp {

// Kernel arguments (passed as one __grid_constant__ parameter).
struct TileArgs {
  CUtensorMap plane[3];  // pools A, B, C; box (k 16, j 16, i 1, field 5, block 1)
  CUtensorMap yhalo[3];  // box (16, 3, 1, 5, 1)
  CUtensorMap zhalo[3];  // box (4, 16, 1, 5, 1)
  double *pool[3];
  int const *order;      // [nstages][nwork] block slots per stage
  int nwork, nsteps, nstages, stage0, trial;
  BlockMeta const *meta;
  int const *nbr26;
  CaseState *cases;
  int *ctrl;             // [0] next item; [1] error bits: 1 dependency, 2 load, 4 dt,
                         // 8 task-order wait ran out (not reset by the launches)
  int *done;             // [slots] last finished (step, stage) + 1 of each block
  int *dtflag;           // [cases] 1 + the step whose dt is ready
  int *cnt;              // [cases] blocks of the case that finished a last stage
  int const *case_nb;    // [cases] blocks of each case in the work list
};

// Launch shape of one instantiation.
struct TileKernelInfo {
  void const *fn;
  int threads;
  size_t smem;
  int ctas_per_sm;
};

// Variants of the kernel (warps per CTA; one CTA per SM).
constexpr int kTileVariants = 2;
constexpr int kTileWarps[kTileVariants] = {16, 12};

template <int SCHEME>
cudaError_t tile_kernel_info(int variant, int precision, TileKernelInfo *out);

// Shared-memory limit and launch shape of the kernel for a scheme id, variant
// and precision.
cudaError_t tile_info(int scheme, int variant, int precision, TileKernelInfo *out);
// TMA descriptors of the three block pools (reference layout, `capacity`
// blocks each) into a; false with a reason when the driver cannot encode them.
bool tile_encode(TileArgs &a, double *const pools[3], int capacity, std::string &why);
// One launch of the kernel with `grid` CTAs.
cudaError_t tile_launch(TileArgs const &a, TileKernelInfo const &k, int grid, cudaStream_t st);

}  // namespace alp
