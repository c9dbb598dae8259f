// alp_space_rhs_static: the right-hand side of alp_space_rhs with its face-flux
// scratch in a fixed device array of this library instead of caller memory.
//
// Who needs it: a caller that may not allocate device memory at the point where
// it evaluates the right-hand side. Examples are a per-block solver object whose
// methods are const and own no device buffer (as ALPACA's convective term
// solvers are), code that must not run cudaFree because it synchronises the
// whole device, and a process whose free HBM is held by another allocator (a
// caching allocator such as torch's) so that a fresh cudaMalloc can fail. Such a
// caller gets the same kernels as alp_space_rhs with no allocation at all.
//
// The scratch array is allocated by the CUDA driver when it loads this file's
// module; this file launches no kernels of its own (the face-flux and divergence
// kernels are the ones alp_space_rhs uses), so the array lives in a module of
// its own and costs nothing until the first call asks for its address.
#include <cuda_runtime.h>

#include <string>

#include "../../include/alpaca_b200.h"

namespace alp {
int fail(int code, std::string const &msg);
int cuda_fail(cudaError_t e, char const *where);
int scheme_id(alp_scheme const *s, int *id, int *precision);
int check_material(alp_material const *m);
}  // namespace alp

namespace {

// 16 MiB: [nb][dim][NE][faces] doubles hold 28 blocks in 3D (589,560 B each),
// 453 in 2D (36,992 B each) and 10,280 in 1D (1,632 B each).
constexpr size_t kStaticScratchBytes = size_t(16) << 20;
static __device__ __align__(256) double g_space_rhs_scratch[kStaticScratchBytes / sizeof(double)];

// Address of the array in the current device's context. It is looked up on
// every call (a symbol lookup in the loaded module, no allocation once the
// module is loaded): after cudaDeviceReset the next context loads the module
// again, possibly at another address, so an address kept from an earlier call
// could be stale.
int scratch_of_current_device(void **out) {
  void *p = nullptr;
  cudaError_t const e = cudaGetSymbolAddress(&p, g_space_rhs_scratch);
  if (e != cudaSuccess) return alp::cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
  *out = p;
  return ALP_OK;
}

}  // namespace

extern "C" {

int alp_space_rhs_static(int dim, const alp_scheme *scheme, const alp_material *mat,
                         const double *d_blocks, int nb, double cell_size, double *d_rhs,
                         alp_stream_t stream) {
  // the argument checks of alp_space_rhs come first, in its order, so a bad
  // call returns the same code from both entry points
  if (dim < 1 || dim > 3) return alp::fail(ALP_ERR_INVALID, "dim must be 1, 2 or 3");
  int sid, prec;
  if (int rc = alp::scheme_id(scheme, &sid, &prec)) return rc;
  if (int rc = alp::check_material(mat)) return rc;
  size_t const need = alp_space_rhs_workspace_size(dim, nb);
  if (nb > 0 && need > kStaticScratchBytes) {
    size_t const per_block = alp_space_rhs_workspace_size(dim, 1);
    return alp::fail(ALP_ERR_CAPACITY,
                     "alp_space_rhs_static: " + std::to_string(nb) + " blocks need " +
                         std::to_string(need) + " bytes of scratch; the static array holds " +
                         std::to_string(kStaticScratchBytes) + " bytes (at most " +
                         std::to_string(kStaticScratchBytes / per_block) + " blocks in " +
                         std::to_string(dim) + "D)");
  }
  if (nb <= 0)  // argument checks and the empty case exactly as alp_space_rhs
    return alp_space_rhs(dim, scheme, mat, d_blocks, nb, cell_size, d_rhs, nullptr, 0, stream);
  void *scratch = nullptr;
  if (int rc = scratch_of_current_device(&scratch)) return rc;
  // Every face the divergence reads is written first by the face-flux kernels
  // (zero for skipped faces), so the array's previous contents never matter
  // and nothing is cleared.
  return alp_space_rhs(dim, scheme, mat, d_blocks, nb, cell_size, d_rhs, scratch,
                       kStaticScratchBytes, stream);
}

}  // extern "C"
