// Device arrays that grow and shrink in place (CUDA virtual memory
// management): the virtual range is reserved once for the largest size, and
// physical memory is mapped into it in fixed chunks as the array grows and
// unmapped from its end as it shrinks. Pointers into the array stay valid, so
// kernels, CUDA graphs and tensor maps built on it need no update. The serving
// loop sizes its 2D and 3D engines this way from one shared HBM budget.
//
// The driver entry points are taken through the runtime
// (cudaGetDriverEntryPoint), so the library needs no link against libcuda.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>
#include <string>

#include "engine.hpp"

namespace alp {
namespace {

struct Vmm {
  PFN_cuMemGetAllocationGranularity_v10020 granularity = nullptr;
  PFN_cuMemAddressReserve_v10020 reserve = nullptr;
  PFN_cuMemAddressFree_v10020 address_free = nullptr;
  PFN_cuMemCreate_v10020 create = nullptr;
  PFN_cuMemRelease_v10020 release = nullptr;
  PFN_cuMemMap_v10020 map = nullptr;
  PFN_cuMemUnmap_v10020 unmap = nullptr;
  PFN_cuMemSetAccess_v10020 set_access = nullptr;
  bool ok = false;
};

Vmm const &vmm() {
  static std::once_flag once;
  static Vmm v;
  std::call_once(once, [] {
    auto get = [](char const *name, void **p) {
      cudaDriverEntryPointQueryResult q;
      return cudaGetDriverEntryPoint(name, p, cudaEnableDefault, &q) == cudaSuccess &&
             q == cudaDriverEntryPointSuccess && *p != nullptr;
    };
    v.ok = get("cuMemGetAllocationGranularity", (void **)&v.granularity) &&
           get("cuMemAddressReserve", (void **)&v.reserve) &&
           get("cuMemAddressFree", (void **)&v.address_free) &&
           get("cuMemCreate", (void **)&v.create) && get("cuMemRelease", (void **)&v.release) &&
           get("cuMemMap", (void **)&v.map) && get("cuMemUnmap", (void **)&v.unmap) &&
           get("cuMemSetAccess", (void **)&v.set_access);
    cudaGetLastError();
  });
  return v;
}

CUmemAllocationProp device_prop(int dev) {
  CUmemAllocationProp p{};
  p.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  p.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  p.location.id = dev;
  return p;
}

int drv_fail(CUresult r, char const *what) {
  return fail(ALP_ERR_CUDA, std::string(what) + " failed (CUresult " + std::to_string((int)r) + ")");
}

size_t round_up(size_t x, size_t q) { return (x + q - 1) / q * q; }

}  // namespace

size_t elastic_chunk_bytes() { return size_t(32) << 20; }

int elastic_reserve(ElasticArray &a, size_t bytes) {
  Vmm const &v = vmm();
  if (!v.ok) return fail(ALP_ERR_CUDA, "CUDA virtual memory management is not available");
  int dev = 0;
  ALP_CUDA(cudaGetDevice(&dev));
  CUmemAllocationProp const prop = device_prop(dev);
  size_t gran = 0;
  if (CUresult r = v.granularity(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_MINIMUM))
    return drv_fail(r, "cuMemGetAllocationGranularity");
  if (elastic_chunk_bytes() % gran != 0)
    return fail(ALP_ERR_CUDA, "allocation granularity does not divide the chunk size");
  a.device = dev;
  a.reserved = round_up(bytes > 0 ? bytes : 1, elastic_chunk_bytes());
  CUdeviceptr p = 0;
  if (CUresult r = v.reserve(&p, a.reserved, 0, 0, 0)) {
    a.reserved = 0;
    return drv_fail(r, "cuMemAddressReserve");
  }
  a.base = (unsigned long long)p;
  a.mapped = 0;
  a.chunks.clear();
  return ALP_OK;
}

int elastic_resize(ElasticArray &a, size_t bytes) {
  Vmm const &v = vmm();
  size_t const want = round_up(bytes, elastic_chunk_bytes());
  if (want > a.reserved) return fail(ALP_ERR_CAPACITY, "elastic array beyond its reservation");
  size_t const chunk = elastic_chunk_bytes();
  CUmemAllocationProp const prop = device_prop(a.device);
  CUmemAccessDesc access{};
  access.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  access.location.id = a.device;
  access.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
  while (a.mapped < want) {
    CUmemGenericAllocationHandle h = 0;
    if (CUresult r = v.create(&h, chunk, &prop, 0)) {
      // out of device memory: the array keeps what it has
      return r == CUDA_ERROR_OUT_OF_MEMORY
                 ? fail(ALP_ERR_CAPACITY, "device memory exhausted while growing an engine")
                 : drv_fail(r, "cuMemCreate");
    }
    CUdeviceptr const at = (CUdeviceptr)(a.base + a.mapped);
    CUresult r = v.map(at, chunk, 0, h, 0);
    if (r == CUDA_SUCCESS) {
      r = v.set_access(at, chunk, &access, 1);
      if (r != CUDA_SUCCESS) v.unmap(at, chunk);
    }
    if (r != CUDA_SUCCESS) {
      v.release(h);
      return drv_fail(r, "cuMemMap / cuMemSetAccess");
    }
    a.chunks.push_back((unsigned long long)h);
    a.mapped += chunk;
  }
  while (a.mapped > want) {
    CUdeviceptr const at = (CUdeviceptr)(a.base + a.mapped - chunk);
    if (CUresult r = v.unmap(at, chunk)) return drv_fail(r, "cuMemUnmap");
    if (CUresult r = v.release((CUmemGenericAllocationHandle)a.chunks.back()))
      return drv_fail(r, "cuMemRelease");
    a.chunks.pop_back();
    a.mapped -= chunk;
  }
  return ALP_OK;
}

void elastic_release(ElasticArray &a) {
  if (!a.reserved) return;
  Vmm const &v = vmm();
  elastic_resize(a, 0);
  v.address_free((CUdeviceptr)a.base, a.reserved);
  a = ElasticArray{};
}

}  // namespace alp
