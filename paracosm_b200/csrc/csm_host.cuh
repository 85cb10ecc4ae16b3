// Host-side helpers shared by the engine's translation units: error text and
// device allocations tracked against the context's HBM budget.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/csm_gpu.h"

namespace csm {

int set_err(int code, const char* fmt, ...);

struct DevMem {
  std::vector<void*> ptrs;
  uint64_t bytes = 0, budget = 0;
  int alloc(void** p, size_t sz) {
    sz = std::max<size_t>(sz, 16);
    if (budget && bytes + sz > budget)
      return set_err(CSM_ENOMEM, "HBM budget of %llu bytes exceeded", (unsigned long long)budget);
    cudaError_t e = cudaMalloc(p, sz);
    if (e != cudaSuccess) return set_err(CSM_ENOMEM, "cudaMalloc(%zu): %s", sz, cudaGetErrorString(e));
    ptrs.push_back(*p);
    bytes += sz;
    return CSM_OK;
  }
  void release(void* p, size_t sz) {
    if (!p) return;
    for (size_t i = 0; i < ptrs.size(); i++)
      if (ptrs[i] == p) { ptrs.erase(ptrs.begin() + (long)i); break; }
    cudaFree(p);
    bytes -= std::min<uint64_t>(bytes, std::max<size_t>(sz, 16));
  }
  void free_all() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
    bytes = 0;
  }
};

}  // namespace csm
