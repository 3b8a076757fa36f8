// Device memory of the engine: every cudaMalloc / cudaFree of the matchers and batches goes
// through these two functions, which count the live allocations and can make an allocation fail
// on purpose (sgm_debug_fail_device_alloc), so that tests can check the out-of-memory paths of the
// initialisation calls -- SGM_ERR_NOMEM and nothing left allocated -- without exhausting a GPU.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

cudaError_t sgm_dev_malloc(void** p, size_t bytes);
cudaError_t sgm_dev_free(void* p);

template <typename T>
inline cudaError_t sgm_dev_malloc(T** p, size_t bytes) {
  return sgm_dev_malloc(reinterpret_cast<void**>(p), bytes);
}
