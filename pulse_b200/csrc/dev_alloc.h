// dev_alloc.h -- the library's one device-allocation call (internal).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace pt {

// cudaMalloc, unless pulse_debug_fail_allocations armed a failure: then the
// call allocates nothing and returns cudaErrorMemoryAllocation, which every
// caller reports as PULSE_ERR_OOM after releasing what it holds.
cudaError_t dev_alloc(void** p, size_t bytes);

}  // namespace pt
