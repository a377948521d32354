// guard.cuh -- guard zones around the library's device buffers (a debugging
// aid in place of a memory checker).
//
// With SVOF_GUARD_BYTES=N in the environment (N > 0, rounded up to a multiple
// of 256), every buffer the 2D and 3D solvers allocate for their fields,
// tables and scratch gets N bytes before and N after it, filled with a canary
// byte; the buffer itself keeps its 256-byte alignment.  svof_guard_check()
// scans every live guard zone of the process on the device and reports the
// first one whose bytes changed: a kernel that wrote outside its buffer.
// Reads outside a buffer are not detected.  Without the variable (the
// default) buffers are allocated exactly as before.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace svof_guard {

// the guard band of new allocations in bytes (0: none), from the environment
size_t guard_bytes();
// cudaMalloc (or cudaMallocManaged) of `bytes` with guard zones around the
// returned pointer when guard_bytes() > 0
cudaError_t alloc(void **ptr, size_t bytes, bool managed);
// frees a pointer from alloc()
cudaError_t release(void *ptr);

}  // namespace svof_guard
