// fault_hook.cuh -- host-side fault injection for the failure-detection
// tests.  With SVOF_FAIL_ALLOC=N in the environment, the N-th device-buffer
// allocation of a solver's creation (svof_create, svof3d_create) reports an
// out-of-memory failure without allocating, so that the error path, and the
// release of what was allocated before it, run without a GPU fault.
#pragma once

#include <cstdlib>

namespace svof_fault {

inline thread_local int g_alloc_seq = 0;   // allocations of the creation in progress
inline thread_local int g_alloc_fail = 0;  // the one that fails (0: none)

// at the start of a creation: reads SVOF_FAIL_ALLOC
inline void begin_creation() {
  g_alloc_seq = 0;
  const char *e = std::getenv("SVOF_FAIL_ALLOC");
  g_alloc_fail = e ? std::atoi(e) : 0;
}

// counts an allocation; true for the one that is to fail
inline bool next_alloc_fails() { return g_alloc_fail > 0 && ++g_alloc_seq == g_alloc_fail; }

}  // namespace svof_fault
