// guard.cu -- guard zones around device buffers (guard.cuh) and
// svof_guard_check() / svof_guard_bytes() of the C ABI (svof_b200.h).
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>

#include "../../include/svof_b200.h"
#include "guard.cuh"
#include "solver_state.cuh"

namespace svof_guard {
namespace {

constexpr unsigned char kCanary = 0xA5;

struct Zone {
  unsigned char *base;  // the allocation (guard before, body, guard after)
  size_t body;          // bytes of the buffer itself
  size_t guard;         // bytes of each guard
  long id;              // allocation number (process-wide, from 0)
};

std::mutex g_mu;
std::map<void *, Zone> g_zones;  // by the pointer handed out
long g_next_id = 0;

// counts the bytes of [p, p + n) that differ from the canary
__global__ void k_guard_count(const unsigned char *__restrict__ p, size_t n, unsigned long long *bad) {
  unsigned long long c = 0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    c += (p[q] != kCanary);
  if (c) atomicAdd(bad, c);
}

}  // namespace

size_t guard_bytes() {
  const char *e = std::getenv("SVOF_GUARD_BYTES");
  if (!e || !*e) return 0;
  const long long v = std::atoll(e);
  if (v <= 0) return 0;
  return ((size_t)v + 255) / 256 * 256;
}

cudaError_t alloc(void **ptr, size_t bytes, bool managed) {
  const size_t g = guard_bytes();
  const size_t total = bytes + 2 * g;
  void *base = nullptr;
  cudaError_t e = managed ? cudaMallocManaged(&base, total) : cudaMalloc(&base, total);
  if (cudaSuccess != e) return e;
  if (0 == g) {
    *ptr = base;
    return cudaSuccess;
  }
  unsigned char *b = static_cast<unsigned char *>(base);
  if (cudaSuccess != (e = cudaMemset(b, kCanary, g)) || cudaSuccess != (e = cudaMemset(b + g + bytes, kCanary, g))) {
    cudaFree(base);
    return e;
  }
  *ptr = b + g;
  std::lock_guard<std::mutex> lock(g_mu);
  g_zones[*ptr] = Zone{b, bytes, g, g_next_id++};
  return cudaSuccess;
}

cudaError_t release(void *ptr) {
  if (!ptr) return cudaSuccess;
  void *base = ptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_zones.find(ptr);
    if (it != g_zones.end()) {
      base = it->second.base;
      g_zones.erase(it);
    }
  }
  return cudaFree(base);
}

}  // namespace svof_guard

using namespace svof_guard;

extern "C" {

size_t svof_guard_bytes(void) { return guard_bytes(); }

int svof_guard_check(size_t *bad_bytes) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (bad_bytes) *bad_bytes = 0;
  if (g_zones.empty()) return 0;
  unsigned long long *d_bad = nullptr, h_bad = 0;
  if (cudaSuccess != cudaDeviceSynchronize() || cudaSuccess != cudaMalloc(&d_bad, sizeof(*d_bad)))
    return svof::fail("svof_guard_check: %s", cudaGetErrorString(cudaGetLastError()));
  size_t total = 0;
  std::string first;
  for (const auto &kv : g_zones) {
    const Zone &z = kv.second;
    for (int side = 0; side < 2; side++) {
      const unsigned char *p = side ? z.base + z.guard + z.body : z.base;
      cudaMemset(d_bad, 0, sizeof(*d_bad));
      k_guard_count<<<(unsigned)((z.guard + 255) / 256), 256>>>(p, z.guard, d_bad);
      cudaMemcpy(&h_bad, d_bad, sizeof(h_bad), cudaMemcpyDeviceToHost);
      if (h_bad && first.empty()) {
        char buf[200];
        std::snprintf(buf, sizeof(buf), "device buffer #%ld (%zu bytes): %llu guard bytes %s it overwritten", z.id,
                      z.body, h_bad, side ? "after" : "before");
        first = buf;
      }
      total += h_bad;
    }
  }
  const cudaError_t e = cudaGetLastError();
  cudaFree(d_bad);
  if (bad_bytes) *bad_bytes = total;
  if (cudaSuccess != e) return svof::fail("svof_guard_check: %s", cudaGetErrorString(e));
  if (total) return svof::fail("svof_guard_check: %s", first.c_str());
  return 0;
}

}  // extern "C"
