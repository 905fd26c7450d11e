// Error reporting, version and device queries of the moraine_b200 C ABI.
#include <atomic>
#include <cstdarg>
#include <mutex>

#include "common.cuh"

namespace mr {

static thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

}  // namespace mr

extern "C" const char* mr_last_error(void) { return mr::g_last_error; }

namespace mr {
static std::atomic<uint64_t> g_launches{0};
void note_launches(int k) { g_launches.fetch_add((uint64_t)k, std::memory_order_relaxed); }
}  // namespace mr

extern "C" uint64_t mr_kernel_launches(void) { return mr::g_launches.load(std::memory_order_relaxed); }

extern "C" int mr_abi_version(void) { return 1; }
