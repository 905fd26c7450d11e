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

// Per-device attribute caches; several host threads may fill an entry at once, all with
// the same value, so the entries are atomics.
int sm_count() {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int c = cached[dev].load(std::memory_order_relaxed);
  if (c == 0) {
    if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0) c = 148;
    cached[dev].store(c, std::memory_order_relaxed);
  }
  return c;
}

int smem_optin() {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  int c = cached[dev].load(std::memory_order_relaxed);
  if (c == 0) {
    if (cudaDeviceGetAttribute(&c, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) c = 0;
    cached[dev].store(c, std::memory_order_relaxed);
  }
  return c;
}

int allow_smem(const void* kernel, size_t bytes) {
  const int optin = smem_optin();
  if (optin <= 0) return fail(MR_ERR_CUDA, "cannot query the shared-memory limit of the device");
  cudaFuncAttributes fa;
  MR_CUDA_TRY(cudaFuncGetAttributes(&fa, kernel));
  const int cap = optin - (int)fa.sharedSizeBytes;  // dynamic share beside the kernel's static one
  if (bytes > (size_t)cap) return fail(MR_ERR_UNSUPPORTED, "%zu bytes of shared memory per CTA > %d", bytes, cap);
  // the device limit, not this launch's size: threads that launch the kernel with other
  // sizes at the same time all write the same value
  MR_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, cap));
  return MR_OK;
}

}  // namespace mr

extern "C" const char* mr_last_error(void) { return mr::g_last_error; }

namespace mr {
static std::atomic<uint64_t> g_launches{0};
void note_launches(int k) { g_launches.fetch_add((uint64_t)k, std::memory_order_relaxed); }
}  // namespace mr

extern "C" uint64_t mr_kernel_launches(void) { return mr::g_launches.load(std::memory_order_relaxed); }

extern "C" int mr_abi_version(void) { return 3; }
