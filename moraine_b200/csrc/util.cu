// Error reporting, version and device queries of the moraine_b200 C ABI.
#include <atomic>
#include <cstdarg>
#include <map>
#include <mutex>
#include <string>
#include <vector>

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

extern "C" int mr_abi_version(void) { return 4; }

// ---------------------------------------------------------------- per-kernel timing

namespace mr {
namespace {
struct TimedLaunch {
  const char* name;
  cudaEvent_t e0, e1;
};
std::atomic<int> g_ktiming{0};
std::mutex g_kt_mu;
std::vector<TimedLaunch> g_kt_pending;
std::vector<std::pair<std::string, std::pair<double, int64_t>>> g_kt_totals;

void kt_collect() {  // caller holds g_kt_mu
  std::map<std::string, std::pair<double, int64_t>> acc;
  for (auto& kv : g_kt_totals) acc[kv.first] = kv.second;
  for (const TimedLaunch& t : g_kt_pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(t.e1) == cudaSuccess && cudaEventElapsedTime(&ms, t.e0, t.e1) == cudaSuccess) {
      auto& a = acc[t.name];
      a.first += ms;
      a.second += 1;
    }
    cudaEventDestroy(t.e0);
    cudaEventDestroy(t.e1);
  }
  g_kt_pending.clear();
  cudaGetLastError();
  g_kt_totals.assign(acc.begin(), acc.end());
}
}  // namespace

KernelTimer::KernelTimer(const char* name, cudaStream_t s) : name_(name), s_(s) {
  if (!g_ktiming.load(std::memory_order_relaxed)) return;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return;
  }
  if (cudaEventCreate(&e0_) != cudaSuccess) { e0_ = nullptr; cudaGetLastError(); return; }
  cudaEventRecord(e0_, s);
}

KernelTimer::~KernelTimer() {
  if (!e0_) return;
  cudaEvent_t e1 = nullptr;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0_); cudaGetLastError(); return; }
  cudaEventRecord(e1, s_);
  std::lock_guard<std::mutex> lk(g_kt_mu);
  g_kt_pending.push_back({name_, e0_, e1});
}
}  // namespace mr

extern "C" void mr_set_kernel_timing(int on) {
  std::lock_guard<std::mutex> lk(mr::g_kt_mu);
  mr::kt_collect();
  mr::g_kt_totals.clear();
  mr::g_ktiming.store(on ? 1 : 0);
}

extern "C" int mr_kernel_timing(int i, const char** name, double* total_ms, int64_t* launches) {
  std::lock_guard<std::mutex> lk(mr::g_kt_mu);
  mr::kt_collect();
  const int n = (int)mr::g_kt_totals.size();
  if (i >= 0 && i < n) {
    if (name) *name = mr::g_kt_totals[i].first.c_str();
    if (total_ms) *total_ms = mr::g_kt_totals[i].second.first;
    if (launches) *launches = mr::g_kt_totals[i].second.second;
  }
  return n;
}
