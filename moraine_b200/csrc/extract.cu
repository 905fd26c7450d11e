// DS-candidate extraction: stream compaction of pixels with shp_num >= min_shp into
// (azimuth, range) indices and, optionally, their window masks, in row-major pixel
// order (the order of numpy.where on the (nlines, width) raster).
#include "common.cuh"

namespace mr {
namespace {

constexpr int kBlk = 1024;      // pixels per block
constexpr int kThreads = 256;   // 4 pixels per thread

__global__ void __launch_bounds__(kThreads) count_kernel(const int32_t* __restrict__ shp_num,
                                                         int64_t npix, int min_shp,
                                                         int64_t* __restrict__ counts) {
  const int64_t base = (int64_t)blockIdx.x * kBlk;
  int c = 0;
  for (int k = threadIdx.x; k < kBlk; k += kThreads) {
    int64_t i = base + k;
    c += (i < npix && shp_num[i] >= min_shp);
  }
  c = warp_sum(c);
  __shared__ int s[kThreads / 32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kThreads / 32; ++w) t += s[w];
    counts[blockIdx.x] = t;
  }
}

// Single-block exclusive scan of the per-block counts (in place), total to *n_ds.
__global__ void __launch_bounds__(1024) scan_kernel(int64_t* __restrict__ counts, int64_t nblocks,
                                                    int64_t* __restrict__ n_ds) {
  __shared__ int64_t s[1024];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b0 = 0; b0 < nblocks; b0 += 1024) {
    int64_t i = b0 + threadIdx.x;
    int64_t v = (i < nblocks) ? counts[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      int64_t t = (threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nblocks) counts[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += s[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_ds = carry;
}

__global__ void __launch_bounds__(kThreads) scatter_kernel(
    const int32_t* __restrict__ shp_num, const uint8_t* __restrict__ is_shp, int64_t npix, int width,
    int win, int min_shp, const int64_t* __restrict__ offsets, int32_t* __restrict__ idx,
    uint8_t* __restrict__ pc_is_shp, int64_t max_ds) {
  __shared__ int s_warp[kThreads / 32];
  __shared__ int64_t s_sel[kBlk];
  __shared__ int s_nsel;
  const int64_t base = (int64_t)blockIdx.x * kBlk;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // each thread owns 4 consecutive pixels -> order preserved by thread-major scan
  int flags[4], c = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int64_t i = base + threadIdx.x * 4 + k;
    flags[k] = (i < npix && shp_num[i] >= min_shp);
    c += flags[k];
  }
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  int wbase = 0;
  for (int w = 0; w < wid; ++w) wbase += s_warp[w];
  if (threadIdx.x == kThreads - 1) s_nsel = wbase + incl;
  int pos = wbase + incl - c;
  const int64_t off = offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (flags[k]) {
      int64_t i = base + threadIdx.x * 4 + k;
      int64_t d = off + pos;
      if (d < max_ds) {
        idx[2 * d] = (int32_t)(i / width);
        idx[2 * d + 1] = (int32_t)(i % width);
      }
      s_sel[pos] = i;
      ++pos;
    }
  }
  __syncthreads();
  if (pc_is_shp) {
    const int nsel = s_nsel;
    for (int k = wid; k < nsel; k += kThreads / 32) {
      int64_t d = off + k;
      if (d >= max_ds) break;
      const uint8_t* src = is_shp + s_sel[k] * win;
      uint8_t* dst = pc_is_shp + d * win;
      for (int e = lane; e < win; e += 32) dst[e] = src[e];
    }
  }
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" size_t mr_ds_extract_workspace_bytes(int64_t npix) {
  if (npix <= 0) return 16;
  return (size_t)((npix + kBlk - 1) / kBlk) * sizeof(int64_t);
}

extern "C" int mr_ds_extract(const int32_t* shp_num, const uint8_t* is_shp, int nlines, int width,
                             int win, int min_shp, int32_t* idx, uint8_t* pc_is_shp, int64_t max_ds,
                             int64_t* n_ds, void* workspace, size_t workspace_bytes,
                             mr_stream_t stream) {
  MR_REQUIRE(shp_num && n_ds, "ds_extract: NULL shp_num or n_ds");
  MR_REQUIRE(nlines >= 0 && width >= 0 && win > 0, "ds_extract: bad shape");
  MR_REQUIRE(max_ds >= 0, "ds_extract: negative max_ds");
  MR_REQUIRE(pc_is_shp == nullptr || is_shp != nullptr, "ds_extract: pc_is_shp needs is_shp");
  MR_REQUIRE(max_ds == 0 || idx != nullptr, "ds_extract: idx is NULL");
  const int64_t npix = (int64_t)nlines * width;
  cudaStream_t s = as_stream(stream);
  if (npix == 0) {
    MR_CUDA_TRY(cudaMemsetAsync(n_ds, 0, sizeof(int64_t), s));
    return MR_OK;
  }
  const int64_t nblocks = (npix + kBlk - 1) / kBlk;
  if (!workspace || workspace_bytes < mr_ds_extract_workspace_bytes(npix))
    return fail(MR_ERR_WORKSPACE, "ds_extract: workspace too small");
  MR_REQUIRE(nblocks < (1ll << 31), "ds_extract: raster too large");
  int64_t* counts = static_cast<int64_t*>(workspace);
  count_kernel<<<(unsigned)nblocks, kThreads, 0, s>>>(shp_num, npix, min_shp, counts);
  scan_kernel<<<1, 1024, 0, s>>>(counts, nblocks, n_ds);
  scatter_kernel<<<(unsigned)nblocks, kThreads, 0, s>>>(shp_num, is_shp, npix, width, win, min_shp,
                                                        counts, idx, pc_is_shp, max_ds);
  return check_launch("ds_extract", 3);
}

// ------------------------------------------------------------------------------------
// Allocation-free variant.
//
// Some callers cannot hand this library a device workspace: a host that owns every
// byte of device memory up front (a fixed-budget tile server, a plugin inside another
// framework's process whose allocator must not be bypassed) or a binding from a language
// with no route to a device allocator. For them mr_ds_extract_noalloc keeps its per-block
// counts in a fixed array compiled into this library instead of a caller workspace.
//
// The array below lives in every GPU that loads the library until the process exits
// (kNoAllocMaxBlocks * 8 bytes = 128 KiB per device). Its address is a device address,
// which host code must look up per device (cudaGetSymbolAddress) before passing it to a
// kernel: the symbol's name in host code is only a host-side stand-in.
#include <cuda.h>

#include <mutex>

namespace mr {
namespace {

constexpr int64_t kNoAllocMaxBlocks = 16384;  // rasters up to 16384 * 1024 = 16,777,216 pixels
static_assert(kNoAllocMaxBlocks * kBlk == MR_DS_EXTRACT_NOALLOC_MAX_PIXELS,
              "the header's pixel limit must match the compiled array");
static __device__ __align__(256) int64_t g_extract_counts[kNoAllocMaxBlocks];

// ID of the calling thread's current CUDA context (0 if none or if the driver cannot tell).
// The driver's functions come through the runtime, so the library needs no libcuda link.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault) == cudaSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault) == cudaSuccess) get_id = reinterpret_cast<GetId>(f);
    cudaGetLastError();
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_extract_counts in the current context. The module that holds the
// array is loaded once per context, so the address is looked up (cudaGetSymbolAddress,
// with the device current) on the first call in a context and kept with that context's
// ID: a context torn down and created again (cudaDeviceReset) gets a new ID, and the
// next call looks the address up again instead of using a stale one.
int noalloc_counts(int64_t** out) {
  static std::mutex mu;
  static unsigned long long ctx_of[64] = {0};
  static int64_t* addr[64] = {nullptr};
  int dev = 0;
  MR_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(MR_ERR_UNSUPPORTED, "ds_extract_noalloc: device index %d", dev);
  std::lock_guard<std::mutex> lock(mu);
  const unsigned long long id = current_context_id();
  if (addr[dev] == nullptr || id == 0 || id != ctx_of[dev]) {
    void* p = nullptr;
    MR_CUDA_TRY(cudaGetSymbolAddress(&p, g_extract_counts));
    addr[dev] = static_cast<int64_t*>(p);
    ctx_of[dev] = current_context_id();  // the lookup made the primary context current if none was
  }
  *out = addr[dev];
  return MR_OK;
}

}  // namespace
}  // namespace mr

extern "C" int mr_ds_extract_noalloc(const int32_t* shp_num, const uint8_t* is_shp, int nlines, int width, int win,
                                     int min_shp, int32_t* idx, uint8_t* pc_is_shp, int64_t max_ds, int64_t* n_ds,
                                     mr_stream_t stream) {
  MR_REQUIRE(shp_num && n_ds, "ds_extract_noalloc: NULL shp_num or n_ds");
  MR_REQUIRE(nlines >= 0 && width >= 0 && win > 0, "ds_extract_noalloc: bad shape");
  MR_REQUIRE(max_ds >= 0, "ds_extract_noalloc: negative max_ds");
  MR_REQUIRE(pc_is_shp == nullptr || is_shp != nullptr, "ds_extract_noalloc: pc_is_shp needs is_shp");
  MR_REQUIRE(max_ds == 0 || idx != nullptr, "ds_extract_noalloc: idx is NULL");
  const int64_t npix = (int64_t)nlines * width;
  const int64_t nblocks = (npix + kBlk - 1) / kBlk;
  if (nblocks > kNoAllocMaxBlocks)
    return fail(MR_ERR_UNSUPPORTED,
                "ds_extract_noalloc: raster of %lld pixels exceeds the %lld-pixel limit of the allocation-free "
                "variant; use mr_ds_extract with a workspace",
                (long long)npix, (long long)(kNoAllocMaxBlocks * kBlk));
  cudaStream_t s = as_stream(stream);
  if (npix == 0) {
    MR_CUDA_TRY(cudaMemsetAsync(n_ds, 0, sizeof(int64_t), s));
    return MR_OK;
  }
  int64_t* counts = nullptr;
  if (int rc = noalloc_counts(&counts)) return rc;
  // count_kernel overwrites counts[0, nblocks) before anything reads them, so what an
  // earlier call left in the array never leaks into this one
  count_kernel<<<(unsigned)nblocks, kThreads, 0, s>>>(shp_num, npix, min_shp, counts);
  scan_kernel<<<1, 1024, 0, s>>>(counts, nblocks, n_ds);
  scatter_kernel<<<(unsigned)nblocks, kThreads, 0, s>>>(shp_num, is_shp, npix, width, win, min_shp, counts, idx,
                                                        pc_is_shp, max_ds);
  return check_launch("ds_extract_noalloc", 3);
}
