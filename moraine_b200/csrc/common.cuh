// Shared helpers for the moraine_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/moraine_b200.h"

namespace mr {

// Last error message of the calling host thread (read through mr_last_error()).
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

// Kernel launches made by the library since the process started (mr_kernel_launches()).
void note_launches(int k);

// Status of the launches just made; counts them.
inline int check_launch(const char* what, int launches = 1) {
  note_launches(launches);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return MR_OK;
}

#define MR_REQUIRE(cond, ...)                        \
  do {                                               \
    if (!(cond)) return ::mr::fail(MR_ERR_INVALID, __VA_ARGS__); \
  } while (0)

#define MR_CUDA_TRY(expr)                                                        \
  do {                                                                           \
    cudaError_t _e = (expr);                                                     \
    if (_e != cudaSuccess)                                                       \
      return ::mr::fail(MR_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e));   \
  } while (0)

inline cudaStream_t as_stream(mr_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Per-kernel device timing for benchmarks (mr_set_kernel_timing): while it is on, an
// instrumented launch records a CUDA event pair around itself on its stream (never inside
// a stream capture), and mr_kernel_timing adds them up per kernel name. Off by default;
// the object does nothing then.
class KernelTimer {
 public:
  KernelTimer(const char* name, cudaStream_t s);
  ~KernelTimer();
  KernelTimer(const KernelTimer&) = delete;
  KernelTimer& operator=(const KernelTimer&) = delete;

 private:
  const char* name_;
  cudaStream_t s_;
  cudaEvent_t e0_ = nullptr;
};

// Number of SMs of the current device (cached per device).
int sm_count();

// Largest dynamic shared memory per CTA of the current device (opt-in limit).
int smem_optin();

// Lets `kernel` launch with up to the device's opt-in shared memory; fails when `bytes`
// exceed it. Safe when several host threads launch the kernel with different sizes.
int allow_smem(const void* kernel, size_t bytes);

// Work sized on the device (graph-capturable chain): the point count lives in device memory
// (*dcount, of which points doff .. doff + n_max - 1 are this call's); the kernels clamp
// to it, so the host launches for the largest count and never reads the real one.
int gram_counted(const float2* rslc, int nlines, int width, int n, const int32_t* idx, int64_t n_max,
                 const int64_t* dcount, int64_t doff, const uint8_t* mask, int az_win, int r_win, float2* coh,
                 int precision, cudaStream_t s);
int emi_counted(const float2* coh, int64_t n_max, const int64_t* dcount, int64_t doff, int n, int precision,
                float2* ph, float* quality, float* tcoh, void* workspace, size_t workspace_bytes, cudaStream_t s);

// Pair index of (m, j), m < j, in the row-major upper triangle of an N x N matrix
// (the order of numpy.triu_indices(N, 1)).
__host__ __device__ __forceinline__ int64_t triu_index(int m, int j, int n) {
  return (int64_t)m * n - ((int64_t)m * (m + 1)) / 2 + (j - m - 1);
}

// ---- complex helpers (float2 / double2 carry numpy complex64 / complex128 layouts) ----
template <typename T> struct cplx;
template <> struct cplx<float> { using type = float2; };
template <> struct cplx<double> { using type = double2; };

template <typename C> __host__ __device__ __forceinline__ C cmake(double re, double im) {
  C c; c.x = re; c.y = im; return c;
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 conjc(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ double2 conjc(double2 a) { return make_double2(a.x, -a.y); }

// ---- warp / block reductions ----
template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace mr
