// PS-side statistics of the stack: amplitude, amplitude dispersion, calibrated amplitude.
//
// Replace moraine.calamp.rslc2amp (moraine/calamp.py:33-41), moraine.ps.amp_disp
// (moraine/ps.py:65-73) and moraine.calamp.calamp (moraine/calamp.py:63-71). All three are
// HBM-streaming passes over the same (nlines, width, nimages) complex64 stack the DS chain
// reads.
//
// |z| is the float32 rounding of the double square root of the exact double sum of squares,
// +inf when either part is infinite: bit-exact with np.abs on complex64 in the reference's
// Numba build (numpy's own hypotf can differ in the last bit). Means and standard
// deviations accumulate in double and the ratio rounds once to float32.
#include <algorithm>

#include "common.cuh"

namespace mr {
namespace {

__device__ __forceinline__ float abs_c64(float2 z) {
  if (isinf(z.x) || isinf(z.y)) return __int_as_float(0x7f800000);
  return (float)sqrt((double)z.x * z.x + (double)z.y * z.y);
}

__global__ void rslc2amp_kernel(const float2* __restrict__ z, int64_t n, float* __restrict__ amp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    amp[i] = abs_c64(z[i]);
}

// One warp per pixel: the pixel's dates are contiguous (image axis innermost), lanes stride
// over them; mean, then the population standard deviation about it.
constexpr int kMaxPerLane = MR_MAX_NIMAGES / 32;

__global__ void amp_disp_kernel(const float2* __restrict__ z, int64_t npix, int n, float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < npix; p += warps) {
    const float2* zp = z + p * n;
    float a[kMaxPerLane];
    double s = 0;
#pragma unroll
    for (int t = 0; t < kMaxPerLane; ++t) {
      const int k = lane + 32 * t;
      a[t] = 0.f;
      if (k < n) {
        a[t] = abs_c64(zp[k]);
        s += a[t];
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double mean = s / n;
    double v = 0;
#pragma unroll
    for (int t = 0; t < kMaxPerLane; ++t) {
      const int k = lane + 32 * t;
      if (k < n) {
        const double d = (double)a[t] - mean;
        v += d * d;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) out[p] = (float)(sqrt(v / n) / mean);  // one rounding: near-constant PS pixels keep their digits
  }
}

// calamp: per-block (sum, count) of the non-NaN amplitudes in double, then one block adds
// the partials in block order, then every sample is divided by the mean.
constexpr int kCalBlocks = 1024;

__global__ void calamp_partial_kernel(const float* __restrict__ amp, int64_t n, double2* __restrict__ part) {
  __shared__ double ss[8], sc[8];
  double s = 0, c = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = amp[i];
    if (v == v) { s += v; c += 1; }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { ss[w] = s; sc[w] = c; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ts = 0, tc = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { ts += ss[q]; tc += sc[q]; }
    part[blockIdx.x] = make_double2(ts, tc);
  }
}

__global__ void calamp_apply_kernel(const float* __restrict__ amp, int64_t n, const double2* __restrict__ part,
                                    int nparts, float* __restrict__ out) {
  __shared__ float mean;
  if (threadIdx.x == 0) {
    double s = 0, c = 0;
    for (int q = 0; q < nparts; ++q) { s += part[q].x; c += part[q].y; }
    mean = (float)(s / c);
  }
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = amp[i] / mean;
}

int grid_of(int64_t n, int per_block) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + per_block - 1) / per_block, (int64_t)sm_count() * 16));
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" int mr_rslc2amp(const mr_complex64* rslc, int64_t n, float* amp, mr_stream_t stream) {
  MR_REQUIRE(n >= 0, "rslc2amp: negative size");
  if (n == 0) return MR_OK;
  MR_REQUIRE(rslc && amp, "rslc2amp: NULL pointer");
  rslc2amp_kernel<<<grid_of(n, 256), 256, 0, as_stream(stream)>>>(reinterpret_cast<const float2*>(rslc), n, amp);
  return check_launch("rslc2amp");
}

extern "C" int mr_amp_disp(const mr_complex64* rslc, int64_t npix, int nimages, float* amp_disp, mr_stream_t stream) {
  MR_REQUIRE(npix >= 0 && nimages >= 1, "amp_disp: bad stack shape");
  if (nimages > MR_MAX_NIMAGES) return fail(MR_ERR_UNSUPPORTED, "amp_disp: nimages %d > %d", nimages, MR_MAX_NIMAGES);
  if (npix == 0) return MR_OK;
  MR_REQUIRE(rslc && amp_disp, "amp_disp: NULL pointer");
  amp_disp_kernel<<<grid_of(npix, 8), 256, 0, as_stream(stream)>>>(reinterpret_cast<const float2*>(rslc), npix,
                                                                   nimages, amp_disp);
  return check_launch("amp_disp");
}

extern "C" size_t mr_calamp_workspace_bytes(void) { return kCalBlocks * sizeof(double2); }

extern "C" int mr_calamp(const float* amp, int64_t n, float* out, void* workspace, size_t workspace_bytes,
                         mr_stream_t stream) {
  MR_REQUIRE(n >= 0, "calamp: negative size");
  if (n == 0) return MR_OK;
  MR_REQUIRE(amp && out, "calamp: NULL pointer");
  if (!workspace || workspace_bytes < mr_calamp_workspace_bytes())
    return fail(MR_ERR_WORKSPACE, "calamp: workspace %zu < %zu bytes", workspace_bytes, mr_calamp_workspace_bytes());
  MR_REQUIRE(((uintptr_t)workspace & 15) == 0, "calamp: workspace not 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  auto* part = static_cast<double2*>(workspace);
  const int nb = (int)std::min<int64_t>(kCalBlocks, std::max<int64_t>(1, (n + 255) / 256));
  calamp_partial_kernel<<<nb, 256, 0, s>>>(amp, n, part);
  calamp_apply_kernel<<<grid_of(n, 256), 256, 0, s>>>(amp, n, part, nb, out);
  return check_launch("calamp", 2);
}
