// GAMMA raster ingest: big-endian samples decoded on the device.
//
// Replaces the host-side decode of moraine.gamma_.read_gamma_image / read_gamma_pdata
// (moraine/gamma_.py:13-56, :59-84): the bytes of the file go to HBM as they are, and one
// pass swaps the byte order and applies the reference's no-data rule (|x| < 1e-30 becomes
// NaN, NaN + NaN j for complex samples; integers are left as they are), writing the
// native samples with an optional output stride so that per-date images interleave
// straight into a (lines, width, dates) stack.
//
// The comparison follows numpy's: for float and fcomplex the magnitude is a float32
// (hypotf for complex, evaluated here as the float32 rounding of the double square root of
// the exact double sum of squares) compared with 1e-30 rounded to float32; for double the
// comparison is in double.
#include <algorithm>

#include "common.cuh"

namespace mr {
namespace {

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }
__device__ __forceinline__ uint64_t bswap64(uint64_t x) {
  const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
  return ((uint64_t)bswap32(lo) << 32) | bswap32(hi);
}

constexpr float kTiny32 = 1.0e-30f;
constexpr double kTiny64 = 1.0e-30;

// One sample per thread iteration; `in` holds n big-endian samples of `bytes` each.
template <int kType>
__global__ void gamma_decode_kernel(const unsigned char* __restrict__ in, int64_t n, void* __restrict__ out,
                                    int64_t stride) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (kType == MR_GAMMA_FLOAT) {
      const uint32_t w = bswap32(reinterpret_cast<const uint32_t*>(in)[i]);
      float v = __uint_as_float(w);
      if (fabsf(v) < kTiny32) v = __int_as_float(0x7fc00000);  // numpy's nan as float32
      static_cast<float*>(out)[i * stride] = v;
    } else if constexpr (kType == MR_GAMMA_INT) {
      const uint32_t w = bswap32(reinterpret_cast<const uint32_t*>(in)[i]);
      static_cast<int32_t*>(out)[i * stride] = (int32_t)w;
    } else if constexpr (kType == MR_GAMMA_DOUBLE) {
      const uint64_t w = bswap64(reinterpret_cast<const unsigned long long*>(in)[i]);
      double v = __longlong_as_double((long long)w);
      if (fabs(v) < kTiny64) v = __longlong_as_double(0x7ff8000000000000ll);
      static_cast<double*>(out)[i * stride] = v;
    } else {  // fcomplex: two big-endian float32, real then imaginary
      const uint2 w = reinterpret_cast<const uint2*>(in)[i];
      float re = __uint_as_float(bswap32(w.x)), im = __uint_as_float(bswap32(w.y));
      const double s = (double)re * re + (double)im * im;  // exact products, one rounding
      const float mag = (float)sqrt(s);
      if (mag < kTiny32) re = im = __int_as_float(0x7fc00000);
      static_cast<float2*>(out)[i * stride] = make_float2(re, im);
    }
  }
}

int grid_for(int64_t n) {
  const int64_t blocks = (n + 255) / 256;
  return (int)std::min<int64_t>(blocks, (int64_t)sm_count() * 16);
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" size_t mr_gamma_sample_bytes(int dtype) {
  switch (dtype) {
    case MR_GAMMA_FLOAT: case MR_GAMMA_INT: return 4;
    case MR_GAMMA_FCOMPLEX: case MR_GAMMA_DOUBLE: return 8;
    default: return 0;
  }
}

extern "C" int mr_gamma_decode(const void* be, int64_t n, int dtype, void* out, int64_t out_stride,
                               mr_stream_t stream) {
  MR_REQUIRE(n >= 0, "gamma_decode: negative sample count");
  MR_REQUIRE(mr_gamma_sample_bytes(dtype) != 0, "gamma_decode: unknown dtype %d", dtype);
  MR_REQUIRE(out_stride >= 1, "gamma_decode: out_stride must be >= 1");
  if (n == 0) return MR_OK;
  MR_REQUIRE(be && out, "gamma_decode: NULL pointer");
  const size_t b = mr_gamma_sample_bytes(dtype);
  MR_REQUIRE(((uintptr_t)be % b) == 0 && ((uintptr_t)out % b) == 0, "gamma_decode: buffers not %zu-byte aligned", b);
  cudaStream_t s = as_stream(stream);
  const auto* in = static_cast<const unsigned char*>(be);
  switch (dtype) {
    case MR_GAMMA_FLOAT: gamma_decode_kernel<MR_GAMMA_FLOAT><<<grid_for(n), 256, 0, s>>>(in, n, out, out_stride); break;
    case MR_GAMMA_FCOMPLEX:
      gamma_decode_kernel<MR_GAMMA_FCOMPLEX><<<grid_for(n), 256, 0, s>>>(in, n, out, out_stride);
      break;
    case MR_GAMMA_INT: gamma_decode_kernel<MR_GAMMA_INT><<<grid_for(n), 256, 0, s>>>(in, n, out, out_stride); break;
    default: gamma_decode_kernel<MR_GAMMA_DOUBLE><<<grid_for(n), 256, 0, s>>>(in, n, out, out_stride); break;
  }
  return check_launch("gamma_decode");
}
