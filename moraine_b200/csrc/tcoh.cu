// Temporal coherence (HBM-streaming, one warp per point) and coherence uncompression.
//
// Reference behaviour followed (kanglcn/moraine):
//   moraine/pl.py:112-120   ds_temp_coh: |sum_q coh_q/|coh_q| conj(ph_m) ph_j| / n_pairs
//   moraine/pqm.py:109-118  temp_coh:    |sum_q intf_q conj(r_m) r_j / sqrt(|intf|^2|r_m|^2|r_j|^2)| / n_pairs
//   moraine/co.py:294-298   uncompress_coh: zeros, pairs and their conjugates, unit diagonal
#include <algorithm>

#include "common.cuh"

namespace mr {
namespace {

// Walk the default upper-triangle pair order: advance (m, j) by t positions.
__device__ __forceinline__ void triu_advance(int& m, int& j, int t, int n) {
  j += t;
  while (j >= n && m < n - 1) { m += 1; j = j - n + m + 1; }
}

template <bool kPqm>
__global__ void __launch_bounds__(256) temp_coh_kernel(const float2* __restrict__ intf,
                                                       const float2* __restrict__ ph, int64_t npts, int n,
                                                       const int32_t* __restrict__ pairs, int npairs,
                                                       float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t pt = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); pt < npts; pt += nw) {
    const float2* c = intf + pt * npairs;
    const float2* p = ph + pt * n;
    float sx = 0.f, sy = 0.f;
    int m = 0, j = 0;
    if (!pairs) { m = 0; j = 1; triu_advance(m, j, lane, n); }
    for (int q = lane; q < npairs; q += 32) {
      int mm, jj;
      if (pairs) {
        mm = pairs[2 * q]; jj = pairs[2 * q + 1];
        if (mm < 0 || mm >= n || jj < 0 || jj >= n) { sx = sy = __int_as_float(0x7fffffff); continue; }
      } else { mm = m; jj = j; triu_advance(m, j, 32, n); }
      const float2 g = c[q], pm = p[mm], pj = p[jj];
      float2 t = cmulc(pj, pm);  // conj(ph_m) ph_j
      float2 v = cmul(g, t);
      float den;
      if (kPqm) {
        den = sqrtf((g.x * g.x + g.y * g.y) * (pm.x * pm.x + pm.y * pm.y) * (pj.x * pj.x + pj.y * pj.y));
      } else {
        den = sqrtf(g.x * g.x + g.y * g.y);
      }
      sx += v.x / den;
      sy += v.y / den;
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    if (lane == 0) out[pt] = sqrtf(sx * sx + sy * sy) / (float)npairs;
  }
}

__global__ void uncompress_fill_kernel(float2* __restrict__ out, int64_t n, int nimg) {
  const int64_t total = n * nimg * nimg;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % ((int64_t)nimg * nimg);
    const int i = (int)(r / nimg), j = (int)(r % nimg);
    out[e] = make_float2(i == j ? 1.f : 0.f, 0.f);
  }
}

__global__ void uncompress_scatter_kernel(const float2* __restrict__ coh, int64_t n, int nimg,
                                          const int32_t* __restrict__ pairs, int npairs, float2* __restrict__ out) {
  const int64_t total = n * npairs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / npairs;
    const int q = (int)(e - i * npairs);
    int m, j;
    if (pairs) { m = pairs[2 * q]; j = pairs[2 * q + 1]; }
    else {
      m = (int)((2.0 * nimg - 1.0 - sqrt((2.0 * nimg - 1.0) * (2.0 * nimg - 1.0) - 8.0 * (double)q)) * 0.5);
      while (m > 0 && triu_index(m, m + 1, nimg) > q) --m;
      while (m + 1 < nimg - 1 && triu_index(m + 1, m + 2, nimg) <= q) ++m;
      j = (int)(q - triu_index(m, m + 1, nimg)) + m + 1;
    }
    if (m < 0 || m >= nimg || j < 0 || j >= nimg) continue;  // pair outside the matrix: ignored
    const float2 v = coh[e];
    float2* o = out + i * nimg * nimg;
    o[(int64_t)m * nimg + j] = v;
    o[(int64_t)j * nimg + m] = make_float2(v.x, -v.y);
  }
}

int grid_for(int64_t items, int per_block) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((items + per_block - 1) / per_block, (int64_t)sm_count() * 32));
}

}  // namespace
}  // namespace mr

using namespace mr;

static int temp_coh_common(bool pqm, const mr_complex64* intf, const mr_complex64* ph, int64_t n, int nimages,
                           const int32_t* image_pairs, int n_pairs, float* t_coh, mr_stream_t stream) {
  MR_REQUIRE(nimages >= 2 && n >= 0, "temp_coh: bad shape");
  if (!image_pairs) n_pairs = nimages * (nimages - 1) / 2;
  MR_REQUIRE(n_pairs > 0, "temp_coh: no pairs");
  if (n == 0) return MR_OK;
  MR_REQUIRE(intf && ph && t_coh, "temp_coh: NULL pointer");
  auto* c = reinterpret_cast<const float2*>(intf);
  auto* p = reinterpret_cast<const float2*>(ph);
  if (pqm)
    temp_coh_kernel<true><<<grid_for(n, 8), 256, 0, as_stream(stream)>>>(c, p, n, nimages, image_pairs, n_pairs, t_coh);
  else
    temp_coh_kernel<false><<<grid_for(n, 8), 256, 0, as_stream(stream)>>>(c, p, n, nimages, image_pairs, n_pairs, t_coh);
  return check_launch("temp_coh");
}

extern "C" int mr_ds_temp_coh(const mr_complex64* coh, const mr_complex64* ph, int64_t n, int nimages,
                              const int32_t* image_pairs, int n_pairs, float* t_coh, mr_stream_t stream) {
  return temp_coh_common(false, coh, ph, n, nimages, image_pairs, n_pairs, t_coh, stream);
}

extern "C" int mr_temp_coh(const mr_complex64* intf, const mr_complex64* rslc, int64_t n, int nimages,
                           const int32_t* image_pairs, int n_pairs, float* t_coh, mr_stream_t stream) {
  return temp_coh_common(true, intf, rslc, n, nimages, image_pairs, n_pairs, t_coh, stream);
}

extern "C" int mr_uncompress_coh(const mr_complex64* coh, int64_t n, int nimages, const int32_t* image_pairs,
                                 int n_pairs, mr_complex64* out, mr_stream_t stream) {
  MR_REQUIRE(nimages >= 1 && n >= 0, "uncompress_coh: bad shape");
  if (!image_pairs) n_pairs = nimages * (nimages - 1) / 2;
  if (n == 0) return MR_OK;
  MR_REQUIRE(coh && out, "uncompress_coh: NULL pointer");
  cudaStream_t s = as_stream(stream);
  auto* o = reinterpret_cast<float2*>(out);
  uncompress_fill_kernel<<<grid_for(n * nimages * nimages, 256), 256, 0, s>>>(o, n, nimages);
  if (n_pairs > 0)
    uncompress_scatter_kernel<<<grid_for(n * n_pairs, 256), 256, 0, s>>>(reinterpret_cast<const float2*>(coh), n,
                                                                        nimages, image_pairs, n_pairs, o);
  return check_launch("uncompress_coh", n_pairs > 0 ? 2 : 1);
}
