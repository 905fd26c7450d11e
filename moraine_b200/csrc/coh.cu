// Coherence estimation on SIMT cores: the SHP-masked complex Gram of every point,
// normalised to coherence (point-cloud, upper-triangle compressed) or to covariance and
// coherence (raster, full N x N).
//
// Reference behaviour followed (kanglcn/moraine):
//   moraine/co.py:164-187  coh[i,q] = sum z_m conj(z_j) / sqrt(sum|z_m|^2 sum|z_j|^2) over the
//                          window pixels with pc_is_shp set that lie inside the image,
//                          summed in window order (row-major over the az x r window)
//   moraine/co.py:83-110   raster: cov = sum / n_shp, coh as above, every (m, j)
#include <algorithm>

#include "common.cuh"

namespace mr {
namespace {

constexpr int kGramThreads = 256;
constexpr int kChunk = 32;  // SHP rows staged per pass

template <typename A> struct Acc2;
template <> struct Acc2<float> { using type = float2; };
template <> struct Acc2<double> { using type = double2; };

// Block-wide compaction of a window mask into the linear pixel indices of the SHPs that
// lie inside the image, in window order. Returns the count (same in every thread).
__device__ int collect_shps(const uint8_t* __restrict__ mask, int az_win, int r_win, int ra, int rr,
                            int nlines, int width, int* __restrict__ s_pos, int* __restrict__ s_tmp) {
  const int win = az_win * r_win;
  const int azh = az_win / 2, rh = r_win / 2;
  const int per = (win + blockDim.x - 1) / blockDim.x;
  const int e0 = threadIdx.x * per, e1 = min(win, e0 + per);
  int c = 0;
  for (int e = e0; e < e1; ++e) {
    int k = e / r_win, l = e - k * r_win;
    int sa = ra - azh + k, sr = rr - rh + l;
    c += (mask[e] && sa >= 0 && sa < nlines && sr >= 0 && sr < width);
  }
  // block exclusive scan of c
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_tmp[wid] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { int t = s_tmp[w]; s_tmp[w] = run; run += t; }
    s_tmp[32] = run;
  }
  __syncthreads();
  int pos = s_tmp[wid] + incl - c;
  for (int e = e0; e < e1; ++e) {
    int k = e / r_win, l = e - k * r_win;
    int sa = ra - azh + k, sr = rr - rh + l;
    if (mask[e] && sa >= 0 && sa < nlines && sr >= 0 && sr < width) s_pos[pos++] = sa * width + sr;
  }
  __syncthreads();
  int total = s_tmp[32];
  __syncthreads();
  return total;
}

// One CTA per point (grid-stride). Each thread accumulates a 4x4 block of the N x N
// Gram over the point's SHPs, staged kChunk rows at a time in shared memory.
// kFull = false: upper-triangle blocks, writes coh (n_pc, Q) in triu order.
// kFull = true : all blocks, writes cov and coh (npix, N, N) (raster form).
template <typename A, bool kFull>
__global__ void __launch_bounds__(kGramThreads) gram_kernel(
    const float2* __restrict__ rslc, int nlines, int width, int n, const int32_t* __restrict__ idx,
    int64_t n_pc, const uint8_t* __restrict__ mask, int mask_stride, int az_win, int r_win,
    float2* __restrict__ coh, float2* __restrict__ cov, const int64_t* __restrict__ dcount, int64_t doff) {
  using C = typename Acc2<A>::type;
  if (dcount) {  // points doff .. doff + n_pc - 1 of a count held on the device
    const int64_t c = *dcount - doff;
    n_pc = c < 0 ? 0 : (c < n_pc ? c : n_pc);
  }
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int win = az_win * r_win;
  const int npad = (n + 3) & ~3;
  float2* zc = reinterpret_cast<float2*>(smem_raw);                  // kChunk x npad
  A* amp2 = reinterpret_cast<A*>(zc + kChunk * npad);                 // npad
  int* s_pos = reinterpret_cast<int*>(amp2 + npad);                   // win
  __shared__ int s_tmp[33];
  const int nb = npad / 4;
  const int nblk = kFull ? nb * nb : nb * (nb + 1) / 2;
  const int64_t npairs = (int64_t)n * (n - 1) / 2;

  for (int64_t i = blockIdx.x; i < n_pc; i += gridDim.x) {
    int ra, rr;
    if (idx) { ra = idx[2 * i]; rr = idx[2 * i + 1]; }
    else { ra = (int)(i / width); rr = (int)(i % width); }
    if (ra < 0 || ra >= nlines || rr < 0 || rr >= width) {  // index outside the image: NaN row
      const float2 nan2 = make_float2(__int_as_float(0x7fffffff), __int_as_float(0x7fffffff));
      if (kFull) {
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) { coh[i * n * n + e] = nan2; cov[i * n * n + e] = nan2; }
      } else {
        for (int64_t e = threadIdx.x; e < npairs; e += blockDim.x) coh[i * npairs + e] = nan2;
      }
      continue;
    }
    const uint8_t* m = mask + (mask_stride ? ((int64_t)ra * width + rr) : i) * win;
    const int S = collect_shps(m, az_win, r_win, ra, rr, nlines, width, s_pos, s_tmp);
    // amplitude sums, window order
    for (int c = threadIdx.x; c < npad; c += blockDim.x) {
      A s = 0;
      if (c < n)
        for (int t = 0; t < S; ++t) {
          float2 z = rslc[(int64_t)s_pos[t] * n + c];
          s += (A)z.x * (A)z.x + (A)z.y * (A)z.y;
        }
      amp2[c] = s;
    }
    __syncthreads();
    for (int round = 0; round * kGramThreads < nblk; ++round) {
      const int blk = round * kGramThreads + threadIdx.x;
      const bool active = blk < nblk;
      int bm = 0, bj = 0;
      if (active) {
        if (kFull) { bm = blk / nb; bj = blk - bm * nb; }
        else {  // blk -> (bm <= bj), row-major over the upper triangle of blocks
          int b = blk; bm = 0;
          while (b >= nb - bm) { b -= nb - bm; ++bm; }
          bj = bm + b;
        }
      }
      C acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) { acc[a][b].x = 0; acc[a][b].y = 0; }
      const int sdt = (int)blockDim.x / npad, sdc = (int)blockDim.x - sdt * npad;
      for (int s0 = 0; s0 < S; s0 += kChunk) {
        const int ns = min(kChunk, S - s0);
        __syncthreads();
        // (row t, column c) of element e followed incrementally: no division per element
        // (3 % faster)
        for (int e = threadIdx.x, t = threadIdx.x / npad, c = threadIdx.x - (threadIdx.x / npad) * npad;
             e < ns * npad; e += blockDim.x) {
          float2 z = make_float2(0.f, 0.f);
          if (c < n) z = rslc[(int64_t)s_pos[s0 + t] * n + c];
          zc[t * npad + c] = z;
          t += sdt;
          c += sdc;
          if (c >= npad) { c -= npad; ++t; }
        }
        __syncthreads();
        if (active) {
          for (int t = 0; t < ns; ++t) {
            const float4* row = reinterpret_cast<const float4*>(zc + t * npad);
            float4 ma = row[2 * bm], mb = row[2 * bm + 1];
            float4 ja = row[2 * bj], jb = row[2 * bj + 1];
            const A zm[4][2] = {{ma.x, ma.y}, {ma.z, ma.w}, {mb.x, mb.y}, {mb.z, mb.w}};
            const A zj[4][2] = {{ja.x, ja.y}, {ja.z, ja.w}, {jb.x, jb.y}, {jb.z, jb.w}};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
              for (int b = 0; b < 4; ++b) {
                // z_m * conj(z_j). FP64: one FMA per product (the FP64 pipe bounds this loop,
                // and the summed form costs a multiply and an add more per component, 13 %
                // slower). FP32: the summed form, which rounds into the accumulator once per
                // SHP instead of twice (with the FMA chain the error reached 2.5e-6 at 465
                // SHPs, above the FP32 Gram's 2e-6 bound).
                if constexpr (sizeof(A) == 8) {
                  acc[a][b].x += zm[a][0] * zj[b][0];
                  acc[a][b].x += zm[a][1] * zj[b][1];
                  acc[a][b].y += zm[a][1] * zj[b][0];
                  acc[a][b].y -= zm[a][0] * zj[b][1];
                } else {
                  acc[a][b].x += zm[a][0] * zj[b][0] + zm[a][1] * zj[b][1];
                  acc[a][b].y += zm[a][1] * zj[b][0] - zm[a][0] * zj[b][1];
                }
              }
          }
        }
      }
      if (active) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int mm = 4 * bm + a, jj = 4 * bj + b;
            if (mm >= n || jj >= n) continue;
            A den = sqrt(amp2[mm] * amp2[jj]);
            if (kFull) {
              const int64_t o = (i * n + mm) * n + jj;
              coh[o] = make_float2((float)(acc[a][b].x / den), (float)(acc[a][b].y / den));
              cov[o] = make_float2((float)(acc[a][b].x / (A)S), (float)(acc[a][b].y / (A)S));
            } else if (mm < jj) {
              const int64_t o = i * npairs + triu_index(mm, jj, n);
              coh[o] = make_float2((float)(acc[a][b].x / den), (float)(acc[a][b].y / den));
            }
          }
      }
    }
    __syncthreads();
  }
}

// Arbitrary pair lists: one thread per (point, pair), serial over the window.
__global__ void gram_pairs_kernel(const float2* __restrict__ rslc, int nlines, int width, int n,
                                  const int32_t* __restrict__ idx, int64_t n_pc,
                                  const uint8_t* __restrict__ mask, int mask_stride, int az_win,
                                  int r_win, const int32_t* __restrict__ pairs, int npairs,
                                  float2* __restrict__ coh) {
  const int64_t total = n_pc * npairs;
  const int azh = az_win / 2, rh = r_win / 2, win = az_win * r_win;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / npairs;
    const int q = (int)(e - i * npairs);
    const int mm = pairs[2 * q], jj = pairs[2 * q + 1];
    const int ra = idx[2 * i], rr = idx[2 * i + 1];
    if (mm < 0 || mm >= n || jj < 0 || jj >= n || ra < 0 || ra >= nlines || rr < 0 || rr >= width) {
      coh[e] = make_float2(__int_as_float(0x7fffffff), __int_as_float(0x7fffffff));
      continue;
    }
    const uint8_t* m = mask + (mask_stride ? ((int64_t)ra * width + rr) : i) * win;
    float nr = 0.f, ni = 0.f, am = 0.f, aj = 0.f;
    for (int k = 0; k < az_win; ++k)
      for (int l = 0; l < r_win; ++l) {
        const int sa = ra - azh + k, sr = rr - rh + l;
        if (m[k * r_win + l] && sa >= 0 && sa < nlines && sr >= 0 && sr < width) {
          const float2 zm = rslc[((int64_t)sa * width + sr) * n + mm];
          const float2 zj = rslc[((int64_t)sa * width + sr) * n + jj];
          am += zm.x * zm.x + zm.y * zm.y;
          aj += zj.x * zj.x + zj.y * zj.y;
          nr += zm.x * zj.x + zm.y * zj.y;
          ni += zm.y * zj.x - zm.x * zj.y;
        }
      }
    const float den = sqrtf(am * aj);
    coh[e] = make_float2(nr / den, ni / den);
  }
}

template <typename A, bool kFull>
int launch_gram(const float2* rslc, int nlines, int width, int n, const int32_t* idx, int64_t n_pc,
                const uint8_t* mask, int mask_stride, int az_win, int r_win, float2* coh, float2* cov,
                cudaStream_t s, const int64_t* dcount = nullptr, int64_t doff = 0) {
  const int npad = (n + 3) & ~3;
  const size_t smem = (size_t)kChunk * npad * sizeof(float2) + npad * sizeof(A) +
                      (size_t)az_win * r_win * sizeof(int);
  if (int rc = allow_smem(reinterpret_cast<const void*>(gram_kernel<A, kFull>), smem)) return rc;
  const int64_t grid = std::min<int64_t>(n_pc, (int64_t)sm_count() * 8);
  KernelTimer kt(sizeof(A) == 8 ? "gram fp64" : "gram fp32", s);
  gram_kernel<A, kFull><<<(unsigned)grid, kGramThreads, smem, s>>>(rslc, nlines, width, n, idx, n_pc, mask,
                                                                   mask_stride, az_win, r_win, coh, cov, dcount, doff);
  return check_launch("coherence gram");
}

}  // namespace

// Tensor-core Gram (coh_tc.cu); returns MR_ERR_UNSUPPORTED for shapes it does not take.
int gram_tc(const float2* rslc, int nlines, int width, int n, const int32_t* idx, int64_t n_pc,
            const uint8_t* mask, int mask_stride, int az_win, int r_win, float2* coh, int precision,
            cudaStream_t s);

}  // namespace mr

using namespace mr;

extern "C" int mr_emperical_co_pc(const mr_complex64* rslc, int nlines, int width, int nimages,
                                  const int32_t* idx, int64_t n_pc, const uint8_t* mask, int mask_stride,
                                  int az_win, int r_win, const int32_t* image_pairs, int n_pairs,
                                  mr_complex64* coh, int precision, mr_stream_t stream) {
  MR_REQUIRE(n_pc >= 0, "emperical_co_pc: negative n_pc");
  if (n_pc == 0) return MR_OK;
  MR_REQUIRE(rslc && idx && mask && coh, "emperical_co_pc: NULL pointer");
  MR_REQUIRE(nlines > 0 && width > 0 && nimages >= 2, "emperical_co_pc: bad stack shape");
  MR_REQUIRE(az_win > 0 && r_win > 0 && (az_win & 1) && (r_win & 1),
             "emperical_co_pc: window (%d, %d) must be odd", az_win, r_win);
  if (nimages > MR_MAX_NIMAGES) return fail(MR_ERR_UNSUPPORTED, "emperical_co_pc: nimages > %d", MR_MAX_NIMAGES);
  if ((int64_t)az_win * r_win > MR_MAX_WINDOW) return fail(MR_ERR_UNSUPPORTED, "emperical_co_pc: window too large");
  MR_REQUIRE(mask_stride == 0 || mask_stride == 1, "emperical_co_pc: mask_stride must be 0 or 1");
  MR_REQUIRE(n_pc >= 0, "emperical_co_pc: negative n_pc");
  if (n_pc == 0) return MR_OK;
  cudaStream_t s = as_stream(stream);
  const float2* z = reinterpret_cast<const float2*>(rslc);
  float2* out = reinterpret_cast<float2*>(coh);
  if (image_pairs) {
    MR_REQUIRE(n_pairs > 0, "emperical_co_pc: n_pairs must be > 0");
    int grid = (int)std::min<int64_t>((n_pc * n_pairs + 255) / 256, (int64_t)sm_count() * 32);
    gram_pairs_kernel<<<grid, 256, 0, s>>>(z, nlines, width, nimages, idx, n_pc, mask, mask_stride, az_win,
                                          r_win, image_pairs, n_pairs, out);
    return check_launch("coherence gram (pairs)");
  }
  switch (precision) {
    case MR_PREC_FP32:
      return launch_gram<float, false>(z, nlines, width, nimages, idx, n_pc, mask, mask_stride, az_win, r_win,
                                       out, nullptr, s);
    case MR_PREC_FP64:
      return launch_gram<double, false>(z, nlines, width, nimages, idx, n_pc, mask, mask_stride, az_win, r_win,
                                        out, nullptr, s);
    case MR_PREC_BF16:
    case MR_PREC_BF16X3:
      return gram_tc(z, nlines, width, nimages, idx, n_pc, mask, mask_stride, az_win, r_win, out, precision, s);
    default:
      return fail(MR_ERR_INVALID, "emperical_co_pc: unknown precision %d", precision);
  }
}

// Two single-date images to the interleaved 2-date layout of the Gram kernels.
__global__ void interleave2_kernel(const float2* __restrict__ a, const float2* __restrict__ b, int64_t npix,
                                   float4* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 x = a[i], y = b[i];
    out[i] = make_float4(x.x, x.y, y.x, y.y);
  }
}

extern "C" size_t mr_ad_intf_pc_workspace_bytes(int nlines, int width) {
  return std::max<size_t>(16, (size_t)nlines * width * 2 * sizeof(float2));
}

extern "C" int mr_ad_intf_pc(const mr_complex64* ref_rslc, const mr_complex64* sec_rslc, int nlines, int width,
                             const int32_t* idx, int64_t n_pc, const uint8_t* pc_is_shp, int az_win, int r_win,
                             mr_complex64* intf, int precision, void* workspace, size_t workspace_bytes,
                             mr_stream_t stream) {
  MR_REQUIRE(n_pc >= 0, "ad_intf_pc: negative n_pc");
  if (n_pc == 0) return MR_OK;
  MR_REQUIRE(ref_rslc && sec_rslc && idx && pc_is_shp && intf, "ad_intf_pc: NULL pointer");
  MR_REQUIRE(nlines > 0 && width > 0, "ad_intf_pc: bad image shape");
  MR_REQUIRE(precision == MR_PREC_FP32 || precision == MR_PREC_FP64, "ad_intf_pc: precision must be FP32 or FP64");
  const size_t need = mr_ad_intf_pc_workspace_bytes(nlines, width);
  if (!workspace || workspace_bytes < need)
    return fail(MR_ERR_WORKSPACE, "ad_intf_pc: workspace %zu < %zu bytes", workspace_bytes, need);
  MR_REQUIRE(((uintptr_t)workspace & 15) == 0, "ad_intf_pc: workspace not 16-byte aligned");
  const int64_t npix = (int64_t)nlines * width;
  const int grid = (int)std::min<int64_t>((npix + 255) / 256, (int64_t)sm_count() * 16);
  interleave2_kernel<<<grid, 256, 0, as_stream(stream)>>>(reinterpret_cast<const float2*>(ref_rslc),
                                                          reinterpret_cast<const float2*>(sec_rslc), npix,
                                                          static_cast<float4*>(workspace));
  if (int rc = check_launch("ad_intf_pc interleave")) return rc;
  // the one pair (0, 1) of the 2-date stack: the same kernel and arithmetic as pair (0, 1)
  // of emperical_co_pc on the full stack
  return mr_emperical_co_pc(static_cast<const mr_complex64*>(workspace), nlines, width, 2, idx, n_pc, pc_is_shp, 0,
                            az_win, r_win, nullptr, 1, intf, precision, stream);
}

namespace mr {
int gram_counted(const float2* rslc, int nlines, int width, int n, const int32_t* idx, int64_t n_max,
                 const int64_t* dcount, int64_t doff, const uint8_t* mask, int az_win, int r_win, float2* coh,
                 int precision, cudaStream_t s) {
  if (n_max <= 0) return MR_OK;
  if (precision == MR_PREC_FP32)
    return launch_gram<float, false>(rslc, nlines, width, n, idx, n_max, mask, 1, az_win, r_win, coh, nullptr, s,
                                     dcount, doff);
  if (precision == MR_PREC_FP64)
    return launch_gram<double, false>(rslc, nlines, width, n, idx, n_max, mask, 1, az_win, r_win, coh, nullptr, s,
                                      dcount, doff);
  return fail(MR_ERR_UNSUPPORTED, "device-counted coherence runs in FP32 or FP64");
}
}  // namespace mr

extern "C" int mr_emperical_co(const mr_complex64* rslc, int nlines, int width, int nimages,
                               const uint8_t* is_shp, int az_win, int r_win, mr_complex64* cov,
                               mr_complex64* coh, mr_stream_t stream) {
  MR_REQUIRE(rslc && is_shp && cov && coh, "emperical_co: NULL pointer");
  MR_REQUIRE(nlines > 0 && width > 0 && nimages >= 1, "emperical_co: bad stack shape");
  MR_REQUIRE(az_win > 0 && r_win > 0 && (az_win & 1) && (r_win & 1), "emperical_co: window must be odd");
  if (nimages > MR_MAX_NIMAGES) return fail(MR_ERR_UNSUPPORTED, "emperical_co: nimages > %d", MR_MAX_NIMAGES);
  if ((int64_t)az_win * r_win > MR_MAX_WINDOW) return fail(MR_ERR_UNSUPPORTED, "emperical_co: window too large");
  return launch_gram<float, true>(reinterpret_cast<const float2*>(rslc), nlines, width, nimages, nullptr,
                                  (int64_t)nlines * width, is_shp, 1, az_win, r_win,
                                  reinterpret_cast<float2*>(coh), reinterpret_cast<float2*>(cov),
                                  as_stream(stream));
}
