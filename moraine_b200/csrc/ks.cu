// SHP identification: per-pixel sort to order-preserving keys, then the two-sample
// Kolmogorov-Smirnov merge of every pixel against its window, with the selection
// (p < p_max, per-pixel count) fused into the epilogue.
//
// Reference behaviour followed (kanglcn/moraine):
//   moraine/shp.py:36-44    merge: ties advance both indices, D*N = max |j2 - j1|
//   moraine/shp.py:20-32    p = sum_{i<=100} (-1)^(i-1) 2 exp(-2 i^2 x^2), early exit p == p_prev
//   moraine/shp.py:74-76    x = (sqrt(N/2) + 0.12 + 0.11/sqrt(N/2)) * D, p stored as float32
//   moraine/shp.py:58-72    NaN outside the image or when either pixel's last sorted value is NaN
//   moraine/shp.py:309-323  is_shp = p < p_max (float32 p against a double p_max), count
#include <atomic>
#include <cmath>
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"

namespace mr {
namespace {

constexpr uint32_t kKeyMax = 0xFFFFFFFFu;  // NaN key and merge sentinel

// Order-preserving map float -> uint32: -0 and +0 share a key (they compare equal in the
// reference merge), NaN maps above +inf (numpy.sort puts NaN last).
__device__ __forceinline__ uint32_t float_key(float f) {
  if (isnan(f)) return kKeyMax;
  uint32_t b = __float_as_uint(f);
  if (b == 0x80000000u) b = 0u;
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Global key stride of one pixel: nimages keys, then sentinels, padded to 16 bytes.
__host__ __device__ __forceinline__ int key_stride(int n) { return (n + 1 + 3) & ~3; }

// ------------------------------------------------------------------------- sort
// One warp per pixel, E keys per lane in the layout i = r*32 + lane; bitonic network
// over 32*E keys (padding keys are kKeyMax and sort last).
template <int E>
__global__ void __launch_bounds__(256) sort_keys_kernel(const float* __restrict__ rmli,
                                                        int64_t npix, int n,
                                                        uint32_t* __restrict__ keys) {
  constexpr int NP = 32 * E;
  const int lane = threadIdx.x & 31;
  const int64_t warps_total = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int ks = key_stride(n);
  for (int64_t pix = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); pix < npix;
       pix += warps_total) {
    uint32_t v[E];
    const float* src = rmli + pix * n;
#pragma unroll
    for (int r = 0; r < E; ++r) {
      int i = r * 32 + lane;
      v[r] = (i < n) ? float_key(__ldg(src + i)) : kKeyMax;
    }
#pragma unroll
    for (int k = 2; k <= NP; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        if (j >= 32) {
          const int rj = j >> 5;
#pragma unroll
          for (int r = 0; r < E; ++r) {
            if ((r & rj) == 0) {
              const int i = r * 32 + lane;
              const bool up = (i & k) == 0;
              uint32_t a = v[r], b = v[r ^ rj];
              if (up ? (a > b) : (a < b)) { v[r] = b; v[r ^ rj] = a; }
            }
          }
        } else {
#pragma unroll
          for (int r = 0; r < E; ++r) {
            const int i = r * 32 + lane;
            const bool up = (i & k) == 0;
            const bool lower = (lane & j) == 0;
            uint32_t o = __shfl_xor_sync(0xffffffffu, v[r], j);
            uint32_t mn = min(v[r], o), mx = max(v[r], o);
            v[r] = (up == lower) ? mn : mx;
          }
        }
      }
    }
    uint32_t* dst = keys + pix * ks;
#pragma unroll
    for (int r = 0; r < E; ++r) {
      int i = r * 32 + lane;
      if (i < ks) dst[i] = (i < n) ? v[r] : kKeyMax;
    }
    for (int i = NP + lane; i < ks; i += 32) dst[i] = kKeyMax;
  }
}

// ------------------------------------------------------------------------- KS merge
struct KsTable {
  float p[MR_MAX_NIMAGES + 1];
  float dist[MR_MAX_NIMAGES + 1];
  uint8_t accept[MR_MAX_NIMAGES + 1];
};

struct KsPlan {
  int th, tw, azc;  // output tile rows/cols, azimuth window offsets per chunk
  int ss;           // shared-memory words per pixel (odd: conflict-free across lanes)
  size_t smem;
};

constexpr int kKsThreads = 256;

// Keys i .. i+3 of a pixel into its shared-memory row (odd stride, so scalar stores); the
// row holds keys 0..n (key n is the sentinel).
__device__ __forceinline__ void stage4(uint32_t* dst, int i, uint4 v, int n) {
  if (i <= n) dst[i] = v.x;
  if (i + 1 <= n) dst[i + 1] = v.y;
  if (i + 2 <= n) dst[i + 2] = v.z;
  if (i + 3 <= n) dst[i + 3] = v.w;
}

__global__ void __launch_bounds__(kKsThreads) ks_merge_kernel(
    const uint32_t* __restrict__ keys, int nlines, int width, int n, int azh, int rh,
    int th, int tw, int azc, int ss, const __grid_constant__ KsTable tab, float* __restrict__ p,
    float* __restrict__ dist, uint8_t* __restrict__ is_shp, int32_t* __restrict__ shp_num) {
  extern __shared__ __align__(16) uint32_t smem[];
  const int az_win = 2 * azh + 1, r_win = 2 * rh + 1, win = az_win * r_win;
  const int nrp = th * tw;
  const int hw = tw + 2 * rh;  // halo width
  uint32_t* ref_tile = smem;                      // nrp pixels
  uint32_t* halo = smem + (size_t)nrp * ss;       // (th + azc - 1) x hw pixels
  __shared__ float s_p[MR_MAX_NIMAGES + 1];
  __shared__ float s_d[MR_MAX_NIMAGES + 1];
  __shared__ uint8_t s_acc[MR_MAX_NIMAGES + 1];
  __shared__ int s_cnt[kKsThreads];
  __shared__ uint8_t s_nan_ref[kKsThreads];

  for (int k = threadIdx.x; k <= n; k += blockDim.x) {
    s_p[k] = tab.p[k];
    s_d[k] = tab.dist[k];
    s_acc[k] = tab.accept[k];
  }
  const int ks = key_stride(n);
  const int tiles_x = (width + tw - 1) / tw;
  const int r0 = (blockIdx.x / tiles_x) * th;
  const int c0 = (blockIdx.x % tiles_x) * tw;

  // reference tile: a warp per pixel, 16-byte loads (ks is a multiple of 4), no per-key
  // index arithmetic
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int kq = ks >> 2;
  for (int rp = wid; rp < nrp; rp += nw) {
    const int r = r0 + rp / tw, c = c0 + rp % tw;
    uint32_t* dst = ref_tile + rp * ss;
    if (r < nlines && c < width) {
      const uint4* src = reinterpret_cast<const uint4*>(keys + ((int64_t)r * width + c) * ks);
      for (int q = lane; q < kq; q += 32) stage4(dst, 4 * q, __ldg(src + q), n);
    } else {
      for (int i = lane; i <= n; i += 32) dst[i] = kKeyMax;
    }
  }
  if (threadIdx.x < nrp) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  if (threadIdx.x < nrp) s_nan_ref[threadIdx.x] = (ref_tile[threadIdx.x * ss + n - 1] == kKeyMax);

  const int rp = threadIdx.x % nrp;
  const int slot = threadIdx.x / nrp, nslots = blockDim.x / nrp;
  const int rr = r0 + rp / tw, rc = c0 + rp % tw;
  const bool ref_in = (rr < nlines) && (rc < width);
  int count = 0;

  for (int z0 = 0; z0 < az_win; z0 += azc) {
    const int nz = min(azc, az_win - z0);
    const int hrows = th + nz - 1;
    __syncthreads();  // previous chunk done with the halo
    // halo rows: image rows r0 - azh + z0 .. + hrows-1, cols c0 - rh .. + hw-1
    for (int hp = wid; hp < hrows * hw; hp += nw) {
      const int r = r0 - azh + z0 + hp / hw, c = c0 - rh + hp % hw;
      uint32_t* dst = halo + hp * ss;
      if (r >= 0 && r < nlines && c >= 0 && c < width) {
        const uint4* src = reinterpret_cast<const uint4*>(keys + ((int64_t)r * width + c) * ks);
        for (int q = lane; q < kq; q += 32) stage4(dst, 4 * q, __ldg(src + q), n);
      } else {
        for (int i = lane; i <= n; i += 32) dst[i] = kKeyMax;
      }
    }
    __syncthreads();
    if (ref_in) {
      const uint32_t* A = ref_tile + rp * ss;
      const bool nan_ref = s_nan_ref[rp];
      for (int o = slot; o < nz * r_win; o += nslots) {
        const int oz = o / r_win, orr = o - oz * r_win;
        const int sr = rr - azh + z0 + oz, sc = rc - rh + orr;
        const int64_t out = ((int64_t)rr * width + rc) * win + (int64_t)(z0 + oz) * r_win + orr;
        float pv = __int_as_float(0x7fffffff), dv = pv;
        uint8_t acc = 0;
        if (sr >= 0 && sr < nlines && sc >= 0 && sc < width && !nan_ref) {
          const uint32_t* B = halo + ((rp / tw + oz) * hw + (rp % tw + orr)) * ss;
          if (B[n - 1] != kKeyMax) {
            uint32_t a = A[0], b = B[0];
            int j1 = 0, j2 = 0, kmax = 0;
            while (j1 < n && j2 < n) {
              const int le = a <= b, ge = a >= b;
              j1 += le;
              j2 += ge;
              a = A[j1];
              b = B[j2];
              kmax = max(kmax, abs(j2 - j1));
            }
            pv = s_p[kmax];
            dv = s_d[kmax];
            acc = s_acc[kmax];
          }
        }
        if (p) p[out] = pv;
        if (dist) dist[out] = dv;
        if (is_shp) is_shp[out] = acc;
        count += acc;
      }
    }
  }
  if (shp_num) {
    if (ref_in && count) atomicAdd(&s_cnt[rp], count);
    __syncthreads();
    if (threadIdx.x < nrp) {
      int r = r0 + threadIdx.x / tw, c = c0 + threadIdx.x % tw;
      if (r < nlines && c < width) shp_num[(int64_t)r * width + c] = s_cnt[threadIdx.x];
    }
  }
}

// The reference p formula (moraine/shp.py:20-32) evaluated in double with the same
// operation order, no contraction; stored as float32 like the reference's output array.
double ks_p_reference(double x) {
  const double x2 = -2.0 * x * x;
  double p = 0.0, p2 = 0.0;
  int sign = 1;
  for (int i = 1; i <= 100; ++i) {
    p += (double)(sign * 2) * std::exp(x2 * (double)i * (double)i);
    if (p == p2) return p;
    sign = -sign;
    p2 = p;
  }
  return p;
}

void fill_table(KsTable& t, int n, double p_max) {
  const double en = std::sqrt((double)n / 2.0);
  const double scale = en + 0.12 + 0.11 / en;
  for (int k = 0; k <= n; ++k) {
    const double d = std::fabs((double)k / (double)n);
    const float pf = (float)ks_p_reference(scale * d);
    t.p[k] = pf;
    t.dist[k] = (float)d;
    t.accept[k] = ((double)pf < p_max) ? 1 : 0;
  }
}

KsPlan plan_ks(int n, int azh, int rh, size_t budget = 200 * 1024) {
  const int az_win = 2 * azh + 1;
  KsPlan best{0, 0, 0, (n + 1) | 1, 0};
  double best_score = -1;
  const int tws[] = {32, 16, 8, 4, 2, 1};
  for (int tw : tws) {
    for (int th = 1; th * tw <= kKsThreads; th *= 2) {
      if (kKsThreads % (th * tw)) continue;
      for (int azc = az_win; azc >= 1; --azc) {
        size_t px = (size_t)th * tw + (size_t)(th + azc - 1) * (tw + 2 * rh);
        size_t bytes = px * best.ss * 4;
        if (bytes > budget) continue;
        // merges per loaded pixel, preferring full warps of reference pixels
        int nchunks = (az_win + azc - 1) / azc;
        double loaded = (double)th * tw + (double)nchunks * (th + azc - 1) * (tw + 2 * rh);
        double score = (double)th * tw / loaded * (th * tw >= 32 ? 1.0 : 0.5);
        if (score > best_score) {
          best_score = score;
          best.th = th; best.tw = tw; best.azc = azc; best.smem = bytes;
        }
        break;  // largest fitting azc for this (tw, th)
      }
    }
  }
  return best;
}

// ------------------------------------------------------------------------- misc
__global__ void intensity_kernel(const float2* __restrict__ z, int64_t n, float* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float2 v = z[i];
    out[i] = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
  }
}

// One warp per pixel: is_shp = (double)p < p_max, shp_num = count.
__global__ void select_shp_kernel(const float* __restrict__ p, int64_t npix, int win, double p_max,
                                  uint8_t* __restrict__ is_shp, int32_t* __restrict__ shp_num) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t pix = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); pix < npix; pix += nw) {
    int cnt = 0;
    for (int o = lane; o < win; o += 32) {
      const int64_t e = pix * win + o;
      const uint8_t s = ((double)p[e] < p_max) ? 1 : 0;
      if (is_shp) is_shp[e] = s;
      cnt += s;
    }
    cnt = warp_sum(cnt);
    if (lane == 0 && shp_num) shp_num[pix] = cnt;
  }
}

template <int E>
void launch_sort(const float* rmli, int64_t npix, int n, uint32_t* keys, cudaStream_t s) {
  int64_t blocks = (npix + 7) / 8;
  int grid = (int)std::min<int64_t>(blocks, (int64_t)sm_count() * 32);
  KernelTimer kt("ks sort keys", s);
  sort_keys_kernel<E><<<grid, 256, 0, s>>>(rmli, npix, n, keys);
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" size_t mr_ks_workspace_bytes(int nlines, int width, int nimages) {
  if (nlines <= 0 || width <= 0 || nimages <= 0) return 0;
  return (size_t)nlines * width * key_stride(nimages) * sizeof(uint32_t);
}

namespace mr {
namespace {

// Autotuned merge plans: the heuristic plans for several shared-memory budgets (large
// tiles with one CTA per SM down to small tiles with several) are timed on the first call
// for a (device, N, window, raster size class) and the fastest is kept. Each candidate is
// timed three times and ranked by its median, so that a burst of other work on the device
// (another stream of a server) does not decide the plan for good. Every plan gives the
// same results.
std::atomic<int> g_autotune{0};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, KsPlan> g_tuned;

// Raster size class: pixel counts within a factor of 4 share a tuned plan.
int size_class(int64_t npix) {
  int c = 0;
  while (npix > 3) { npix >>= 2; ++c; }
  return c;
}

std::vector<KsPlan> plan_candidates(int n, int azh, int rh) {
  std::vector<KsPlan> out;
  for (size_t budget : {200u * 1024u, 100u * 1024u, 64u * 1024u, 40u * 1024u, 28u * 1024u, 20u * 1024u}) {
    const KsPlan c = plan_ks(n, azh, rh, budget);
    if (c.th == 0) continue;
    bool dup = false;
    for (const KsPlan& o : out) dup |= (o.th == c.th && o.tw == c.tw && o.azc == c.azc);
    if (!dup) out.push_back(c);
  }
  return out;
}

int launch_merge(const KsPlan& plan, const uint32_t* keys, int nlines, int width, int n, int azh, int rh,
                 const KsTable& tab, float* p, float* dist, uint8_t* is_shp, int32_t* shp_num, cudaStream_t s) {
  if (int rc = allow_smem(reinterpret_cast<const void*>(ks_merge_kernel), plan.smem)) return rc;
  const int64_t tiles = (int64_t)((nlines + plan.th - 1) / plan.th) * ((width + plan.tw - 1) / plan.tw);
  MR_REQUIRE(tiles < (1ll << 31), "ks_test: image too large");
  KernelTimer kt("ks merge", s);
  ks_merge_kernel<<<(unsigned)tiles, kKsThreads, plan.smem, s>>>(keys, nlines, width, n, azh, rh, plan.th, plan.tw,
                                                                 plan.azc, plan.ss, tab, p, dist, is_shp, shp_num);
  return check_launch("ks_test merge");
}

// The plan for this call: tuned when asked and possible (never inside a stream capture).
int choose_plan(KsPlan& plan, const uint32_t* keys, int nlines, int width, int n, int azh, int rh,
                const KsTable& tab, float* p, float* dist, uint8_t* is_shp, int32_t* shp_num, cudaStream_t s) {
  plan = plan_ks(n, azh, rh);
  if (!g_autotune.load() || plan.th == 0) return MR_OK;
  int dev = 0;
  MR_CUDA_TRY(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, n, azh, rh, size_class((int64_t)nlines * width));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) { plan = it->second; return MR_OK; }
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  MR_CUDA_TRY(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone) return MR_OK;
  cudaEvent_t e0, e1;
  MR_CUDA_TRY(cudaEventCreate(&e0));
  MR_CUDA_TRY(cudaEventCreate(&e1));
  float best = 0.f;
  KsPlan pick = plan;
  int rc = MR_OK;
  for (const KsPlan& c : plan_candidates(n, azh, rh)) {
    if ((rc = launch_merge(c, keys, nlines, width, n, azh, rh, tab, p, dist, is_shp, shp_num, s))) break;  // warm
    float t[3] = {0.f, 0.f, 0.f};
    for (int r = 0; r < 3 && !rc; ++r) {
      cudaEventRecord(e0, s);
      if ((rc = launch_merge(c, keys, nlines, width, n, azh, rh, tab, p, dist, is_shp, shp_num, s))) break;
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) { rc = fail(MR_ERR_CUDA, "ks_test: autotune timing failed"); break; }
      cudaEventElapsedTime(&t[r], e0, e1);
    }
    if (rc) break;
    std::sort(t, t + 3);
    if (best == 0.f || t[1] < best) { best = t[1]; pick = c; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  plan = pick;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[key] = pick;
  return MR_OK;
}

}  // namespace
}  // namespace mr

extern "C" void mr_set_autotune(int on) { mr::g_autotune.store(on ? 1 : 0); }

extern "C" int mr_ks_plan(int nimages, int az_half_win, int r_half_win, int* tile_rows, int* tile_cols,
                          int* az_chunk) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  mr::KsPlan plan = mr::plan_ks(nimages, az_half_win, r_half_win);
  {
    // the tuned plan of the largest raster size class seen for this shape, if any
    std::lock_guard<std::mutex> lk(mr::g_tune_mu);
    for (const auto& kv : mr::g_tuned)
      if (std::get<0>(kv.first) == dev && std::get<1>(kv.first) == nimages && std::get<2>(kv.first) == az_half_win &&
          std::get<3>(kv.first) == r_half_win)
        plan = kv.second;
  }
  if (tile_rows) *tile_rows = plan.th;
  if (tile_cols) *tile_cols = plan.tw;
  if (az_chunk) *az_chunk = plan.azc;
  return plan.th == 0 ? MR_ERR_UNSUPPORTED : MR_OK;
}

extern "C" int mr_ks_test(const float* rmli, int nlines, int width, int nimages, int az_half_win,
                          int r_half_win, float* p, float* dist, double p_max, uint8_t* is_shp,
                          int32_t* shp_num, void* workspace, size_t workspace_bytes,
                          mr_stream_t stream) {
  MR_REQUIRE(rmli != nullptr, "ks_test: rmli is NULL");
  MR_REQUIRE(nlines > 0 && width > 0, "ks_test: empty image (%d x %d)", nlines, width);
  MR_REQUIRE(nimages >= 1, "ks_test: nimages must be >= 1 (got %d)", nimages);
  if (nimages > MR_MAX_NIMAGES)
    return fail(MR_ERR_UNSUPPORTED, "ks_test: nimages %d > %d", nimages, MR_MAX_NIMAGES);
  MR_REQUIRE(az_half_win >= 0 && r_half_win >= 0, "ks_test: negative half window");
  const int64_t win = (int64_t)(2 * az_half_win + 1) * (2 * r_half_win + 1);
  if (win > MR_MAX_WINDOW) return fail(MR_ERR_UNSUPPORTED, "ks_test: window %lld > %d", (long long)win, MR_MAX_WINDOW);
  MR_REQUIRE((is_shp == nullptr) == (shp_num == nullptr), "ks_test: is_shp and shp_num go together");
  const size_t need = mr_ks_workspace_bytes(nlines, width, nimages);
  if (workspace == nullptr || workspace_bytes < need)
    return fail(MR_ERR_WORKSPACE, "ks_test: workspace %zu < %zu bytes", workspace_bytes, need);
  MR_REQUIRE(((uintptr_t)workspace & 15) == 0, "ks_test: workspace not 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  const int64_t npix = (int64_t)nlines * width;
  uint32_t* keys = static_cast<uint32_t*>(workspace);
  if (nimages <= 32) launch_sort<1>(rmli, npix, nimages, keys, s);
  else if (nimages <= 64) launch_sort<2>(rmli, npix, nimages, keys, s);
  else if (nimages <= 128) launch_sort<4>(rmli, npix, nimages, keys, s);
  else if (nimages <= 256) launch_sort<8>(rmli, npix, nimages, keys, s);
  else launch_sort<16>(rmli, npix, nimages, keys, s);
  if (int rc = check_launch("ks_test sort")) return rc;
  if (!p && !dist && !is_shp) return MR_OK;

  // host staging of the table; the launch copies it into the kernel's parameter buffer
  static thread_local KsTable tab_local;
  fill_table(tab_local, nimages, p_max);
  KsPlan plan;
  if (int rc = choose_plan(plan, keys, nlines, width, nimages, az_half_win, r_half_win, tab_local, p, dist, is_shp,
                           shp_num, s))
    return rc;
  if (plan.th == 0)
    return fail(MR_ERR_UNSUPPORTED, "ks_test: nimages %d with half windows (%d, %d) does not fit shared memory",
                nimages, az_half_win, r_half_win);
  return launch_merge(plan, keys, nlines, width, nimages, az_half_win, r_half_win, tab_local, p, dist, is_shp,
                      shp_num, s);
}

extern "C" int mr_select_shp(const float* p, int64_t npix, int win, double p_max, uint8_t* is_shp,
                             int32_t* shp_num, mr_stream_t stream) {
  MR_REQUIRE(p != nullptr, "select_shp: p is NULL");
  MR_REQUIRE(npix >= 0 && win > 0, "select_shp: bad shape");
  if (npix == 0) return MR_OK;
  int64_t blocks = (npix + 7) / 8;
  int grid = (int)std::min<int64_t>(blocks, (int64_t)sm_count() * 16);
  select_shp_kernel<<<grid, 256, 0, as_stream(stream)>>>(p, npix, win, p_max, is_shp, shp_num);
  return check_launch("select_shp");
}

extern "C" int mr_intensity(const mr_complex64* rslc, int64_t n, float* rmli, mr_stream_t stream) {
  MR_REQUIRE(rslc && rmli, "intensity: NULL pointer");
  if (n <= 0) return MR_OK;
  int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 16);
  intensity_kernel<<<grid, 256, 0, as_stream(stream)>>>(reinterpret_cast<const float2*>(rslc), n, rmli);
  return check_launch("intensity");
}
