// Coherence Gram on the 5th-generation tensor cores (tcgen05, sm_100a), BF16 inputs with
// FP32 accumulation in tensor memory.
//
// Per point the SHP samples Z (S x N complex) are re-read as a real matrix with 2N
// features, the real and imaginary parts of image m at features 2m and 2m+1. The real
// Gram G = X^T X (2N x 2N, accumulated in TMEM) contains the complex Gram:
//   Re sum_s z_m conj(z_j) = G[2m][2j] + G[2m+1][2j+1],
//   Im sum_s z_m conj(z_j) = G[2m+1][2j] - G[2m][2j+1].
// X is staged K-major (K = SHP index) in the canonical no-swizzle core-matrix layout
// (8 feature rows x 16 bytes per core matrix), so the same shared-memory buffer is both
// MMA operands (A = X^T, B = X). With the hi/lo split (MR_PREC_BF16X3) every value is
// hi + lo, hi = bf16(x), lo = bf16(x - hi), and G ~ hi^T hi + hi^T lo + lo^T hi, which
// carries FP32-level accuracy; MR_PREC_BF16 uses hi^T hi only. The amplitude sums
// sum_s |z_m|^2 are accumulated in FP32 on the CUDA cores in a fixed order.
//
// Reference behaviour followed (kanglcn/moraine): moraine/co.py:164-187 (coherence of each
// pair over the in-image SHPs, window order), moraine/co.py:230-266 (point-cloud layout).
//
// One CTA of 128 threads per point (persistent over points). K is processed in chunks of
// 64 SHPs, double-buffered: the gather of chunk c+1 overlaps the MMAs of chunk c, whose
// completion is signalled by tcgen05.commit on an mbarrier. Every mbarrier wait is bounded;
// a wait that runs out marks the point's coherence NaN and the CTA stops after freeing its
// tensor memory.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"

namespace mr {
namespace {

constexpr int kTcThreads = 128;
constexpr int kKc = 64;                  // SHP rows (K) per chunk
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, K-major, no swizzle: LBO = byte distance between the two
// 8-element K halves of an MMA, SBO = byte distance between groups of 8 rows (sm100 layout
// version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;               // base offset 0, legacy LBO mode, SWIZZLE_NONE
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> F32, both operands K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4)                        // D format F32
         | (1u << 7)                      // A format BF16
         | (1u << 10)                     // B format BF16
         | ((uint32_t)(n >> 3) << 17)     // N / 8
         | ((uint32_t)(m >> 4) << 24);    // M / 16
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Block-wide compaction of the window mask into the pixel indices of the in-image SHPs,
// in window order; returns the count.
__device__ int tc_collect(const uint8_t* __restrict__ m, int az_win, int r_win, int ra, int rr, int nlines, int width,
                          int* __restrict__ s_pos, int* __restrict__ s_tmp) {
  const int win = az_win * r_win, azh = az_win / 2, rh = r_win / 2;
  const int per = (win + blockDim.x - 1) / blockDim.x;
  const int e0 = threadIdx.x * per, e1 = min(win, e0 + per);
  int c = 0;
  for (int e = e0; e < e1; ++e) {
    const int k = e / r_win, l = e - k * r_win, sa = ra - azh + k, sr = rr - rh + l;
    c += (m[e] && sa >= 0 && sa < nlines && sr >= 0 && sr < width);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s_tmp[wid] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { const int t = s_tmp[w]; s_tmp[w] = run; run += t; }
    s_tmp[8] = run;
  }
  __syncthreads();
  int pos = s_tmp[wid] + incl - c;
  for (int e = e0; e < e1; ++e) {
    const int k = e / r_win, l = e - k * r_win, sa = ra - azh + k, sr = rr - rh + l;
    if (m[e] && sa >= 0 && sa < nlines && sr >= 0 && sr < width) s_pos[pos++] = sa * width + sr;
  }
  __syncthreads();
  const int total = s_tmp[8];
  __syncthreads();
  return total;
}

struct TcLayout {
  int mt;          // 128-row M tiles
  int rows;        // 128 * mt feature rows staged
  int fn;          // MMA N (features rounded up to 16)
  size_t buf;      // bytes of one operand buffer (rows x kKc bf16)
  size_t off_pos, off_part, off_amp, off_bar, bytes;
  int items;       // gather items per chunk: n images x kKc/8 k-groups
  int ncols;       // TMEM columns allocated
};

__host__ __device__ inline TcLayout tc_layout(int n, int win) {
  TcLayout l;
  const int f = 2 * n;
  l.mt = (f + 127) / 128;
  l.rows = 128 * l.mt;
  l.fn = (f + 15) & ~15;
  l.buf = (size_t)l.rows * kKc * 2;
  l.items = n * (kKc / 8);
  l.off_pos = 4 * l.buf;  // [stage 0 hi, stage 0 lo, stage 1 hi, stage 1 lo]
  l.off_part = l.off_pos + (((size_t)win * 4 + 15) & ~(size_t)15);
  l.off_amp = l.off_part + (((size_t)l.items * 4 + 15) & ~(size_t)15);
  l.off_bar = l.off_amp + (((size_t)n * 4 + 15) & ~(size_t)15);
  l.bytes = l.off_bar + 64;
  l.ncols = l.mt == 1 ? 128 : 512;
  return l;
}

template <bool kSplit>
__global__ void __launch_bounds__(kTcThreads, 1) gram_tc_kernel(
    const float2* __restrict__ rslc, int nlines, int width, int n, const int32_t* __restrict__ idx, int64_t n_pc,
    const uint8_t* __restrict__ mask, int mask_stride, int az_win, int r_win, float2* __restrict__ coh) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ int s_tmp[9];
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  const int win = az_win * r_win;
  const TcLayout L = tc_layout(n, win);
  const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
  int* s_pos = reinterpret_cast<int*>(smem + L.off_pos);
  float* s_part = reinterpret_cast<float*>(smem + L.off_part);
  float* s_amp = reinterpret_cast<float*>(smem + L.off_amp);
  uint64_t* s_bar = reinterpret_cast<uint64_t*>(smem + L.off_bar);
  const uint32_t bar0 = smem_u32(&s_bar[0]), bar1 = smem_u32(&s_bar[1]);
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const uint32_t sbo = kKc / 8 * 128;  // 8 feature rows x all k groups of a chunk
  const uint32_t idesc = umma_idesc_bf16(128, L.fn);
  const float fnan = __int_as_float(0x7fffffff);

  if (wid == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(L.ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1));
    s_fail = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  uint32_t phase0 = 0, phase1 = 0;
  bool pend0 = false, pend1 = false;

  for (int64_t pt = blockIdx.x; pt < n_pc; pt += gridDim.x) {
    int ra, rr;
    if (idx) { ra = idx[2 * pt]; rr = idx[2 * pt + 1]; }
    else { ra = (int)(pt / width); rr = (int)(pt % width); }
    if (ra < 0 || ra >= nlines || rr < 0 || rr >= width) {
      for (int64_t e = tid; e < npairs; e += kTcThreads) coh[pt * npairs + e] = make_float2(fnan, fnan);
      continue;
    }
    const uint8_t* m = mask + (mask_stride ? ((int64_t)ra * width + rr) : pt) * win;
    const int S = tc_collect(m, az_win, r_win, ra, rr, nlines, width, s_pos, s_tmp);
    const int nch = max(1, (S + kKc - 1) / kKc);
    float part[8];  // FP32 amplitude partials of this thread's gather items (fixed order)
#pragma unroll
    for (int j = 0; j < 8; ++j) part[j] = 0.f;
    for (int ch = 0; ch < nch; ++ch) {
      const int st = ch & 1;
      // the buffers of this stage are free once the MMAs that read them completed
      if (st == 0 && pend0) {
        if (!mbar_wait(bar0, phase0)) s_fail = 1;
        phase0 ^= 1; pend0 = false;
      }
      if (st == 1 && pend1) {
        if (!mbar_wait(bar1, phase1)) s_fail = 1;
        phase1 ^= 1; pend1 = false;
      }
      unsigned char* hi = smem + (size_t)(2 * st) * L.buf;
      unsigned char* lo = hi + L.buf;
      // gather: item w = kg * n + mi covers image mi, SHPs ch*kKc + 8kg .. +7
#pragma unroll 1
      for (int j = 0, w = tid; w < L.items; ++j, w += kTcThreads) {
        const int kg = w / n, mi = w - kg * n;
        uint32_t hr[4], hm[4], lr[4], lm[4];
        float a2 = 0.f;
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
          float2 z0 = make_float2(0.f, 0.f), z1 = z0;
          const int k0 = ch * kKc + kg * 8 + e;
          if (k0 < S) z0 = rslc[(int64_t)s_pos[k0] * n + mi];
          if (k0 + 1 < S) z1 = rslc[(int64_t)s_pos[k0 + 1] * n + mi];
          a2 += z0.x * z0.x + z0.y * z0.y;
          a2 += z1.x * z1.x + z1.y * z1.y;
          const __nv_bfloat162 h_re = __floats2bfloat162_rn(z0.x, z1.x);
          const __nv_bfloat162 h_im = __floats2bfloat162_rn(z0.y, z1.y);
          hr[e / 2] = *reinterpret_cast<const uint32_t*>(&h_re);
          hm[e / 2] = *reinterpret_cast<const uint32_t*>(&h_im);
          if (kSplit) {
            const float2 fre = __bfloat1622float2(h_re), fim = __bfloat1622float2(h_im);
            const __nv_bfloat162 l_re = __floats2bfloat162_rn(z0.x - fre.x, z1.x - fre.y);
            const __nv_bfloat162 l_im = __floats2bfloat162_rn(z0.y - fim.x, z1.y - fim.y);
            lr[e / 2] = *reinterpret_cast<const uint32_t*>(&l_re);
            lm[e / 2] = *reinterpret_cast<const uint32_t*>(&l_im);
          }
        }
        if (j < 8) part[j] += a2;
        const int f = 2 * mi;  // real part at feature f, imaginary at f + 1
        const size_t o_re = (size_t)(f >> 3) * sbo + (size_t)kg * 128 + (size_t)(f & 7) * 16;
        const size_t o_im = (size_t)((f + 1) >> 3) * sbo + (size_t)kg * 128 + (size_t)((f + 1) & 7) * 16;
        *reinterpret_cast<uint4*>(hi + o_re) = make_uint4(hr[0], hr[1], hr[2], hr[3]);
        *reinterpret_cast<uint4*>(hi + o_im) = make_uint4(hm[0], hm[1], hm[2], hm[3]);
        if (kSplit) {
          *reinterpret_cast<uint4*>(lo + o_re) = make_uint4(lr[0], lr[1], lr[2], lr[3]);
          *reinterpret_cast<uint4*>(lo + o_im) = make_uint4(lm[0], lm[1], lm[2], lm[3]);
        }
      }
      fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t a_hi = smem_u32(hi), a_lo = smem_u32(lo);
        for (int t = 0; t < L.mt; ++t) {
          const uint32_t d = tmem + (uint32_t)(t * 256);
          const uint32_t toff = (uint32_t)(t * 16) * sbo;  // 128 rows = 16 groups of 8
          for (int ks = 0; ks < kKc / 16; ++ks) {
            const uint32_t koff = (uint32_t)ks * 256;      // 16 k = two 16-byte core columns
            const uint64_t dah = umma_desc(a_hi + toff + koff, 128, sbo);
            const uint64_t dbh = umma_desc(a_hi + koff, 128, sbo);
            const uint32_t acc = (ch > 0 || ks > 0) ? 1u : 0u;
            umma_bf16(d, dah, dbh, idesc, acc);
            if (kSplit) {
              const uint64_t dal = umma_desc(a_lo + toff + koff, 128, sbo);
              const uint64_t dbl = umma_desc(a_lo + koff, 128, sbo);
              umma_bf16(d, dah, dbl, idesc, 1u);
              umma_bf16(d, dal, dbh, idesc, 1u);
            }
          }
        }
        umma_commit(st == 0 ? bar0 : bar1);
      }
      if (st == 0) pend0 = true; else pend1 = true;
    }
    // all MMAs of this point done
    if (pend0) { if (!mbar_wait(bar0, phase0)) s_fail = 1; phase0 ^= 1; pend0 = false; }
    if (pend1) { if (!mbar_wait(bar1, phase1)) s_fail = 1; phase1 ^= 1; pend1 = false; }
    tc_fence_after();
    // amplitude sums: items of image mi are w = kg * n + mi, reduced in kg order
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int w = tid + j * kTcThreads;
      if (w < L.items) s_part[w] = part[j];
    }
    __syncthreads();
    for (int mi = tid; mi < n; mi += kTcThreads) {
      float a = 0.f;
      for (int kg = 0; kg < kKc / 8; ++kg) a += s_part[kg * n + mi];
      s_amp[mi] = a;
    }
    __syncthreads();
    const bool failed = s_fail != 0;
    // epilogue: thread t reads TMEM lane t (feature row 128 T + t) of its warp's quarter
    float2* out = coh + pt * npairs;
    for (int t = 0; t < L.mt; ++t) {
      const int f = 128 * t + tid;
      const int mi = f >> 1;
      const bool even = (f & 1) == 0, valid = f < 2 * n;
      for (int cc = 0; cc * 32 < L.fn; ++cc) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(32 * wid) << 16) + (uint32_t)(t * 256 + cc * 32), v);
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const float a = v[2 * e], b = v[2 * e + 1];          // G[f][2j], G[f][2j+1]
          const float pa = __shfl_xor_sync(0xffffffffu, a, 1);  // G[f^1][2j]
          const float pb = __shfl_xor_sync(0xffffffffu, b, 1);  // G[f^1][2j+1]
          const int jj = cc * 16 + e;
          if (even && valid && jj > mi && jj < n) {
            const float re = a + pb, im = pa - b;
            const float den = sqrtf(s_amp[mi] * s_amp[jj]);
            float2 o = make_float2(re / den, im / den);
            if (failed) o = make_float2(fnan, fnan);
            out[triu_index(mi, jj, n)] = o;
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    if (failed) break;
  }
  __syncthreads();
  if (wid == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L.ncols));
}

}  // namespace

// Tensor-core Gram. Supports nimages <= 128 (two 128-row tiles of 2N features).
int gram_tc(const float2* rslc, int nlines, int width, int n, const int32_t* idx, int64_t n_pc, const uint8_t* mask,
            int mask_stride, int az_win, int r_win, float2* coh, int precision, cudaStream_t s) {
  if (n > 128) return fail(MR_ERR_UNSUPPORTED, "emperical_co_pc: tensor-core precision supports nimages <= 128");
  const TcLayout L = tc_layout(n, az_win * r_win);
  if (L.bytes > 200 * 1024) return fail(MR_ERR_UNSUPPORTED, "emperical_co_pc: window too large for the tensor-core Gram");
  const bool split = precision == MR_PREC_BF16X3;
  auto kern = split ? gram_tc_kernel<true> : gram_tc_kernel<false>;
  if (int rc_ = allow_smem(reinterpret_cast<const void*>(kern), (size_t)(L.bytes))) return rc_;
  // one CTA per SM when it claims all 512 TMEM columns, up to four with 128 columns each
  int occ = 0;
  MR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kTcThreads, L.bytes));
  occ = std::max(1, std::min(occ, 512 / L.ncols));
  const int64_t grid = std::min<int64_t>(n_pc, (int64_t)sm_count() * occ);
  KernelTimer kt(split ? "gram tc bf16x3" : "gram tc bf16", s);
  kern<<<(unsigned)grid, kTcThreads, L.bytes, s>>>(rslc, nlines, width, n, idx, n_pc, mask, mask_stride, az_win,
                                                   r_win, coh);
  return check_launch("coherence gram (tensor cores)");
}

}  // namespace mr
