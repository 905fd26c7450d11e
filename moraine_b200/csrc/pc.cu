// Raster <-> point-cloud gathers and scatters by grid index (gix: (n, 2) int32 rows of
// (line, pixel)).
//
// Replace moraine.pc.ras2pc (moraine/pc.py:239-241, ras[gix[:, 0], gix[:, 1]]) and
// moraine.pc.pc2ras (moraine/pc.py:223-236, a NaN-filled raster with pc_data scattered at
// gix), the glue on either side of the DS chain: rasters of per-pixel records (a record is
// the trailing dimensions of the array, any element type, elem_bytes long) in and out of
// (n, record) point clouds. Indices follow numpy's rules: -lines <= line < lines (negative
// ones count from the end), the same for pixels; an index outside that range sets the error
// word (1) and its point is skipped, so the host can raise IndexError as numpy does.
//
// One warp per point, lanes over the record in the widest word that the record size and
// both base addresses allow (16, 8, 4 or 1 bytes): each point's record moves as one
// coalesced run.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace mr {
namespace {

__device__ __forceinline__ bool resolve(int32_t line, int32_t pixel, int64_t nlines, int64_t width, int64_t& cell) {
  int64_t l = line, p = pixel;
  if (l < 0) l += nlines;
  if (p < 0) p += width;
  if (l < 0 || l >= nlines || p < 0 || p >= width) return false;
  cell = l * width + p;
  return true;
}

// kScatter false: out[i] = ras[gix[i]]; true: ras[gix[i]] = pc[i]
template <typename W, bool kScatter>
__global__ void gix_copy_kernel(const unsigned char* __restrict__ src, unsigned char* __restrict__ dst,
                                const int32_t* __restrict__ gix, int64_t n, int64_t nlines, int64_t width,
                                int64_t words, int* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
    int64_t cell;
    if (!resolve(gix[2 * i], gix[2 * i + 1], nlines, width, cell)) {
      if (lane == 0) atomicExch(err, 1);
      continue;
    }
    const W* s = reinterpret_cast<const W*>(src) + (kScatter ? i : cell) * words;
    W* d = reinterpret_cast<W*>(dst) + (kScatter ? cell : i) * words;
    for (int64_t w = lane; w < words; w += 32) d[w] = s[w];
  }
}

// Every record of the raster set to the fill pattern (fill_bytes long, repeated).
template <typename W>
__global__ void fill_kernel(W* __restrict__ ras, int64_t nwords, W pattern0, W pattern1, int period) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += (int64_t)gridDim.x * blockDim.x)
    ras[i] = (period == 2 && (i & 1)) ? pattern1 : pattern0;
}

int word_bytes(uintptr_t a, uintptr_t b, int64_t elem_bytes) {
  for (int w : {16, 8, 4}) {
    if (elem_bytes % w == 0 && a % w == 0 && b % w == 0) return w;
  }
  return 1;
}

int warp_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, (int64_t)sm_count() * 32));
}

template <bool kScatter>
void launch_copy(int wb, const void* src, void* dst, const int32_t* gix, int64_t n, int64_t nlines, int64_t width,
                 int64_t elem_bytes, int* err, cudaStream_t s) {
  const auto* a = static_cast<const unsigned char*>(src);
  auto* b = static_cast<unsigned char*>(dst);
  const int g = warp_grid(n);
  const int64_t words = elem_bytes / wb;
  switch (wb) {
    case 16: gix_copy_kernel<uint4, kScatter><<<g, 256, 0, s>>>(a, b, gix, n, nlines, width, words, err); break;
    case 8: gix_copy_kernel<uint2, kScatter><<<g, 256, 0, s>>>(a, b, gix, n, nlines, width, words, err); break;
    case 4: gix_copy_kernel<uint32_t, kScatter><<<g, 256, 0, s>>>(a, b, gix, n, nlines, width, words, err); break;
    default: gix_copy_kernel<uint8_t, kScatter><<<g, 256, 0, s>>>(a, b, gix, n, nlines, width, words, err); break;
  }
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" int mr_ras2pc(const void* ras, int64_t nlines, int64_t width, int64_t elem_bytes, const int32_t* gix,
                         int64_t n, void* pc, int* err, mr_stream_t stream) {
  MR_REQUIRE(nlines >= 0 && width >= 0 && elem_bytes > 0 && n >= 0, "ras2pc: bad shape");
  if (n == 0) return MR_OK;
  MR_REQUIRE(ras && gix && pc && err, "ras2pc: NULL pointer");
  MR_REQUIRE(((uintptr_t)gix & 3) == 0 && ((uintptr_t)err & 3) == 0, "ras2pc: gix or err not 4-byte aligned");
  const int wb = word_bytes((uintptr_t)ras, (uintptr_t)pc, elem_bytes);
  launch_copy<false>(wb, ras, pc, gix, n, nlines, width, elem_bytes, err, as_stream(stream));
  return check_launch("ras2pc");
}

extern "C" int mr_pc2ras(const void* pc, const int32_t* gix, int64_t n, int64_t nlines, int64_t width,
                         int64_t elem_bytes, const void* fill, int fill_bytes, void* ras, int* err,
                         mr_stream_t stream) {
  MR_REQUIRE(nlines >= 0 && width >= 0 && elem_bytes > 0 && n >= 0, "pc2ras: bad shape");
  MR_REQUIRE(fill_bytes == 0 || fill_bytes == 4 || fill_bytes == 8 || fill_bytes == 16,
             "pc2ras: fill_bytes must be 0, 4, 8 or 16");
  MR_REQUIRE(fill_bytes == 0 || elem_bytes % fill_bytes == 0, "pc2ras: record of %lld bytes is not a whole number "
             "of %d-byte fill patterns", (long long)elem_bytes, fill_bytes);
  cudaStream_t s = as_stream(stream);
  const int64_t cells = nlines * width;
  int launches = 0;
  if (fill_bytes && cells) {
    MR_REQUIRE(ras && fill, "pc2ras: NULL pointer");
    MR_REQUIRE(((uintptr_t)ras % fill_bytes) == 0, "pc2ras: raster not %d-byte aligned", fill_bytes);
    uint64_t pat[2] = {0, 0};
    std::memcpy(pat, fill, (size_t)fill_bytes);
    const int64_t total = cells * elem_bytes;
    const int64_t blocks = (total / fill_bytes + 255) / 256;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)sm_count() * 16));
    if (fill_bytes == 4) {
      fill_kernel<uint32_t><<<grid, 256, 0, s>>>(static_cast<uint32_t*>(ras), total / 4, (uint32_t)pat[0], 0u, 1);
    } else if (fill_bytes == 8) {
      fill_kernel<uint64_t><<<grid, 256, 0, s>>>(static_cast<uint64_t*>(ras), total / 8, pat[0], 0ull, 1);
    } else {
      fill_kernel<uint64_t><<<grid, 256, 0, s>>>(static_cast<uint64_t*>(ras), total / 8, pat[0], pat[1], 2);
    }
    ++launches;
  }
  if (n) {
    MR_REQUIRE(pc && gix && ras && err, "pc2ras: NULL pointer");
    MR_REQUIRE(((uintptr_t)gix & 3) == 0 && ((uintptr_t)err & 3) == 0, "pc2ras: gix or err not 4-byte aligned");
    const int wb = word_bytes((uintptr_t)pc, (uintptr_t)ras, elem_bytes);
    launch_copy<true>(wb, pc, ras, gix, n, nlines, width, elem_bytes, err, s);
    ++launches;
  }
  return launches ? check_launch("pc2ras", launches) : MR_OK;
}
