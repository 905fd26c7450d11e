// The whole DS chain behind one C-ABI call: intensity or amplitude -> KS test + SHP selection -> DS
// extraction -> [coherence -> EMI + temporal coherence] per batch of DS points.
//
// The production caller of the kernels for hosts that bind the library directly (no
// Python): it replaces the reference's file-based stage drivers (moraine/cli/shp.py:33,
// moraine/cli/co.py:33, moraine/cli/pl.py:223) for one tile resident in device memory.
// Every intermediate stays in the caller's workspace. mr_ds_chain synchronises the stream
// once, to read the number of DS points that sizes the batch loop; mr_ds_chain_async keeps
// that count on the device (the kernels clamp to it) so that the call can be captured in a
// CUDA graph.
#include <algorithm>

#include "common.cuh"

namespace mr {
namespace {

struct ChainWs {
  float* rmli;
  unsigned char* ks;
  uint8_t* is_shp;
  int32_t* shp_num;
  unsigned char* ex;
  int64_t* n_ds;
  float2* coh;
  unsigned char* emi;
  size_t ks_bytes, ex_bytes, emi_bytes, total;
};

ChainWs layout(unsigned char* base, int nlines, int width, int n, int win, int64_t batch) {
  const int64_t npix = (int64_t)nlines * width;
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  ChainWs w{};
  w.ks_bytes = mr_ks_workspace_bytes(nlines, width, n);
  w.ex_bytes = mr_ds_extract_workspace_bytes(npix);
  w.emi_bytes = mr_emi_workspace_bytes(batch, n);
  auto a16 = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t o = 0;
  auto take = [&](size_t bytes) { unsigned char* p = base ? base + o : nullptr; o += a16(bytes); return p; };
  w.rmli = reinterpret_cast<float*>(take((size_t)npix * n * sizeof(float)));
  w.ks = take(w.ks_bytes);
  w.is_shp = take((size_t)npix * win);
  w.shp_num = reinterpret_cast<int32_t*>(take((size_t)npix * sizeof(int32_t)));
  w.ex = take(w.ex_bytes);
  w.n_ds = reinterpret_cast<int64_t*>(take(sizeof(int64_t)));
  w.coh = reinterpret_cast<float2*>(take((size_t)batch * npairs * sizeof(float2)));
  w.emi = take(w.emi_bytes);
  w.total = o;
  return w;
}

// The rmli the KS test reads: |z|^2 (the API notebooks) or |z| (the CLI's rslc2amp).
int ks_prologue(const mr_complex64* rslc, int64_t n, int ks_input, float* rmli, mr_stream_t stream) {
  if (ks_input == MR_KS_INTENSITY) return mr_intensity(rslc, n, rmli, stream);
  if (ks_input == MR_KS_AMPLITUDE) return mr_rslc2amp(rslc, n, rmli, stream);
  return fail(MR_ERR_INVALID, "ds_chain: ks_input %d is neither MR_KS_INTENSITY nor MR_KS_AMPLITUDE", ks_input);
}

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" size_t mr_ds_chain_workspace_bytes(int nlines, int width, int nimages, int az_half_win, int r_half_win,
                                              int64_t batch) {
  if (nlines <= 0 || width <= 0 || nimages < 2 || az_half_win < 0 || r_half_win < 0 || batch <= 0) return 0;
  const int win = (2 * az_half_win + 1) * (2 * r_half_win + 1);
  return layout(nullptr, nlines, width, nimages, win, batch).total;
}

extern "C" int mr_ds_chain(const mr_complex64* rslc, int nlines, int width, int nimages, int az_half_win,
                           int r_half_win, int ks_input, double p_max, int min_shp, int gram_precision,
                           int emi_precision, int32_t* idx, mr_complex64* ph, float* quality, float* t_coh,
                           int64_t max_ds, int64_t* n_ds, int64_t batch, void* workspace, size_t workspace_bytes,
                           mr_stream_t stream) {
  MR_REQUIRE(rslc && idx && ph && quality && t_coh && n_ds, "ds_chain: NULL pointer");
  MR_REQUIRE(nlines > 0 && width > 0 && nimages >= 2, "ds_chain: bad stack shape");
  MR_REQUIRE(az_half_win >= 0 && r_half_win >= 0, "ds_chain: negative half window");
  MR_REQUIRE(batch > 0 && max_ds >= 0, "ds_chain: batch must be > 0 and max_ds >= 0");
  MR_REQUIRE(emi_precision == MR_PREC_FP32 || emi_precision == MR_PREC_FP64 || emi_precision == MR_PREC_MIXED ||
                 emi_precision == MR_PREC_REFINE,
             "ds_chain: emi_precision must be FP32, FP64, MIXED or REFINE");
  const int az_win = 2 * az_half_win + 1, r_win = 2 * r_half_win + 1, win = az_win * r_win;
  const size_t need = mr_ds_chain_workspace_bytes(nlines, width, nimages, az_half_win, r_half_win, batch);
  if (!workspace || workspace_bytes < need)
    return fail(MR_ERR_WORKSPACE, "ds_chain: workspace %zu < %zu bytes", workspace_bytes, need);
  MR_REQUIRE(((uintptr_t)workspace & 255) == 0, "ds_chain: workspace not 256-byte aligned");
  const ChainWs w = layout(static_cast<unsigned char*>(workspace), nlines, width, nimages, win, batch);
  const int64_t npix = (int64_t)nlines * width;
  const int64_t npairs = (int64_t)nimages * (nimages - 1) / 2;
  cudaStream_t s = as_stream(stream);
  *n_ds = 0;
  if (int rc = ks_prologue(rslc, npix * nimages, ks_input, w.rmli, stream)) return rc;
  if (int rc = mr_ks_test(w.rmli, nlines, width, nimages, az_half_win, r_half_win, nullptr, nullptr, p_max, w.is_shp,
                          w.shp_num, w.ks, w.ks_bytes, stream))
    return rc;
  if (int rc = mr_ds_extract(w.shp_num, nullptr, nlines, width, win, min_shp, idx, nullptr, max_ds, w.n_ds, w.ex,
                             w.ex_bytes, stream))
    return rc;
  int64_t count = 0;
  MR_CUDA_TRY(cudaMemcpyAsync(&count, w.n_ds, sizeof(count), cudaMemcpyDeviceToHost, s));
  MR_CUDA_TRY(cudaStreamSynchronize(s));
  if (count > max_ds) return fail(MR_ERR_INVALID, "ds_chain: %lld DS points > max_ds %lld", (long long)count,
                                  (long long)max_ds);
  *n_ds = count;
  for (int64_t b0 = 0; b0 < count; b0 += batch) {
    const int64_t nb = std::min<int64_t>(batch, count - b0);
    if (int rc = mr_emperical_co_pc(rslc, nlines, width, nimages, idx + 2 * b0, nb, w.is_shp, 1, az_win, r_win,
                                    nullptr, (int)npairs, reinterpret_cast<mr_complex64*>(w.coh), gram_precision,
                                    stream))
      return rc;
    const mr_complex64* c = reinterpret_cast<const mr_complex64*>(w.coh);
    const int rc = emi_precision == MR_PREC_MIXED
                       ? mr_emi_routed(c, nb, nimages, 0, MR_EMI_COND_MAX, ph + b0 * nimages, quality + b0,
                                       t_coh + b0, nullptr, w.emi, w.emi_bytes, stream)
                       : mr_emi(c, nb, nimages, 0, emi_precision, ph + b0 * nimages, quality + b0, t_coh + b0, w.emi,
                                w.emi_bytes, stream);
    if (rc) return rc;
  }
  return MR_OK;
}

extern "C" int mr_ds_chain_async(const mr_complex64* rslc, int nlines, int width, int nimages, int az_half_win,
                                 int r_half_win, int ks_input, double p_max, int min_shp, int gram_precision,
                                 int emi_precision, int32_t* idx, mr_complex64* ph, float* quality, float* t_coh,
                                 int64_t max_ds, int64_t* n_ds_dev, int64_t batch, void* workspace,
                                 size_t workspace_bytes, mr_stream_t stream) {
  MR_REQUIRE(rslc && idx && ph && quality && t_coh && n_ds_dev, "ds_chain_async: NULL pointer");
  MR_REQUIRE(nlines > 0 && width > 0 && nimages >= 2, "ds_chain_async: bad stack shape");
  MR_REQUIRE(az_half_win >= 0 && r_half_win >= 0, "ds_chain_async: negative half window");
  MR_REQUIRE(batch > 0 && max_ds >= 0, "ds_chain_async: batch must be > 0 and max_ds >= 0");
  if (nimages > 128)
    return fail(MR_ERR_UNSUPPORTED, "ds_chain_async: nimages %d > 128 (use mr_ds_chain)", nimages);
  if ((gram_precision != MR_PREC_FP32 && gram_precision != MR_PREC_FP64) ||
      (emi_precision != MR_PREC_FP32 && emi_precision != MR_PREC_FP64 && emi_precision != MR_PREC_REFINE))
    return fail(MR_ERR_UNSUPPORTED, "ds_chain_async: gram precision must be FP32 or FP64, emi FP32, FP64 or REFINE");
  const int az_win = 2 * az_half_win + 1, r_win = 2 * r_half_win + 1, win = az_win * r_win;
  const size_t need = mr_ds_chain_workspace_bytes(nlines, width, nimages, az_half_win, r_half_win, batch);
  if (!workspace || workspace_bytes < need)
    return fail(MR_ERR_WORKSPACE, "ds_chain_async: workspace %zu < %zu bytes", workspace_bytes, need);
  MR_REQUIRE(((uintptr_t)workspace & 255) == 0, "ds_chain_async: workspace not 256-byte aligned");
  const ChainWs w = layout(static_cast<unsigned char*>(workspace), nlines, width, nimages, win, batch);
  const int64_t npix = (int64_t)nlines * width;
  const int64_t npairs = (int64_t)nimages * (nimages - 1) / 2;
  cudaStream_t s = as_stream(stream);
  if (int rc = ks_prologue(rslc, npix * nimages, ks_input, w.rmli, stream)) return rc;
  if (int rc = mr_ks_test(w.rmli, nlines, width, nimages, az_half_win, r_half_win, nullptr, nullptr, p_max, w.is_shp,
                          w.shp_num, w.ks, w.ks_bytes, stream))
    return rc;
  if (int rc = mr_ds_extract(w.shp_num, nullptr, nlines, width, win, min_shp, idx, nullptr, max_ds, n_ds_dev, w.ex,
                             w.ex_bytes, stream))
    return rc;
  // every batch that max_ds allows; the kernels read the DS count and skip what is past it
  for (int64_t b0 = 0; b0 < max_ds; b0 += batch) {
    const int64_t nb = std::min<int64_t>(batch, max_ds - b0);
    if (int rc = gram_counted(reinterpret_cast<const float2*>(rslc), nlines, width, nimages, idx + 2 * b0, nb,
                              n_ds_dev, b0, w.is_shp, az_win, r_win, w.coh, gram_precision, s))
      return rc;
    if (int rc = emi_counted(w.coh, nb, n_ds_dev, b0, nimages, emi_precision,
                             reinterpret_cast<float2*>(ph) + b0 * nimages, quality + b0, t_coh + b0, w.emi,
                             w.emi_bytes, s))
      return rc;
  }
  (void)npairs;
  return MR_OK;
}
