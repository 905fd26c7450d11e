/*
 * moraine_b200 — C ABI of the B200 (sm_100a) distributed-scatterer chain.
 *
 * Every entry point takes DEVICE pointers to caller-allocated buffers, plain sizes and
 * a CUDA stream (cudaStream_t passed as void*; NULL = legacy default stream). Work is
 * enqueued on that stream and nothing synchronises the host, except where a function
 * says so. Return value: MR_OK (0) or a negative MR_ERR_* code; mr_last_error() gives
 * the message of the calling thread's last failure.
 *
 * Array layouts are those of the Python functions each entry point replaces (C order,
 * numpy complex64 = interleaved float re, im):
 *   rslc / rmli   (nlines, width, nimages)
 *   p / dist      (nlines, width, az_win, r_win)         float32
 *   is_shp        (nlines, width, az_win, r_win)         uint8 (numpy bool)
 *   shp_num       (nlines, width)                        int32
 *   idx           (n_pc, 2) int32, columns (azimuth, range)
 *   pc_is_shp     (n_pc, az_win, r_win)                  uint8
 *   coh           (n_pc, n_pairs) complex64, pairs in image_pairs order; image_pairs
 *                 NULL means all pairs m < j in row-major upper-triangle order
 *                 (numpy.triu_indices(nimages, 1)), n_pairs = nimages*(nimages-1)/2
 *   ph            (n_pc, nimages) complex64
 *
 * Reference interfaces cited as path:line inside the kanglcn/moraine source tree.
 */
#ifndef MORAINE_B200_H
#define MORAINE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* mr_stream_t; /* cudaStream_t */

typedef struct {
  float re, im;
} mr_complex64;

enum {
  MR_OK = 0,
  MR_ERR_INVALID = -1,     /* bad shape, size or argument */
  MR_ERR_CUDA = -2,        /* a CUDA launch or API call failed */
  MR_ERR_UNSUPPORTED = -3, /* valid request outside this build's limits */
  MR_ERR_WORKSPACE = -4,   /* workspace missing or too small */
};

/* Arithmetic of the coherence Gram and of EMI. */
enum {
  MR_PREC_FP32 = 0,   /* FP32 SIMT Gram; FP32 EMI reduction */
  MR_PREC_BF16 = 1,   /* BF16 tensor-core Gram, FP32 accumulate */
  MR_PREC_BF16X3 = 2, /* BF16 hi/lo split tensor-core Gram (3 products) */
  MR_PREC_FP64 = 3,   /* FP64 Gram; FP64 EMI */
  MR_PREC_MIXED = 4,  /* EMI only: FP32, with points whose cond_1(|Gamma|) estimate exceeds
                         the threshold (or that are singular in FP32) redone in FP64 */
  MR_PREC_REFINE = 5, /* EMI only: inv(|Gamma|) in FP64, the Householder reduction in FP32,
                         the eigenvector refined by one FP64 Newton step through the FP32
                         factors, then checked in FP64; points whose phase error bound exceeds
                         the tolerance (MR_EMI_REFINE_TOL) are redone in FP64 */
};

/* What the whole chain feeds the KS test (the test depends only on ranks, but the two
 * roundings make different ties, so the mask follows the choice bit for bit). */
enum {
  MR_KS_INTENSITY = 0, /* |z|^2 (mr_intensity): the rmli of the reference's API notebooks */
  MR_KS_AMPLITUDE = 1, /* |z| (mr_rslc2amp): moraine/cli/shp.py:98, rslc2amp before ks_test */
};

/* Condition threshold of MR_PREC_MIXED in mr_emi. */
#define MR_EMI_COND_MAX 1.0e4
/* Phase error bound (rad) under which MR_PREC_REFINE keeps a refined point in mr_emi. */
#define MR_EMI_REFINE_TOL 1.0e-4

/* Limits of this build. */
#define MR_MAX_NIMAGES 512
#define MR_MAX_WINDOW 4096 /* az_win * r_win */

const char* mr_last_error(void);

/* Number of kernels the library has launched in this process (all devices, all
 * streams), for accounting by benchmarks and tests. No reference counterpart. */
uint64_t mr_kernel_launches(void);
int mr_abi_version(void);

/* Per-kernel device time, for benchmarks. mr_set_kernel_timing(1) clears the totals and
 * starts recording a CUDA event pair around every launch of the chain's main kernels (KS,
 * coherence, EMI) on the launch's stream; (0) stops. mr_kernel_timing synchronises the
 * recorded events, returns the number of kernels seen and, for 0 <= i < that number, gives
 * kernel i's name, total milliseconds and launch count. Timing adds an event pair per launch,
 * so time a separate pass with it, not the headline one. No reference counterpart. */
void mr_set_kernel_timing(int on);
int mr_kernel_timing(int i, const char** name, double* total_ms, int64_t* launches);

/* ---------------------------------------------------------------- intensity prologue
 * rmli = re*re + im*im (float32, each product and the sum rounded once): the |slc|^2
 * that the notebooks feed to ks_test (nbs/API/pl.ipynb cell 15, `np.abs(rslc)**2`),
 * written without a fused multiply-add. */
int mr_intensity(const mr_complex64* rslc, int64_t n, float* rmli, mr_stream_t stream);

/* ---------------------------------------------------------------- SHP identification
 * Replaces moraine.shp.ks_test (moraine/shp.py:269-305) and, when is_shp / shp_num are
 * given, moraine.shp.select_shp (moraine/shp.py:309-323) in the same pass.
 * Two-sample KS test of every pixel against every pixel of its
 * (2*az_half_win+1) x (2*r_half_win+1) window. The statistic is the exact integer
 * k = max |j2 - j1| of the reference merge (moraine/shp.py:36-44); p and dist are
 * float32 lookups of k through the reference formula evaluated on the host in double
 * precision (moraine/shp.py:20-32, 74-76), so they equal the reference CPU path bit for
 * bit; is_shp = (double)p < p_max and shp_num counts it. NaN (and is_shp = 0) where the
 * neighbour is outside the image or either pixel holds a NaN.
 * Any of p, dist, is_shp, shp_num may be NULL (is_shp and shp_num go together).
 * workspace: >= mr_ks_workspace_bytes(), 16-byte aligned. */
size_t mr_ks_workspace_bytes(int nlines, int width, int nimages);
int mr_ks_test(const float* rmli, int nlines, int width, int nimages, int az_half_win,
               int r_half_win, float* p, float* dist, double p_max, uint8_t* is_shp,
               int32_t* shp_num, void* workspace, size_t workspace_bytes, mr_stream_t stream);

/* Replaces moraine.shp.select_shp (moraine/shp.py:309-323): is_shp = p < p_max (p
 * widened to double; NaN gives 0), shp_num = per-pixel count. */
/* Tile plans of the KS merge: with autotuning on (off by default), the first mr_ks_test for a
 * (device, nimages, window, raster size within a factor of 4) times the plans for several
 * shared-memory budgets on its own input, three times each (synchronising the stream; never
 * inside a stream capture), and keeps the one with the fastest median; results do not depend
 * on the plan. Timings are most reliable when nothing else runs on the device, e.g. in a
 * first call before a server starts its slots. mr_ks_plan reports the plan in use (for the
 * largest raster size tuned so far). No reference counterpart (the reference kernel has no
 * tiles). */
void mr_set_autotune(int on);
int mr_ks_plan(int nimages, int az_half_win, int r_half_win, int* tile_rows, int* tile_cols,
               int* az_chunk);

int mr_select_shp(const float* p, int64_t npix, int win, double p_max, uint8_t* is_shp,
                  int32_t* shp_num, mr_stream_t stream);

/* ---------------------------------------------------------------- DS candidates
 * The glue the reference notebooks write between select_shp and emperical_co_pc
 * (nbs/API/pl.ipynb cell 15: is_ds_can = shp_num >= 50; idx = stack(where(is_ds_can));
 * pc_is_shp = is_shp[is_ds_can]), and the CLI's pc_logic_ras / ras2pc_ras_chunk
 * (moraine/cli/pc.py:764, :239). Writes, in row-major pixel order, idx (n, 2) and,
 * unless NULL, pc_is_shp (n, win); *n_ds (device int64) receives n. At most max_ds
 * entries are written (n itself is always the full count).
 * workspace: >= mr_ds_extract_workspace_bytes(). */
size_t mr_ds_extract_workspace_bytes(int64_t npix);
int mr_ds_extract(const int32_t* shp_num, const uint8_t* is_shp, int nlines, int width,
                  int win, int min_shp, int32_t* idx, uint8_t* pc_is_shp, int64_t max_ds,
                  int64_t* n_ds, void* workspace, size_t workspace_bytes, mr_stream_t stream);

/* Allocation-free variant of mr_ds_extract. This entry point has no counterpart in the
 * reference; it exists for callers that cannot provide device workspace memory (a host
 * that plans every device byte up front, a plugin that must not bypass its host
 * framework's allocator, a binding with no route to a device allocator). Same arguments
 * and results as mr_ds_extract without the workspace: the per-block counts live in a
 * fixed array inside the library (128 KiB per device, held until the process exits), so
 * rasters are limited to MR_DS_EXTRACT_NOALLOC_MAX_PIXELS pixels (larger ones return
 * MR_ERR_UNSUPPORTED). It calls no allocator. The first call in a CUDA context looks up
 * that array's device address (cudaGetSymbolAddress) and keeps it with the context's ID
 * (a context created again after cudaDeviceReset gets a new lookup); make that first call
 * before any stream capture. Every call shares the one array: calls that overlap on the
 * GPU (other streams, other host threads) race on it, so serialise them. */
#define MR_DS_EXTRACT_NOALLOC_MAX_PIXELS (16384LL * 1024LL)
int mr_ds_extract_noalloc(const int32_t* shp_num, const uint8_t* is_shp, int nlines, int width,
                          int win, int min_shp, int32_t* idx, uint8_t* pc_is_shp, int64_t max_ds,
                          int64_t* n_ds, mr_stream_t stream);

/* ---------------------------------------------------------------- coherence
 * Replaces moraine.co.emperical_co_pc (moraine/co.py:230-266; kernel :141-190, CPU
 * :194-227): coh[i, q] = sum_s z_m conj(z_j) / sqrt(sum_s |z_m|^2 * sum_s |z_j|^2) over
 * the SHPs s of point i that lie inside the image, (m, j) = image_pairs[q].
 * mask_stride selects where each point's window mask lives: mask_stride == 0 reads
 * pc_is_shp (n_pc, az_win, r_win); mask_stride == 1 reads a raster is_shp
 * (nlines, width, az_win, r_win) at the point's own pixel (the chain's layout).
 * precision: MR_PREC_FP32, MR_PREC_BF16, MR_PREC_BF16X3 or MR_PREC_FP64 (custom
 * image_pairs: FP32 only). */
int mr_emperical_co_pc(const mr_complex64* rslc, int nlines, int width, int nimages,
                       const int32_t* idx, int64_t n_pc, const uint8_t* mask, int mask_stride,
                       int az_win, int r_win, const int32_t* image_pairs, int n_pairs,
                       mr_complex64* coh, int precision, mr_stream_t stream);

/* Replaces moraine.co.emperical_co (moraine/co.py:117-137; kernel :61-114): full
 * (nlines, width, nimages, nimages) covariance cov = sum/n_shp and coherence. */
int mr_emperical_co(const mr_complex64* rslc, int nlines, int width, int nimages,
                    const uint8_t* is_shp, int az_win, int r_win, mr_complex64* cov,
                    mr_complex64* coh, mr_stream_t stream);

/* Replaces moraine.co.ad_intf_pc (moraine/co.py:376-406; GPU kernel :334-374): adaptive
 * multilook interferogram of one pair for point-cloud data, intf = sum ref conj(sec) /
 * sqrt(sum |ref|^2 sum |sec|^2) over each point's SHPs (pc_is_shp (n_pc, az_win, r_win)).
 * Equal to pair (0, 1) of mr_emperical_co_pc on the stack (ref, sec, ...), as the
 * reference's own test requires (nbs/API/co.ipynb#cell46). precision: MR_PREC_FP32
 * (the reference GPU kernel's accumulation) or MR_PREC_FP64. workspace: >=
 * mr_ad_intf_pc_workspace_bytes() (the two images interleaved). */
size_t mr_ad_intf_pc_workspace_bytes(int nlines, int width);
int mr_ad_intf_pc(const mr_complex64* ref_rslc, const mr_complex64* sec_rslc, int nlines, int width,
                  const int32_t* idx, int64_t n_pc, const uint8_t* pc_is_shp, int az_win, int r_win,
                  mr_complex64* intf, int precision, void* workspace, size_t workspace_bytes,
                  mr_stream_t stream);

/* Replaces moraine.co.uncompress_coh (moraine/co.py:281-299): (n, n_pairs) ->
 * (n, nimages, nimages) Hermitian, zero where no pair is given, unit diagonal. */
int mr_uncompress_coh(const mr_complex64* coh, int64_t n, int nimages,
                      const int32_t* image_pairs, int n_pairs, mr_complex64* out,
                      mr_stream_t stream);

/* ---------------------------------------------------------------- PS-side statistics */
/* Replaces moraine.calamp.rslc2amp (moraine/calamp.py:33-41): amp = |rslc| (float32, as
 * numpy's complex64 abs), any shape flattened to n samples. */
int mr_rslc2amp(const mr_complex64* rslc, int64_t n, float* amp, mr_stream_t stream);

/* Replaces moraine.ps.amp_disp (moraine/ps.py:65-73): per pixel of a (npix, nimages)
 * complex64 stack, std(|z|) / mean(|z|) over the dates (population std), float32. */
int mr_amp_disp(const mr_complex64* rslc, int64_t npix, int nimages, float* amp_disp,
                mr_stream_t stream);

/* Replaces moraine.calamp.calamp (moraine/calamp.py:63-71): amp / nanmean(amp) over the n
 * samples of one image. workspace: >= mr_calamp_workspace_bytes(). */
size_t mr_calamp_workspace_bytes(void);
int mr_calamp(const float* amp, int64_t n, float* out, void* workspace, size_t workspace_bytes,
              mr_stream_t stream);

/* ---------------------------------------------------------------- GAMMA ingest
 * Sample types of GAMMA rasters (moraine/gamma_.py:24-31: float, fcomplex, int, double). */
enum {
  MR_GAMMA_FLOAT = 0,    /* big-endian float32 */
  MR_GAMMA_FCOMPLEX = 1, /* big-endian complex64 (real, imaginary) */
  MR_GAMMA_INT = 2,      /* big-endian int32 */
  MR_GAMMA_DOUBLE = 3,   /* big-endian float64 */
};

/* Bytes per sample of a GAMMA dtype (0 for an unknown one). */
size_t mr_gamma_sample_bytes(int dtype);

/* Replaces the decode step of moraine.gamma_.read_gamma_image / read_gamma_pdata
 * (moraine/gamma_.py:46-56, :75-84): n big-endian samples at `be` (device memory, the
 * file's bytes as read) to native samples at out[i * out_stride], |x| < 1e-30 -> NaN
 * (NaN + NaN j for fcomplex; int unchanged). Both buffers aligned to the sample size. */
int mr_gamma_decode(const void* be, int64_t n, int dtype, void* out, int64_t out_stride,
                    mr_stream_t stream);

/* ---------------------------------------------------------------- phase linking
 * Replaces moraine.pl.emi (moraine/pl.py:68-77; GPU :19-42, CPU :46-65): for every
 * point, M = inv(|Gamma|) o Gamma from the full-triangle compressed coherence, its
 * algebraically smallest eigenpair (lambda, v), ph = v conj(v[ref]) / |v conj(v[ref])|,
 * emi_quality = lambda. inv(|Gamma|) by Gauss-Jordan with partial pivoting; eigenpair by
 * Householder tridiagonalisation, Sturm multisection and inverse iteration; all in the
 * arithmetic given by precision: MR_PREC_FP32, MR_PREC_FP64, MR_PREC_MIXED (FP32, and
 * FP64 for the points whose cond_1(|Gamma|) estimate exceeds MR_EMI_COND_MAX) or
 * MR_PREC_REFINE (see mr_emi_refined, tolerance MR_EMI_REFINE_TOL); FP64 throughout when
 * nimages > 128. t_coh (may be NULL) receives moraine.pl.ds_temp_coh of
 * the result (moraine/pl.py:126) computed in the same pass. Points whose |Gamma| is
 * singular at the arithmetic used get NaN (the reference's inv raises on them).
 * workspace: >= mr_emi_workspace_bytes() (the same for every precision). */
size_t mr_emi_workspace_bytes(int64_t n_pc, int nimages);

/* EMI for N <= 128 runs in sub-batches of points (per-point state in the workspace, at most
 * 4 GiB of it by default: about 34,600 points at N = 100). mr_set_emi_sub_batch(m) caps a
 * sub-batch at m points (0 restores the default; negative: MR_ERR_INVALID), which lowers
 * mr_emi_workspace_bytes for later calls; a workspace sized before a larger cap was set is
 * rejected (MR_ERR_WORKSPACE). Process-wide. No reference counterpart. */
int mr_set_emi_sub_batch(int64_t max_points);
int mr_emi(const mr_complex64* coh, int64_t n_pc, int nimages, int ref, int precision,
           mr_complex64* ph, float* emi_quality, float* t_coh, void* workspace,
           size_t workspace_bytes, mr_stream_t stream);

/* mr_emi with MR_PREC_MIXED and a caller-chosen threshold cond_max (> 0). Every point is
 * computed in FP32, cond_1(|Gamma|) = |A|_1 |inv(A)|_1 (A = |Gamma|) is evaluated from the
 * FP32 inverse, and the points above cond_max or singular in FP32 are recomputed in FP64.
 * route (may be NULL, n_pc bytes) receives per point 0 = FP32, 1 = FP64 (condition),
 * 2 = FP64 (singular in FP32); 1 for every point when nimages > 128 (FP64 throughout).
 * Same computation as moraine.pl.emi (moraine/pl.py:68-77); the routing has no reference
 * counterpart (the reference runs complex64 LAPACK / cuSOLVER throughout). */
int mr_emi_routed(const mr_complex64* coh, int64_t n_pc, int nimages, int ref, double cond_max,
                  mr_complex64* ph, float* emi_quality, float* t_coh, uint8_t* route,
                  void* workspace, size_t workspace_bytes, mr_stream_t stream);

/* mr_emi with MR_PREC_REFINE and a caller-chosen tolerance tol (> 0, radians). inv(|Gamma|)
 * is computed in FP64 (for N <= 128 by the symmetric sweep: diagonal pivots in natural order;
 * a point whose pivot falls below 1e-9 in magnitude is recomputed in FP64 with partial
 * pivoting) and M = inv(|Gamma|) o Gamma is reduced to tridiagonal form in FP32.
 * The FP32 eigenvector v is then improved by one Newton (Jacobi-Davidson) step in FP64:
 * r = M v - lambda v with M and lambda = v^H M v in FP64, the correction solved through the
 * FP32 factors M ~ Q T Q^H with T's own eigenvector projected out. The refined pair is
 * checked in FP64: residual r', gap g = lambda_2(T) - lambda and smallest component
 * min|v_i| bound the phase error of every date by |r'| / (g min|v_i|); points whose
 * bound exceeds tol (decided by a Sturm count of T at the shift where it would equal tol)
 * are recomputed in FP64. route (may be NULL, n_pc bytes) receives per
 * point 0 = refined, 1 = recomputed in FP64, 2 = |Gamma| singular in FP64 (NaN output);
 * 1 for every point when nimages > 128 (FP64 throughout). Same computation as
 * moraine.pl.emi (moraine/pl.py:68-77); the refinement has no reference counterpart. */
int mr_emi_refined(const mr_complex64* coh, int64_t n_pc, int nimages, int ref, double tol,
                   mr_complex64* ph, float* emi_quality, float* t_coh, uint8_t* route,
                   void* workspace, size_t workspace_bytes, mr_stream_t stream);

/* ---------------------------------------------------------------- raster <-> point cloud
 * Replace moraine.pc.ras2pc (moraine/pc.py:239-241: pc = ras[gix[:, 0], gix[:, 1]]) and
 * moraine.pc.pc2ras with a grid index (moraine/pc.py:223-236: a raster filled with NaN, then
 * ras[gix[:, 0], gix[:, 1]] = pc). A record is one pixel's trailing dimensions, elem_bytes
 * long (the raster is (nlines, width, record), the point cloud (n, record)); gix is (n, 2)
 * int32 (line, pixel) with numpy's index rules (-nlines <= line < nlines, negative from the
 * end; the same for pixels). An index outside that range sets *err (device int) to 1 and its
 * point is skipped; the caller clears *err first and reads it afterwards. pc2ras first sets
 * every record to the fill pattern (fill: fill_bytes = 4, 8 or 16 host bytes, repeated; 0 =
 * no fill), then scatters; with repeated indices one of the records lands, unspecified which. */
int mr_ras2pc(const void* ras, int64_t nlines, int64_t width, int64_t elem_bytes,
              const int32_t* gix, int64_t n, void* pc, int* err, mr_stream_t stream);
int mr_pc2ras(const void* pc, const int32_t* gix, int64_t n, int64_t nlines, int64_t width,
              int64_t elem_bytes, const void* fill, int fill_bytes, void* ras, int* err,
              mr_stream_t stream);

/* ---------------------------------------------------------------- the whole chain
 * Replaces the stage drivers moraine/cli/shp.py:33 (ks_test, select_shp), the DS selection
 * of nbs/API/pl.ipynb#cell15, moraine/cli/co.py:33 (emperical_co_pc) and
 * moraine/cli/pl.py:223 (emi, ds_temp_coh) for one tile in device memory:
 * KS input (ks_input: MR_KS_INTENSITY or MR_KS_AMPLITUDE) -> KS test + SHP selection
 * (window (2 az_half_win + 1) x (2 r_half_win + 1), p < p_max) -> DS points (SHP count
 * >= min_shp, row-major order) -> per batch of at most `batch` points: coherence
 * (gram_precision) -> EMI with temporal coherence (emi_precision: MR_PREC_FP32,
 * MR_PREC_FP64, MR_PREC_MIXED or MR_PREC_REFINE). Outputs for the first *n_ds points: idx
 * (max_ds, 2), ph (max_ds, nimages), quality and t_coh (max_ds). *n_ds is a host pointer:
 * the call synchronises `stream` once to read the DS count (fails with MR_ERR_INVALID when
 * it exceeds max_ds). workspace: >= mr_ds_chain_workspace_bytes(), 256-byte aligned. */
size_t mr_ds_chain_workspace_bytes(int nlines, int width, int nimages, int az_half_win,
                                   int r_half_win, int64_t batch);
int mr_ds_chain(const mr_complex64* rslc, int nlines, int width, int nimages, int az_half_win,
                int r_half_win, int ks_input, double p_max, int min_shp, int gram_precision,
                int emi_precision, int32_t* idx, mr_complex64* ph, float* quality, float* t_coh, int64_t max_ds,
                int64_t* n_ds, int64_t batch, void* workspace, size_t workspace_bytes,
                mr_stream_t stream);

/* mr_ds_chain without the host synchronisation, for capture in a CUDA graph: the DS count
 * goes to n_ds_dev (device memory) and the kernels read it there, processing every batch
 * that max_ds allows (batches past the count do no work). Only stream-ordered work, no
 * allocation. Limits: nimages <= 128, gram precision MR_PREC_FP32 or MR_PREC_FP64, emi
 * precision MR_PREC_FP32, MR_PREC_FP64 or MR_PREC_REFINE (tolerance MR_EMI_REFINE_TOL).
 * Points past max_ds are not processed: compare *n_ds_dev with max_ds afterwards. Same
 * results as mr_ds_chain. No reference counterpart. */
int mr_ds_chain_async(const mr_complex64* rslc, int nlines, int width, int nimages, int az_half_win,
                      int r_half_win, int ks_input, double p_max, int min_shp, int gram_precision,
                      int emi_precision, int32_t* idx, mr_complex64* ph, float* quality, float* t_coh, int64_t max_ds,
                      int64_t* n_ds_dev, int64_t batch, void* workspace, size_t workspace_bytes,
                      mr_stream_t stream);

/* ---------------------------------------------------------------- temporal coherence
 * Replaces moraine.pl.ds_temp_coh (moraine/pl.py:126-145; kernel :104-123):
 * t = |sum_q coh_q/|coh_q| conj(ph_m) ph_j| / n_pairs. */
int mr_ds_temp_coh(const mr_complex64* coh, const mr_complex64* ph, int64_t n, int nimages,
                   const int32_t* image_pairs, int n_pairs, float* t_coh, mr_stream_t stream);

/* Replaces moraine.pqm.temp_coh (moraine/pqm.py:124-159; kernel :100-121):
 * t = |sum_q intf_q conj(r_m) r_j / sqrt(|intf_q|^2 |r_m|^2 |r_j|^2)| / n_pairs.
 * Inputs are not modified (the reference CPU path normalises them in place). */
int mr_temp_coh(const mr_complex64* intf, const mr_complex64* rslc, int64_t n, int nimages,
                const int32_t* image_pairs, int n_pairs, float* t_coh, mr_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* MORAINE_B200_H */
