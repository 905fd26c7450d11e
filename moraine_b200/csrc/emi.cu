// EMI phase linking on the GPU: host entry point and the general kernel (any N).
//
// Reference behaviour followed (kanglcn/moraine):
//   moraine/pl.py:34-41, 56-64  Gamma = uncompress(coh); M = inv(|Gamma|) o Gamma;
//                               (lambda, v) = eigh(M)[0]  (algebraically smallest);
//                               ph = v conj(v[ref]) / |v conj(v[ref])|; quality = lambda
//   moraine/tnet.py:123-130     N from the number of pairs (all pairs m < j)
//   moraine/pl.py:112-120       temporal coherence of the result (fused epilogue)
//
// |Gamma| is frequently indefinite when a point has fewer SHPs than images, so M is then
// indefinite too and its smallest eigenvalue is large and negative. The algorithm is
// therefore valid for any Hermitian M:
//   1. inv(|Gamma|) by Gauss-Jordan elimination with partial pivoting;
//   2. M = inv(|Gamma|) o Gamma;
//   3. Householder reduction M = Q T Q^H, T Hermitian tridiagonal, then a diagonal unitary
//      scaling T = D R D^H with R real symmetric tridiagonal;
//   4. lambda_min(R) by Sturm-count multisection on one warp;
//   5. its eigenvector y by inverse iteration on R - lambda I (pivoted tridiagonal LU);
//   6. v = Q D y.
// All arithmetic is FP64.
//
// Two implementations: for N <= 128 the two-kernel path of emi_fast.cu (FP64 inverse in
// registers, then M reduced in shared memory in FP32 or FP64 as requested); for larger N
// the kernel below (FP64 throughout), whose N x N working matrices live in a per-CTA
// slice of a global workspace.
#include <algorithm>
#include <atomic>

#include "emi_common.cuh"

namespace mr {
namespace emi {

// emi_fast.cu
extern std::atomic<int64_t> g_sub_batch_cap;
int fast_supported(int n);
size_t fast_workspace_bytes(int64_t n_pc, int n);
int fast_run(const float2* coh, int64_t n_pc, int n, int ref, int precision, float cond_max, float2* ph,
             float* quality, float* tcoh, uint8_t* route, void* workspace, cudaStream_t s,
             const int64_t* dcount = nullptr, int64_t doff = 0);

namespace {

// argmax of |x| over the block (ties -> smaller index); idx < 0 means "no candidate".
__device__ int block_argmax(double x, int idx, Red& r) {
  double ax = idx >= 0 ? fabs(x) : -1.0;
  int bi = idx;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double oa = __shfl_xor_sync(0xffffffffu, ax, o);
    int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (oa > ax || (oa == ax && oi >= 0 && (bi < 0 || oi < bi))) { ax = oa; bi = oi; }
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) { r.v[threadIdx.x >> 5] = ax; r.i[threadIdx.x >> 5] = bi; }
  __syncthreads();
  ax = r.v[0];
  bi = r.i[0];
#pragma unroll
  for (int k = 1; k < kWarps; ++k)
    if (r.v[k] > ax || (r.v[k] == ax && r.i[k] >= 0 && (bi < 0 || r.i[k] < bi))) { ax = r.v[k]; bi = r.i[k]; }
  return bi;
}

// Doubles of workspace per CTA: M (complex, n*n) then |Gamma| (real, n*n), rounded to an
// even count so that every CTA's complex matrix starts on a 16-byte boundary.
__host__ __device__ __forceinline__ size_t general_slice(int n) { return ((size_t)3 * n * n + 1) & ~(size_t)1; }

struct GeneralShared {
  double2 u[MR_MAX_NIMAGES];
  double2 pw[MR_MAX_NIMAGES];
  double2 z[MR_MAX_NIMAGES];
  double2 e[MR_MAX_NIMAGES];
  double2 phs[MR_MAX_NIMAGES];
  double d[MR_MAX_NIMAGES];
  double b[MR_MAX_NIMAGES];
  double b2[MR_MAX_NIMAGES];
  double tau[MR_MAX_NIMAGES];
  double y[MR_MAX_NIMAGES];
  double w1[MR_MAX_NIMAGES];
  double w2[MR_MAX_NIMAGES];
  double w3[MR_MAX_NIMAGES];
  int perm[MR_MAX_NIMAGES];
  Red red;
};

__global__ void __launch_bounds__(kThreads) general_kernel(const float2* __restrict__ coh, int64_t n_pc, int n,
                                                           int ref, float2* __restrict__ ph,
                                                           float* __restrict__ quality, float* __restrict__ tcoh,
                                                           double* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GeneralShared& sh = *reinterpret_cast<GeneralShared*>(smem_raw);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const int nn = n * n;
  double2* M = reinterpret_cast<double2*>(work + (size_t)blockIdx.x * general_slice(n));  // 16-byte aligned
  double* A = work + (size_t)blockIdx.x * general_slice(n) + 2 * (size_t)nn;

  for (int64_t pt = blockIdx.x; pt < n_pc; pt += gridDim.x) {
    const float2* c = coh + pt * npairs;
    // 1. Gamma and |Gamma|
    for (int e = tid; e < nn; e += nt) {
      const int i = e / n, j = e - i * n;
      double2 g;
      if (i == j) g = make_double2(1.0, 0.0);
      else if (i < j) { float2 v = c[triu_index(i, j, n)]; g = make_double2(v.x, v.y); }
      else { float2 v = c[triu_index(j, i, n)]; g = make_double2(v.x, -v.y); }
      M[e] = g;
      A[e] = sqrt(g.x * g.x + g.y * g.y);
    }
    if (tid == 0) sh.red.flag = 0;
    __syncthreads();
    // 2. Gauss-Jordan inverse of A with partial pivoting (in place)
    for (int k = 0; k < n; ++k) {
      int cand = -1;
      double cv = 0.0;
      for (int i = k + tid; i < n; i += nt) {
        double v = A[i * n + k];
        if (cand < 0 || fabs(v) > fabs(cv)) { cand = i; cv = v; }
      }
      const int p = block_argmax(cv, cand, sh.red);
      if (tid == 0) sh.perm[k] = p;
      if (p != k)
        for (int j = tid; j < n; j += nt) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
      __syncthreads();
      double piv = A[k * n + k];
      if (piv == 0.0) { if (tid == 0) sh.red.flag = 1; piv = DBL_MIN; }
      const double rp = 1.0 / piv;
      for (int j = tid; j < n; j += nt) {
        sh.w1[j] = (j == k) ? rp : A[k * n + j] * rp;  // scaled pivot row
        sh.w2[j] = A[j * n + k];                       // column k (factors)
      }
      __syncthreads();
      for (int e = tid; e < nn; e += nt) {
        const int i = e / n, j = e - i * n;
        if (i == k) A[e] = sh.w1[j];
        else A[e] = ((j == k) ? 0.0 : A[e]) - sh.w2[i] * sh.w1[j];
      }
      __syncthreads();
    }
    for (int k = n - 1; k >= 0; --k) {
      const int p = sh.perm[k];
      if (p != k)
        for (int i = tid; i < n; i += nt) { double t = A[i * n + k]; A[i * n + k] = A[i * n + p]; A[i * n + p] = t; }
      __syncthreads();
    }
    // 3. M = inv(|Gamma|) o Gamma
    for (int e = tid; e < nn; e += nt) { double2 g = M[e]; double a = A[e]; M[e] = make_double2(a * g.x, a * g.y); }
    __syncthreads();
    // 4. Householder tridiagonalisation (full Hermitian storage)
    for (int k = 0; k + 2 < n; ++k) {
      const int m = n - k - 1;
      double xn2 = 0.0;
      for (int i = 1 + tid; i < m; i += nt) { double2 x = M[(k + 1 + i) * n + k]; xn2 += x.x * x.x + x.y * x.y; }
      xn2 = block_sum(xn2, sh.red);
      const double2 alpha = M[(k + 1) * n + k];
      if (xn2 == 0.0) {
        if (tid == 0) { sh.e[k] = alpha; sh.tau[k] = 0.0; }
        __syncthreads();
        continue;
      }
      const double aa = sqrt(alpha.x * alpha.x + alpha.y * alpha.y);
      const double nrm = sqrt(aa * aa + xn2);
      const double2 phs = aa > 0.0 ? make_double2(alpha.x / aa, alpha.y / aa) : make_double2(1.0, 0.0);
      const double tau = 2.0 / ((aa + nrm) * (aa + nrm) + xn2);
      for (int i = tid; i < m; i += nt)
        sh.u[i] = (i == 0) ? make_double2(phs.x * (aa + nrm), phs.y * (aa + nrm)) : M[(k + 1 + i) * n + k];
      if (tid == 0) { sh.e[k] = make_double2(-phs.x * nrm, -phs.y * nrm); sh.tau[k] = tau; }
      __syncthreads();
      const int lane = tid & 31, wid = tid >> 5;
      for (int i = wid; i < m; i += kWarps) {  // p = tau * M22 u, one warp per row
        const double2* row = M + (size_t)(k + 1 + i) * n + (k + 1);
        double sx = 0.0, sy = 0.0;
        for (int j = lane; j < m; j += 32) {
          const double2 a = row[j], uj = sh.u[j];
          sx += a.x * uj.x - a.y * uj.y;
          sy += a.x * uj.y + a.y * uj.x;
        }
        sx = warp_sum(sx);
        sy = warp_sum(sy);
        if (lane == 0) sh.pw[i] = make_double2(tau * sx, tau * sy);
      }
      __syncthreads();
      double kp = 0.0;  // Re(u^H p)
      for (int i = tid; i < m; i += nt) { double2 ui = sh.u[i], pi = sh.pw[i]; kp += ui.x * pi.x + ui.y * pi.y; }
      kp = 0.5 * tau * block_sum(kp, sh.red);
      for (int i = tid; i < m; i += nt) {
        const double2 ui = sh.u[i], pi = sh.pw[i];
        sh.pw[i] = make_double2(pi.x - kp * ui.x, pi.y - kp * ui.y);
      }
      __syncthreads();
      for (int e = tid; e < m * m; e += nt) {  // M22 -= u w^H + w u^H
        const int i = e / m, j = e - i * m;
        const double2 ui = sh.u[i], uj = sh.u[j], wi = sh.pw[i], wj = sh.pw[j];
        double2* a = M + (size_t)(k + 1 + i) * n + (k + 1 + j);
        double2 v = *a;
        v.x -= ui.x * wj.x + ui.y * wj.y + wi.x * uj.x + wi.y * uj.y;
        v.y -= ui.y * wj.x - ui.x * wj.y + wi.y * uj.x - wi.x * uj.y;
        *a = v;
      }
      for (int i = tid; i < m; i += nt) M[(k + 1 + i) * n + k] = sh.u[i];  // keep the reflector
      __syncthreads();
    }
    for (int i = tid; i < n; i += nt) sh.d[i] = M[i * n + i].x;
    if (tid == 0) sh.e[n - 2] = M[(n - 1) * n + (n - 2)];
    __syncthreads();
    TailVecs<double> tv{sh.d, sh.e, sh.tau, sh.b, sh.b2, sh.y, sh.w1, sh.w2, sh.w3, sh.z, sh.phs};
    auto uk = [&](int k, int i) { return M[(size_t)(k + 1 + i) * n + k]; };
    tail<double>(n, ref, tv, uk, sh.red, sh.red.flag != 0, ph + pt * n, quality + pt, tcoh ? tcoh + pt : nullptr, c, npairs);
  }
}

int general_grid(int64_t n_pc) { return (int)std::min<int64_t>(n_pc, (int64_t)sm_count() * 2); }

size_t general_workspace_bytes(int64_t n_pc, int n) {
  return (size_t)general_grid(n_pc) * general_slice(n) * sizeof(double);
}

}  // namespace
}  // namespace emi
}  // namespace mr

using namespace mr;
using namespace mr::emi;

extern "C" int mr_set_emi_sub_batch(int64_t max_points) {
  if (max_points < 0) return fail(MR_ERR_INVALID, "set_emi_sub_batch: max_points %lld < 0", (long long)max_points);
  mr::emi::g_sub_batch_cap.store(max_points);
  return MR_OK;
}

extern "C" size_t mr_emi_workspace_bytes(int64_t n_pc, int nimages) {
  if (n_pc <= 0 || nimages <= 0) return 16;
  if (fast_supported(nimages)) return fast_workspace_bytes(n_pc, nimages);
  return general_workspace_bytes(n_pc, nimages);
}

namespace {

int emi_entry(const mr_complex64* coh, int64_t n_pc, int nimages, int ref, int precision, double cond_max,
              mr_complex64* ph, float* emi_quality, float* t_coh, uint8_t* route, void* workspace,
              size_t workspace_bytes, mr_stream_t stream) {
  MR_REQUIRE(nimages >= 2, "emi: nimages must be >= 2 (got %d)", nimages);
  if (nimages > MR_MAX_NIMAGES) return fail(MR_ERR_UNSUPPORTED, "emi: nimages %d > %d", nimages, MR_MAX_NIMAGES);
  MR_REQUIRE(ref >= 0 && ref < nimages, "emi: ref %d out of range [0, %d)", ref, nimages);
  MR_REQUIRE(n_pc >= 0, "emi: negative n_pc");
  MR_REQUIRE(precision == MR_PREC_FP32 || precision == MR_PREC_FP64 || precision == MR_PREC_MIXED ||
                 precision == MR_PREC_REFINE,
             "emi: precision must be FP32, FP64, MIXED or REFINE");
  MR_REQUIRE(cond_max > 0, "emi: cond_max (or the refinement tolerance) must be positive");
  if (n_pc == 0) return MR_OK;
  MR_REQUIRE(coh && ph && emi_quality, "emi: NULL pointer");
  const size_t need = mr_emi_workspace_bytes(n_pc, nimages);
  if (!workspace || workspace_bytes < need)
    return fail(MR_ERR_WORKSPACE, "emi: workspace %zu < %zu bytes", workspace_bytes, need);
  MR_REQUIRE(((uintptr_t)workspace & 15) == 0, "emi: workspace not 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  auto* c = reinterpret_cast<const float2*>(coh);
  auto* p = reinterpret_cast<float2*>(ph);
  if (fast_supported(nimages))
    return fast_run(c, n_pc, nimages, ref, precision, (float)std::min(cond_max, 3.0e38), p, emi_quality, t_coh,
                    route, workspace, s);
  // N > 128: FP64 throughout
  const size_t smem = sizeof(GeneralShared);
  if (int rc_ = allow_smem(reinterpret_cast<const void*>(general_kernel), (size_t)(smem))) return rc_;
  KernelTimer kt("emi general fp64", s);
  general_kernel<<<general_grid(n_pc), kThreads, smem, s>>>(c, n_pc, nimages, ref, p, emi_quality, t_coh,
                                                            static_cast<double*>(workspace));
  if (int rc = check_launch("emi")) return rc;
  if (route) MR_CUDA_TRY(cudaMemsetAsync(route, 1, (size_t)n_pc, s));
  return MR_OK;
}

}  // namespace

extern "C" int mr_emi(const mr_complex64* coh, int64_t n_pc, int nimages, int ref, int precision,
                      mr_complex64* ph, float* emi_quality, float* t_coh, void* workspace, size_t workspace_bytes,
                      mr_stream_t stream) {
  return emi_entry(coh, n_pc, nimages, ref, precision,
                   precision == MR_PREC_REFINE ? MR_EMI_REFINE_TOL : MR_EMI_COND_MAX, ph, emi_quality, t_coh,
                   nullptr, workspace, workspace_bytes, stream);
}

extern "C" int mr_emi_refined(const mr_complex64* coh, int64_t n_pc, int nimages, int ref, double tol,
                              mr_complex64* ph, float* emi_quality, float* t_coh, uint8_t* route, void* workspace,
                              size_t workspace_bytes, mr_stream_t stream) {
  return emi_entry(coh, n_pc, nimages, ref, MR_PREC_REFINE, tol, ph, emi_quality, t_coh, route, workspace,
                   workspace_bytes, stream);
}

extern "C" int mr_emi_routed(const mr_complex64* coh, int64_t n_pc, int nimages, int ref, double cond_max,
                             mr_complex64* ph, float* emi_quality, float* t_coh, uint8_t* route, void* workspace,
                             size_t workspace_bytes, mr_stream_t stream) {
  return emi_entry(coh, n_pc, nimages, ref, MR_PREC_MIXED, cond_max, ph, emi_quality, t_coh, route, workspace,
                   workspace_bytes, stream);
}

namespace mr {
int emi_counted(const float2* coh, int64_t n_max, const int64_t* dcount, int64_t doff, int n, int precision,
                float2* ph, float* quality, float* tcoh, void* workspace, size_t workspace_bytes, cudaStream_t s) {
  if (n_max <= 0) return MR_OK;
  if (!emi::fast_supported(n)) return fail(MR_ERR_UNSUPPORTED, "emi: device-counted points need nimages <= 128");
  if (precision != MR_PREC_FP32 && precision != MR_PREC_FP64 && precision != MR_PREC_REFINE)
    return fail(MR_ERR_UNSUPPORTED, "emi: device-counted points run in FP32, FP64 or refined");
  if (!workspace || workspace_bytes < mr_emi_workspace_bytes(n_max, n))
    return fail(MR_ERR_WORKSPACE, "emi: workspace too small");
  const float tol = precision == MR_PREC_REFINE ? (float)MR_EMI_REFINE_TOL : 0.f;  // the refinement's bound
  return emi::fast_run(coh, n_max, n, 0, precision, tol, ph, quality, tcoh, nullptr, workspace, s, dcount, doff);
}
}  // namespace mr
