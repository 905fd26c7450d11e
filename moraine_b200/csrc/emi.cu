// EMI phase linking on the GPU, one CTA per point.
//
// Reference behaviour followed (kanglcn/moraine):
//   moraine/pl.py:34-41, 56-64  Gamma = uncompress(coh); M = inv(|Gamma|) o Gamma;
//                               (lambda, v) = eigh(M)[0]  (algebraically smallest);
//                               ph = v conj(v[ref]) / |v conj(v[ref])|; quality = lambda
//   moraine/tnet.py:123-130     N from the number of pairs (all pairs m < j)
//   moraine/pl.py:112-120       temporal coherence of the result (fused epilogue)
//
// |Gamma| is frequently indefinite when a point has fewer SHPs than images, so M is then
// indefinite too and its smallest eigenvalue is large and negative. The algorithm here
// is therefore valid for any Hermitian M:
//   1. inv(|Gamma|) by Gauss-Jordan elimination with partial pivoting;
//   2. M = inv(|Gamma|) o Gamma;
//   3. Householder reduction M = Q T Q^H, T Hermitian tridiagonal, then a diagonal unitary
//      scaling T = D R D^H with R real symmetric tridiagonal;
//   4. lambda_min(R) by Sturm-count multisection on one warp;
//   5. its eigenvector y by inverse iteration on R - lambda I (pivoted tridiagonal LU);
//   6. v = Q D y.
// All arithmetic is FP64. The N x N working matrices of each CTA live in a global
// workspace slice (L2-resident for moderate N); vectors live in shared memory.
#include <algorithm>
#include <cfloat>

#include "common.cuh"

namespace mr {
namespace {

constexpr int kEmiThreads = 256;
constexpr int kWarps = kEmiThreads / 32;

struct Red {
  double v[kWarps];
  double w[kWarps];
  int i[kWarps];
};

__device__ double block_sum(double x, Red& r) {
  x = warp_sum(x);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) r.v[threadIdx.x >> 5] = x;
  __syncthreads();
  double t = 0;
#pragma unroll
  for (int k = 0; k < kWarps; ++k) t += r.v[k];
  return t;
}

__device__ double2 block_sum2(double2 x, Red& r) {
  x.x = warp_sum(x.x);
  x.y = warp_sum(x.y);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) { r.v[threadIdx.x >> 5] = x.x; r.w[threadIdx.x >> 5] = x.y; }
  __syncthreads();
  double2 t = make_double2(0, 0);
#pragma unroll
  for (int k = 0; k < kWarps; ++k) { t.x += r.v[k]; t.y += r.w[k]; }
  return t;
}

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
  ax = r.v[0]; bi = r.i[0];
#pragma unroll
  for (int k = 1; k < kWarps; ++k)
    if (r.v[k] > ax || (r.v[k] == ax && r.i[k] >= 0 && (bi < 0 || r.i[k] < bi))) { ax = r.v[k]; bi = r.i[k]; }
  return bi;
}

// Number of eigenvalues of the real symmetric tridiagonal (d, b) below sigma.
__device__ int sturm_count(const double* d, const double* b2, int n, double sigma, double pivmin) {
  int c = 0;
  double q = d[0] - sigma;
  if (fabs(q) < pivmin) q = -pivmin;
  c += (q < 0);
  for (int i = 1; i < n; ++i) {
    q = (d[i] - sigma) - b2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    c += (q < 0);
  }
  return c;
}

// Solve (R - lambda I) y = y in place (pivoted tridiagonal elimination); R given by
// diagonal d and off-diagonal b. Work arrays of length n: dd, du, dl.
__device__ void tridiag_solve(const double* d, const double* b, int n, double lambda, double tiny,
                              double* y, double* dd, double* du, double* dl) {
  for (int i = 0; i < n; ++i) {
    dd[i] = d[i] - lambda;
    if (i < n - 1) { du[i] = b[i]; dl[i] = b[i]; }
  }
  // dl[i] on exit holds the second super-diagonal of row i (0 when no interchange)
  for (int i = 0; i < n - 1; ++i) {
    const double sub = dl[i];
    if (fabs(dd[i]) >= fabs(sub)) {
      if (dd[i] == 0.0) dd[i] = tiny;
      const double f = sub / dd[i];
      dd[i + 1] -= f * du[i];
      y[i + 1] -= f * y[i];
      dl[i] = 0.0;
    } else {
      const double f = dd[i] / sub;
      dd[i] = sub;
      const double t = dd[i + 1];
      dd[i + 1] = du[i] - f * t;
      if (i < n - 2) {
        dl[i] = du[i + 1];
        du[i + 1] = -f * dl[i];
      } else {
        dl[i] = 0.0;
      }
      du[i] = t;
      const double ty = y[i];
      y[i] = y[i + 1];
      y[i + 1] = ty - f * y[i + 1];
    }
  }
  if (dd[n - 1] == 0.0) dd[n - 1] = tiny;
  y[n - 1] /= dd[n - 1];
  if (n > 1) y[n - 2] = (y[n - 2] - du[n - 2] * y[n - 1]) / dd[n - 2];
  for (int i = n - 3; i >= 0; --i) y[i] = (y[i] - du[i] * y[i + 1] - dl[i] * y[i + 2]) / dd[i];
}

struct EmiShared {
  double2 u[MR_MAX_NIMAGES];
  double2 pw[MR_MAX_NIMAGES];
  double2 z[MR_MAX_NIMAGES];
  double2 e[MR_MAX_NIMAGES];
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
  double lam;
  int singular;
};

__global__ void __launch_bounds__(kEmiThreads) emi_kernel(const float2* __restrict__ coh, int64_t n_pc,
                                                          int n, int ref, float2* __restrict__ ph,
                                                          float* __restrict__ quality,
                                                          float* __restrict__ tcoh,
                                                          double* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EmiShared& sh = *reinterpret_cast<EmiShared*>(smem_raw);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int64_t npairs = (int64_t)n * (n - 1) / 2;
  const int nn = n * n;
  double2* M = reinterpret_cast<double2*>(work + (size_t)blockIdx.x * 3 * nn);
  double* A = work + (size_t)blockIdx.x * 3 * nn + 2 * (size_t)nn;

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
    if (tid == 0) sh.singular = 0;
    __syncthreads();
    // 2. Gauss-Jordan inverse of A with partial pivoting (in place)
    for (int k = 0; k < n; ++k) {
      int cand = -1; double cv = 0.0;
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
      if (piv == 0.0) { if (tid == 0) sh.singular = 1; piv = DBL_MIN; }
      const double rp = 1.0 / piv;
      for (int j = tid; j < n; j += nt) {
        double v = (j == k) ? rp : A[k * n + j] * rp;
        sh.w1[j] = v;                          // scaled pivot row
        sh.w2[j] = A[j * n + k];               // column k (factors)
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
      for (int i = tid; i < m; i += nt) {
        double2 x = (i == 0) ? make_double2(phs.x * (aa + nrm), phs.y * (aa + nrm)) : M[(k + 1 + i) * n + k];
        sh.u[i] = x;
      }
      if (tid == 0) { sh.e[k] = make_double2(-phs.x * nrm, -phs.y * nrm); sh.tau[k] = tau; }
      __syncthreads();
      // p = tau * M22 u : one warp per row
      const int lane = tid & 31, wid = tid >> 5;
      for (int i = wid; i < m; i += kWarps) {
        const double2* row = M + (size_t)(k + 1 + i) * n + (k + 1);
        double sx = 0.0, sy = 0.0;
        for (int j = lane; j < m; j += 32) {
          double2 a = row[j], uj = sh.u[j];
          sx += a.x * uj.x - a.y * uj.y;
          sy += a.x * uj.y + a.y * uj.x;
        }
        sx = warp_sum(sx); sy = warp_sum(sy);
        if (lane == 0) sh.pw[i] = make_double2(tau * sx, tau * sy);
      }
      __syncthreads();
      double kp = 0.0;  // Re(u^H p)
      for (int i = tid; i < m; i += nt) { double2 ui = sh.u[i], pi = sh.pw[i]; kp += ui.x * pi.x + ui.y * pi.y; }
      kp = 0.5 * tau * block_sum(kp, sh.red);
      for (int i = tid; i < m; i += nt) { double2 ui = sh.u[i], pi = sh.pw[i]; sh.pw[i] = make_double2(pi.x - kp * ui.x, pi.y - kp * ui.y); }
      __syncthreads();
      // M22 -= u w^H + w u^H
      for (int e = tid; e < m * m; e += nt) {
        const int i = e / m, j = e - i * m;
        double2 ui = sh.u[i], uj = sh.u[j], wi = sh.pw[i], wj = sh.pw[j];
        double2* a = M + (size_t)(k + 1 + i) * n + (k + 1 + j);
        double2 v = *a;
        v.x -= ui.x * wj.x + ui.y * wj.y + wi.x * uj.x + wi.y * uj.y;
        v.y -= ui.y * wj.x - ui.x * wj.y + wi.y * uj.x - wi.x * uj.y;
        *a = v;
      }
      // keep the reflector for the back-transformation
      for (int i = tid; i < m; i += nt) M[(k + 1 + i) * n + k] = sh.u[i];
      __syncthreads();
    }
    for (int i = tid; i < n; i += nt) sh.d[i] = M[i * n + i].x;
    if (tid == 0 && n >= 2) { sh.e[n - 2] = M[(n - 1) * n + (n - 2)]; if (n == 2) sh.tau[0] = 0.0; }
    __syncthreads();
    // 5. real tridiagonal, phases (serial, thread 0)
    if (tid == 0) {
      double2 dl = make_double2(1.0, 0.0);
      sh.z[0] = dl;
      for (int k = 0; k + 1 < n; ++k) {
        double2 ek = sh.e[k];
        double a = sqrt(ek.x * ek.x + ek.y * ek.y);
        sh.b[k] = a;
        sh.b2[k] = a * a;
        if (a > 0.0) dl = cmul(dl, make_double2(ek.x / a, ek.y / a));
        sh.z[k + 1] = dl;  // delta
      }
    }
    __syncthreads();
    // 6. lambda_min by multisection on warp 0
    if (tid < 32) {
      double lo = DBL_MAX, hi = -DBL_MAX, tnorm = 0.0;
      for (int i = 0; i < n; ++i) {
        double r = (i > 0 ? sh.b[i - 1] : 0.0) + (i + 1 < n ? sh.b[i] : 0.0);
        lo = fmin(lo, sh.d[i] - r);
        hi = fmax(hi, sh.d[i] + r);
        tnorm = fmax(tnorm, fabs(sh.d[i]) + r);
      }
      const double pivmin = fmax(DBL_MIN, DBL_EPSILON * DBL_EPSILON * tnorm * tnorm) + DBL_MIN;
      const double pad = 2.0 * DBL_EPSILON * fmax(tnorm, DBL_MIN) + 2.0 * pivmin;
      lo -= pad; hi += pad;
      for (int it = 0; it < 64; ++it) {
        const double width = hi - lo;
        if (width <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + 4.0 * pivmin) break;
        const double sg = lo + width * (double)(tid + 1) / 33.0;
        const int cnt = sturm_count(sh.d, sh.b2, n, sg, pivmin);
        const unsigned ball = __ballot_sync(0xffffffffu, cnt >= 1);
        const int first = ball ? __ffs(ball) - 1 : 32;  // first lane with an eigenvalue below
        const double nlo = (first == 0) ? lo : lo + width * (double)first / 33.0;
        const double nhi = (first == 32) ? hi : lo + width * (double)(first + 1) / 33.0;
        lo = nlo; hi = nhi;
      }
      if (tid == 0) {
        const double lam = 0.5 * (lo + hi);
        sh.lam = lam;
        // 7. inverse iteration on R - lambda I
        for (int i = 0; i < n; ++i) sh.y[i] = 1.0 + 0.5 * sin(1.0 + 3.7 * i);
        const double tiny = DBL_EPSILON * fmax(tnorm, DBL_MIN);
        for (int it = 0; it < 3; ++it) {
          tridiag_solve(sh.d, sh.b, n, lam, tiny, sh.y, sh.w1, sh.w2, sh.w3);
          double s = 0.0;
          for (int i = 0; i < n; ++i) s = fmax(s, fabs(sh.y[i]));
          if (!(s > 0.0) || !isfinite(s)) break;
          for (int i = 0; i < n; ++i) sh.y[i] /= s;
        }
      }
    }
    __syncthreads();
    // 8. v = Q D y
    for (int i = tid; i < n; i += nt) { double2 dl = sh.z[i]; double yi = sh.y[i]; sh.z[i] = make_double2(dl.x * yi, dl.y * yi); }
    __syncthreads();
    for (int k = n - 3; k >= 0; --k) {
      const double tau = sh.tau[k];
      if (tau == 0.0) continue;
      const int m = n - k - 1;
      double2 s = make_double2(0, 0);
      for (int i = tid; i < m; i += nt) {  // u^H z
        double2 ui = M[(k + 1 + i) * n + k], zi = sh.z[k + 1 + i];
        s.x += ui.x * zi.x + ui.y * zi.y;
        s.y += ui.x * zi.y - ui.y * zi.x;
      }
      s = block_sum2(s, sh.red);
      for (int i = tid; i < m; i += nt) {
        double2 ui = M[(k + 1 + i) * n + k];
        double2 t = cmul(ui, s);
        sh.z[k + 1 + i].x -= tau * t.x;
        sh.z[k + 1 + i].y -= tau * t.y;
      }
      __syncthreads();
    }
    // 9. normalise to the reference image
    const double2 zr = sh.z[ref];
    for (int i = tid; i < n; i += nt) {
      double2 v = cmulc(sh.z[i], zr);
      double a = sqrt(v.x * v.x + v.y * v.y);
      float2 o = make_float2((float)(v.x / a), (float)(v.y / a));
      if (sh.singular) o = make_float2(__int_as_float(0x7fffffff), __int_as_float(0x7fffffff));
      ph[pt * n + i] = o;
      sh.u[i] = make_double2(o.x, o.y);
    }
    if (tid == 0) quality[pt] = sh.singular ? __int_as_float(0x7fffffff) : (float)sh.lam;
    __syncthreads();
    // 10. temporal coherence of the result
    if (tcoh) {
      double2 t = make_double2(0, 0);
      for (int64_t q = tid; q < npairs; q += nt) {
        // (m, j) of q: m from the triangular root, then fixed up
        int mm = (int)((2.0 * n - 1.0 - sqrt((2.0 * n - 1.0) * (2.0 * n - 1.0) - 8.0 * (double)q)) * 0.5);
        while (mm > 0 && triu_index(mm, mm + 1, n) > q) --mm;
        while (mm + 1 < n - 1 && triu_index(mm + 1, mm + 2, n) <= q) ++mm;
        const int jj = (int)(q - triu_index(mm, mm + 1, n)) + mm + 1;
        float2 g = c[q];
        double ga = sqrt((double)g.x * g.x + (double)g.y * g.y);
        double2 gm = make_double2(g.x / ga, g.y / ga);
        double2 pr = cmulc(sh.u[jj], sh.u[mm]);  // conj(ph_m) ph_j
        double2 v = cmul(gm, pr);
        t.x += v.x; t.y += v.y;
      }
      t = block_sum2(t, sh.red);
      if (tid == 0) tcoh[pt] = (float)(sqrt(t.x * t.x + t.y * t.y) / (double)npairs);
    }
    __syncthreads();
  }
}

int emi_grid(int64_t n_pc) { return (int)std::min<int64_t>(n_pc, (int64_t)sm_count() * 2); }

}  // namespace
}  // namespace mr

using namespace mr;

extern "C" size_t mr_emi_workspace_bytes(int64_t n_pc, int nimages) {
  if (n_pc <= 0 || nimages <= 0) return 16;
  return (size_t)emi_grid(n_pc) * 3 * (size_t)nimages * nimages * sizeof(double);
}

extern "C" int mr_emi(const mr_complex64* coh, int64_t n_pc, int nimages, int ref, mr_complex64* ph,
                      float* emi_quality, float* t_coh, void* workspace, size_t workspace_bytes,
                      mr_stream_t stream) {
  MR_REQUIRE(coh && ph && emi_quality, "emi: NULL pointer");
  MR_REQUIRE(nimages >= 2, "emi: nimages must be >= 2 (got %d)", nimages);
  if (nimages > MR_MAX_NIMAGES) return fail(MR_ERR_UNSUPPORTED, "emi: nimages %d > %d", nimages, MR_MAX_NIMAGES);
  MR_REQUIRE(ref >= 0 && ref < nimages, "emi: ref %d out of range [0, %d)", ref, nimages);
  MR_REQUIRE(n_pc >= 0, "emi: negative n_pc");
  if (n_pc == 0) return MR_OK;
  if (!workspace || workspace_bytes < mr_emi_workspace_bytes(n_pc, nimages))
    return fail(MR_ERR_WORKSPACE, "emi: workspace %zu < %zu bytes", workspace_bytes,
                mr_emi_workspace_bytes(n_pc, nimages));
  const size_t smem = sizeof(EmiShared);
  MR_CUDA_TRY(cudaFuncSetAttribute(emi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  emi_kernel<<<emi_grid(n_pc), kEmiThreads, smem, as_stream(stream)>>>(
      reinterpret_cast<const float2*>(coh), n_pc, nimages, ref, reinterpret_cast<float2*>(ph), emi_quality,
      t_coh, static_cast<double*>(workspace));
  return check_launch("emi");
}
